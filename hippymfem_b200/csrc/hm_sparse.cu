// CSR products, deterministic reductions and the Jacobi-PCG of the incremental solves.
//
// Every reduction is two-pass over a fixed grid (kReduceBlocks blocks, grid-stride),
// so its summation order depends on n alone: repeated solves are bit-identical.
// The PCG keeps alpha, beta and the residual norms on the device; the host only
// launches and, every check_every iterations, reads one flag.  After convergence the
// step length is frozen at zero, so the result is that of the exact iteration count
// whatever check_every is.
#include <cmath>

#include "hm_common.cuh"
#include "hm_internal.h"

namespace hm {

constexpr int kReduceBlocks = 1184;  // 8 x 148 SMs
constexpr int kReduceThreads = 256;

// ------------------------------------------------------------------------ SpMV
// G lanes per row (G = 8): a warp covers 4 consecutive rows, which are contiguous in
// the CSR arrays; each group reduces its row with shuffles in a fixed order.
template <int G, bool TRANS>
__global__ void __launch_bounds__(256)
    k_spmv(int64_t nrow, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
           const int32_t* __restrict__ tpos, const double* __restrict__ vals,
           const double* __restrict__ x, double* __restrict__ y, double alpha, double beta) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
  const int lane = threadIdx.x % G;
  double acc = 0.0;
  if (row < nrow) {
    const int b = indptr[row], e = indptr[row + 1];
    for (int s = b + lane; s < e; s += G) {
      const double v = TRANS ? vals[tpos[s]] : vals[s];
      acc = fma(v, __ldg(x + indices[s]), acc);
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, G);
  if (row < nrow && lane == 0) y[row] = beta == 0.0 ? alpha * acc : fma(beta, y[row], alpha * acc);
}

__global__ void k_csr_diag(int64_t nrow, const int32_t* __restrict__ indptr,
                           const double* __restrict__ vals, double* __restrict__ diag) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < nrow) diag[r] = vals[indptr[r]];
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

__global__ void __launch_bounds__(kReduceThreads)
    k_dot_partial(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                  double* __restrict__ part) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v = fma(a[i], b[i], v);
  v = block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// sum of nq interleaved partial arrays part[q * kReduceBlocks + b] -> out[q]
__global__ void k_reduce_final(const double* __restrict__ part, int nq, double* __restrict__ out) {
  __shared__ double sh[32];
  for (int q = 0; q < nq; ++q) {
    double v = 0.0;
    for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) v += part[q * kReduceBlocks + b];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) out[q] = v;
  }
}

// ----------------------------------------------------------------------- PCG
// device scalars
enum { SC_RZ = 0, SC_PQ, SC_ALPHA, SC_BETA, SC_RR, SC_BB, SC_TOL2, SC_CONV, SC_TMP0, SC_TMP1, SC_TMP2, SC_N };

// r = b - q, z = dinv r, p = z; partials of r.z, r.r, b.b
__global__ void __launch_bounds__(kReduceThreads)
    k_pcg_init(int64_t n, const double* __restrict__ b, const double* __restrict__ q,
               const double* __restrict__ dinv_src, double* __restrict__ r, double* __restrict__ z,
               double* __restrict__ p, double* __restrict__ part) {
  __shared__ double sh[32];
  double rz = 0.0, rr = 0.0, bb = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = b[i] - q[i];
    const double zi = ri / dinv_src[i];
    r[i] = ri; z[i] = zi; p[i] = zi;
    rz = fma(ri, zi, rz); rr = fma(ri, ri, rr); bb = fma(b[i], b[i], bb);
  }
  rz = block_sum(rz, sh);
  rr = block_sum(rr, sh);
  bb = block_sum(bb, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rz;
    part[kReduceBlocks + blockIdx.x] = rr;
    part[2 * kReduceBlocks + blockIdx.x] = bb;
  }
}

__global__ void k_pcg_init_final(const double* __restrict__ part, double* __restrict__ sc, double rtol) {
  __shared__ double sh[32];
  double v[3];
  for (int q = 0; q < 3; ++q) {
    double t = 0.0;
    for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) t += part[q * kReduceBlocks + b];
    v[q] = block_sum(t, sh);
  }
  if (threadIdx.x == 0) {
    sc[SC_RZ] = v[0];
    sc[SC_RR] = v[1];
    sc[SC_BB] = v[2];
    sc[SC_TOL2] = rtol * rtol;
    sc[SC_CONV] = (v[1] <= rtol * rtol * v[2]) ? 0.0 : -1.0;
  }
}

__global__ void k_pcg_alpha(const double* __restrict__ part, int64_t nparts, double* __restrict__ sc) {
  __shared__ double sh[32];
  double t = 0.0;
  for (int64_t b = threadIdx.x; b < nparts; b += blockDim.x) t += part[b];
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    sc[SC_PQ] = t;
    const double a = sc[SC_RZ] / t;
    sc[SC_ALPHA] = (sc[SC_CONV] >= 0.0 || t == 0.0 || !isfinite(a)) ? 0.0 : a;
  }
}

// x += alpha p, r -= alpha q, z = r / diag; partials of r.z and r.r
__global__ void __launch_bounds__(kReduceThreads)
    k_pcg_update(int64_t n, const double* __restrict__ sc, double* __restrict__ x,
                 double* __restrict__ r, double* __restrict__ z, const double* __restrict__ p,
                 const double* __restrict__ q, const double* __restrict__ diag,
                 double* __restrict__ part) {
  __shared__ double sh[32];
  const double alpha = sc[SC_ALPHA];
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    const double zi = ri / diag[i];
    r[i] = ri; z[i] = zi;
    rz = fma(ri, zi, rz); rr = fma(ri, ri, rr);
  }
  rz = block_sum(rz, sh);
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rz;
    part[kReduceBlocks + blockIdx.x] = rr;
  }
}

__global__ void k_pcg_beta(const double* __restrict__ part, double* __restrict__ sc, int it) {
  __shared__ double sh[32];
  double v[2];
  for (int q = 0; q < 2; ++q) {
    double t = 0.0;
    for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) t += part[q * kReduceBlocks + b];
    v[q] = block_sum(t, sh);
  }
  if (threadIdx.x == 0) {
    const bool was = sc[SC_CONV] >= 0.0;
    if (!was) {
      sc[SC_RR] = v[1];
      if (v[1] <= sc[SC_TOL2] * sc[SC_BB]) sc[SC_CONV] = (double)it;
      const double beta = sc[SC_RZ] == 0.0 ? 0.0 : v[0] / sc[SC_RZ];
      sc[SC_BETA] = isfinite(beta) ? beta : 0.0;
      sc[SC_RZ] = v[0];
    }
  }
}

__global__ void k_pcg_pupdate(int64_t n, const double* __restrict__ sc, const double* __restrict__ z,
                              double* __restrict__ p) {
  if (sc[SC_CONV] >= 0.0) return;
  const double beta = sc[SC_BETA];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = fma(beta, p[i], z[i]);
}

}  // namespace hm

using namespace hm;

namespace {
inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline int grid1(int64_t n, int block) { return (int)((n + block - 1) / block); }
inline int ok_or_cuda() { return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA; }
}  // namespace

extern "C" int hm_csr_spmv(int64_t nrow, const int32_t* indptr, const int32_t* indices,
                           const double* vals, const double* x, double* y, double alpha,
                           double beta, void* stream) {
  if (nrow < 0 || (nrow > 0 && (!indptr || !indices || !vals || !x || !y))) return HM_ERR_ARG;
  if (nrow == 0) return HM_OK;
  k_spmv<8, false><<<grid1(nrow * 8, 256), 256, 0, S_(stream)>>>(nrow, indptr, indices, nullptr, vals, x, y, alpha, beta);
  return ok_or_cuda();
}

extern "C" int hm_csr_spmv_t(int64_t nrow, const int32_t* indptr, const int32_t* indices,
                             const int32_t* tpos, const double* vals, const double* x, double* y,
                             double alpha, double beta, void* stream) {
  if (nrow < 0 || (nrow > 0 && (!indptr || !indices || !tpos || !vals || !x || !y))) return HM_ERR_ARG;
  if (nrow == 0) return HM_OK;
  k_spmv<8, true><<<grid1(nrow * 8, 256), 256, 0, S_(stream)>>>(nrow, indptr, indices, tpos, vals, x, y, alpha, beta);
  return ok_or_cuda();
}

extern "C" int hm_csr_diag(int64_t nrow, const int32_t* indptr, const double* vals, double* diag,
                           void* stream) {
  if (nrow < 0 || (nrow > 0 && (!indptr || !vals || !diag))) return HM_ERR_ARG;
  if (nrow == 0) return HM_OK;
  k_csr_diag<<<grid1(nrow, 256), 256, 0, S_(stream)>>>(nrow, indptr, vals, diag);
  return ok_or_cuda();
}

extern "C" int64_t hm_dot_workspace_bytes(int64_t n) {
  (void)n;
  return (int64_t)kReduceBlocks * (int64_t)sizeof(double);
}

extern "C" int hm_dot(int64_t n, const double* x, const double* y, double* out, void* work,
                      void* stream) {
  if (n < 0 || !out || !work || (n > 0 && (!x || !y))) return HM_ERR_ARG;
  double* part = static_cast<double*>(work);
  k_dot_partial<<<kReduceBlocks, kReduceThreads, 0, S_(stream)>>>(n, x, y, part);
  k_reduce_final<<<1, 1024, 0, S_(stream)>>>(part, 1, out);
  return ok_or_cuda();
}

extern "C" int64_t hm_pcg_workspace_bytes(int64_t n) {
  // r, z, p, q, the partial sums of p.q (at most one per node), scalars, partials
  return (int64_t)sizeof(double) * (5 * n + SC_N + 3 * (int64_t)kReduceBlocks + 8);
}

int hm_launch_apply_A_dot(const hm::Lattice& L, void* jac, int precision, const uint8_t* ess,
                          const double* x, double* y, double* part, void* stream);
int64_t hm_apply_dot_parts(const hm::Lattice& L);

int hm_pcg_operator(int64_t n, const int32_t* indptr, const int32_t* indices, const double* vals,
                    const hm::Lattice* L, const void* quad, int precision, const uint8_t* ess,
                    const double* x, double* y, void* stream);

extern "C" int hm_pcg_impl(int64_t n, const int32_t* indptr, const int32_t* indices,
                           const double* vals, const hm::Lattice* L, const void* quad,
                           int precision, const uint8_t* ess, const double* diag, const double* b,
                           double* x, double rtol, int maxiter, int check_every, void* work,
                           int* iterations, double* relres, void* stream) {
  if (n <= 0 || !diag || !b || !x || !work || maxiter < 0) return HM_ERR_ARG;
  if (check_every <= 0) check_every = 1;
  cudaStream_t s = S_(stream);
  double* w = static_cast<double*>(work);
  double* r = w;
  double* z = w + n;
  double* p = w + 2 * n;
  double* q = w + 3 * n;
  double* pq_part = w + 4 * n;
  double* sc = w + 5 * n;
  double* part = sc + SC_N;
  int rc = hm_pcg_operator(n, indptr, indices, vals, L, quad, precision, ess, x, q, stream);
  if (rc) return rc;
  k_pcg_init<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, b, q, diag, r, z, p, part);
  k_pcg_init_final<<<1, 1024, 0, s>>>(part, sc, rtol);
  double host[SC_N];
  int it = 0;
  for (;;) {
    if (cudaMemcpyAsync(host, sc, sizeof(host), cudaMemcpyDeviceToHost, s) != cudaSuccess) return HM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HM_ERR_CUDA;
    if (host[SC_CONV] >= 0.0 || it >= maxiter) break;
    const int stop = it + check_every < maxiter ? it + check_every : maxiter;
    for (; it < stop;) {
      ++it;
      int64_t nparts = kReduceBlocks;
      if (L != nullptr) {
        // the lattice operator sums p.q as it writes q
        rc = hm_launch_apply_A_dot(*L, const_cast<void*>(quad), precision, ess, p, q, pq_part, stream);
        nparts = hm_apply_dot_parts(*L);
      } else {
        rc = hm_pcg_operator(n, indptr, indices, vals, L, quad, precision, ess, p, q, stream);
        if (!rc) k_dot_partial<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, p, q, pq_part);
      }
      if (rc) return rc;
      k_pcg_alpha<<<1, 1024, 0, s>>>(pq_part, nparts, sc);
      k_pcg_update<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, sc, x, r, z, p, q, diag, part);
      k_pcg_beta<<<1, 1024, 0, s>>>(part, sc, it);
      k_pcg_pupdate<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, sc, z, p);
    }
    if (cudaGetLastError() != cudaSuccess) return HM_ERR_CUDA;
  }
  const bool conv = host[SC_CONV] >= 0.0;
  if (iterations) *iterations = conv ? (int)host[SC_CONV] : it;
  if (relres) *relres = host[SC_BB] > 0.0 ? std::sqrt(host[SC_RR] / host[SC_BB]) : 0.0;
  return conv ? HM_OK : HM_ERR_NOCONV;
}
