// CSR products, deterministic reductions and the Jacobi-PCG of the incremental solves.
//
// Every reduction is two-pass over a fixed grid (kReduceBlocks blocks, grid-stride),
// so its summation order depends on n alone: repeated solves are bit-identical.
// The PCG keeps alpha, beta and the residual norms on the device; the host only
// launches and, every check_every iterations, reads one flag.  After convergence the
// step length is frozen at zero, so the result is that of the exact iteration count
// whatever check_every is.
#include <new>
#include <cmath>
#include <type_traits>
#include <vector>

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

// Vector kernels, templated on the vector type T (double, or float for the inner solves
// of the mixed-precision PCG); sums are accumulated in double.

// r = b - q, z = r / diag, p = z; partials of r.z, r.r, b.b
template <typename T>
__global__ void __launch_bounds__(kReduceThreads)
    k_pcg_init(int64_t n, const T* __restrict__ b, const T* __restrict__ q,
               const double* __restrict__ diag, T* __restrict__ r, T* __restrict__ z,
               T* __restrict__ p, double* __restrict__ part) {
  __shared__ double sh[32];
  double rz = 0.0, rr = 0.0, bb = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = b[i] - q[i];
    const T zi = ri / (T)diag[i];
    r[i] = ri; z[i] = zi; p[i] = zi;
    rz = fma((double)ri, (double)zi, rz);
    rr = fma((double)ri, (double)ri, rr);
    bb = fma((double)b[i], (double)b[i], bb);
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
    sc[SC_IT] = 0.0;
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

// beta = ((r.z)_new - rzc) / (r.z)_old, the convergence test and the iteration count
// (thread 0).  rzc = 0: Fletcher-Reeves; rzc = r_new . z_old: a Polak-Ribiere-type step
// for a preconditioner that is symmetric only to rounding.  The textbook flexible step
// (Golub and Ye 1999) takes z_new . r_old instead; for a symmetric preconditioner the
// two cross terms are equal, and both vanish in exact arithmetic.  With the FP32 V-cycle
// at high contrast the textbook step stalled on fields where this one converged.
__device__ __forceinline__ void beta_step(double rz, double rr, double* sc, double rzc = 0.0) {
  const bool was = sc[SC_CONV] >= 0.0;
  if (!was) {
    const double it = sc[SC_IT] + 1.0;
    sc[SC_IT] = it;
    sc[SC_RR] = rr;
    if (rr <= sc[SC_TOL2] * sc[SC_BB]) sc[SC_CONV] = it;
    const double beta = sc[SC_RZ] == 0.0 ? 0.0 : (rz - rzc) / sc[SC_RZ];
    sc[SC_BETA] = isfinite(beta) ? beta : 0.0;
    sc[SC_RZ] = rz;
  }
}

// x += alpha p, r -= alpha q, z = r / diag; partials of r.z and r.r; with counter, the
// last block to finish takes the step's beta (else k_pcg_beta does)
template <typename T>
__global__ void __launch_bounds__(kReduceThreads)
    k_pcg_update(int64_t n, double* __restrict__ sc, T* __restrict__ x, T* __restrict__ r,
                 T* __restrict__ z, const T* __restrict__ p, const T* __restrict__ q,
                 const double* __restrict__ diag, double* __restrict__ part,
                 unsigned* __restrict__ counter) {
  __shared__ double sh[32];
  const T alpha = (T)sc[SC_ALPHA];
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = fma(alpha, p[i], x[i]);
    const T ri = fma(-alpha, q[i], r[i]);
    const T zi = ri / (T)diag[i];
    r[i] = ri; z[i] = zi;
    rz = fma((double)ri, (double)zi, rz);
    rr = fma((double)ri, (double)ri, rr);
  }
  rz = block_sum(rz, sh);
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rz;
    part[kReduceBlocks + blockIdx.x] = rr;
  }
  if (counter != nullptr && last_block(counter)) {
    double v0 = 0.0, v1 = 0.0;
    for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) {
      v0 += __ldcg(part + b);
      v1 += __ldcg(part + kReduceBlocks + b);
    }
    v0 = block_sum(v0, sh);
    v1 = block_sum(v1, sh);
    if (threadIdx.x == 0) {
      beta_step(v0, v1, sc);
      *counter = 0u;
    }
  }
}

// the iteration count lives on the device (sc[SC_IT]), so that every batch of
// iterations launches the same kernels with the same arguments (a graph replays it)
__global__ void k_pcg_beta(const double* __restrict__ part, double* __restrict__ sc) {
  __shared__ double sh[32];
  double v[2];
  for (int q = 0; q < 2; ++q) {
    double t = 0.0;
    for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) t += part[q * kReduceBlocks + b];
    v[q] = block_sum(t, sh);
  }
  if (threadIdx.x == 0) beta_step(v[0], v[1], sc);
}

template <typename T>
__global__ void k_pcg_pupdate(int64_t n, const double* __restrict__ sc, const T* __restrict__ z,
                              T* __restrict__ p) {
  if (sc[SC_CONV] >= 0.0) return;
  const T beta = (T)sc[SC_BETA];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = fma(beta, p[i], z[i]);
}

// x += alpha p, r -= alpha q; partials of r.r (for a preconditioner applied after it)
// and, given the last preconditioned residual zold, of r.zold (slot 2: the flexible step)
__global__ void __launch_bounds__(kReduceThreads)
    k_pcg_update_rr(int64_t n, const double* __restrict__ sc, double* __restrict__ x,
                    double* __restrict__ r, const double* __restrict__ p,
                    const double* __restrict__ q, double* __restrict__ part,
                    const double* __restrict__ zold = nullptr) {
  __shared__ double sh[32];
  const double alpha = sc[SC_ALPHA];
  double rr = 0.0, rzc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    rr = fma(ri, ri, rr);
    if (zold != nullptr) rzc = fma(ri, zold[i], rzc);
  }
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) part[kReduceBlocks + blockIdx.x] = rr;
  if (zold != nullptr) {
    rzc = block_sum(rzc, sh);
    if (threadIdx.x == 0) part[2 * kReduceBlocks + blockIdx.x] = rzc;
  }
}

// partials of r.z; the last block takes beta from them and the r.r partials (flex: and
// the r.zold partials of k_pcg_update_rr, the flexible step)
__global__ void __launch_bounds__(kReduceThreads)
    k_pcg_rz_beta(int64_t n, const double* __restrict__ r, const double* __restrict__ z,
                  double* __restrict__ part, unsigned* __restrict__ counter,
                  double* __restrict__ sc, int flex = 0) {
  __shared__ double sh[32];
  double rz = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    rz = fma(r[i], z[i], rz);
  rz = block_sum(rz, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = rz;
  if (last_block(counter)) {
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) {
      v0 += __ldcg(part + b);
      v1 += __ldcg(part + kReduceBlocks + b);
      if (flex) v2 += __ldcg(part + 2 * kReduceBlocks + b);
    }
    v0 = block_sum(v0, sh);
    v1 = block_sum(v1, sh);
    if (flex) v2 = block_sum(v2, sh);
    if (threadIdx.x == 0) {
      beta_step(v0, v1, sc, v2);
      *counter = 0u;
    }
  }
}

// r = b - q; partials of r.r and b.b (slots 1 and 2)
__global__ void __launch_bounds__(kReduceThreads)
    k_pcg_mg_init(int64_t n, const double* __restrict__ b, const double* __restrict__ q,
                  double* __restrict__ r, double* __restrict__ part) {
  __shared__ double sh[32];
  double rr = 0.0, bb = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = b[i] - q[i];
    r[i] = ri;
    rr = fma(ri, ri, rr);
    bb = fma(b[i], b[i], bb);
  }
  rr = block_sum(rr, sh);
  bb = block_sum(bb, sh);
  if (threadIdx.x == 0) {
    part[kReduceBlocks + blockIdx.x] = rr;
    part[2 * kReduceBlocks + blockIdx.x] = bb;
  }
}

template <typename T>
__global__ void __launch_bounds__(kReduceThreads)
    k_dot_partial_t(int64_t n, const T* __restrict__ a, const T* __restrict__ b, double* __restrict__ part) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v = fma((double)a[i], (double)b[i], v);
  v = block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// Mixed precision (reliable updates): the FP32 vectors are scaled by s, the FP64 norm of
// the residual at the last anchor (sc[SC_S]); sc[SC_SOLD] is the scale before it.
enum { SC_S = SC_TMP0, SC_SOLD = SC_TMP1, SC_TRUE = SC_TMP2 };

// x64 += s x32, x32 = 0
__global__ void k_mx_accum(int64_t n, const double* __restrict__ sc, float* __restrict__ x32,
                           double* __restrict__ x) {
  const double s = sc[SC_S];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = fma(s, (double)x32[i], x[i]);
    x32[i] = 0.0f;
  }
}

// r64 = b - t64; partials of r64.r64
__global__ void __launch_bounds__(kReduceThreads)
    k_residual64(int64_t n, const double* __restrict__ b, const double* __restrict__ t,
                 const uint8_t* __restrict__ ess, double* __restrict__ r, double* __restrict__ part) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double ri = (ess && ess[i]) ? 0.0 : b[i] - (t ? t[i] : 0.0);
    r[i] = ri;
    v = fma(ri, ri, v);
  }
  v = block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// the true residual's r.r; the new scale
__global__ void k_mx_scale(const double* __restrict__ part, double* __restrict__ sc) {
  __shared__ double sh[32];
  double t = 0.0;
  for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) t += part[b];
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    sc[SC_TRUE] = t;
    sc[SC_SOLD] = sc[SC_S];
    sc[SC_S] = t > 0.0 ? sqrt(t) : 1.0;
  }
}

// r32 = r64 / s, z32 = r32 / diag, p32 = z32 (reset) or p32 * s_old / s; partials r.z, r.r
__global__ void __launch_bounds__(kReduceThreads)
    k_mx_anchor(int64_t n, const double* __restrict__ r64, const double* __restrict__ diag,
                const double* __restrict__ sc, int reset_p, float* __restrict__ r,
                float* __restrict__ z, float* __restrict__ p, double* __restrict__ part) {
  __shared__ double sh[32];
  const double inv = 1.0 / sc[SC_S];
  const float pscale = (float)(sc[SC_SOLD] * inv);
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float ri = (float)(r64[i] * inv);
    const float zi = ri / (float)diag[i];
    r[i] = ri; z[i] = zi;
    p[i] = reset_p ? zi : p[i] * pscale;
    rz = fma((double)ri, (double)zi, rz);
    rr = fma((double)ri, (double)ri, rr);
  }
  rz = block_sum(rz, sh);
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = rz;
    part[kReduceBlocks + blockIdx.x] = rr;
  }
}

// scalars of the recurrence after an anchor; bb and tol2 are in the scaled units
__global__ void k_mx_anchor_final(const double* __restrict__ part, double* __restrict__ sc,
                                  const double* __restrict__ bbp, double rtol) {
  __shared__ double sh[32];
  double v[2];
  for (int q = 0; q < 2; ++q) {
    double t = 0.0;
    for (int b = threadIdx.x; b < kReduceBlocks; b += blockDim.x) t += part[q * kReduceBlocks + b];
    v[q] = block_sum(t, sh);
  }
  if (threadIdx.x == 0) {
    const double s = sc[SC_S];
    sc[SC_RZ] = v[0];
    sc[SC_RR] = v[1];
    sc[SC_BB] = *bbp / (s * s);
    sc[SC_TOL2] = rtol * rtol;
    sc[SC_CONV] = -1.0;
  }
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

// slots for the partial sums of p.q: one per block of the lattice operator's gather
// (at most n), or the fixed reduction grid after a CSR product
inline int64_t pq_slots(int64_t n) { return n > kReduceBlocks ? n : (int64_t)kReduceBlocks; }

extern "C" int64_t hm_pcg_workspace_bytes(int64_t n) {
  // r, z, p, q, the partial sums of p.q, scalars, partials
  return (int64_t)sizeof(double) * (4 * n + pq_slots(n) + SC_N + 3 * (int64_t)kReduceBlocks + 8);
}

int64_t hm_apply_dot_parts(const hm::Lattice& L);
int hm_pcg_operator(int64_t n, const int32_t* indptr, const int32_t* indices, const double* vals,
                    const hm::Lattice* L, const void* quad, int precision, const uint8_t* ess,
                    const double* x, double* y, void* stream);

namespace {

// The operator of one PCG: y = A x, and, when part is given, the partial sums of x.y
// (returns their count through *nparts).
struct PcgOp {
  int64_t n;
  const int32_t* indptr;
  const int32_t* indices;
  const double* vals;
  const hm::Lattice* L;
  void* jac;
  int precision;
  const uint8_t* ess;
};

// With sc and counter, the lattice operator's last block also takes the step's alpha
// (*fused = true); the CSR product leaves it to k_pcg_alpha.
int op_apply(const PcgOp& o, const double* x, double* y, double* part, int64_t* nparts, void* stream,
             double* sc = nullptr, unsigned* counter = nullptr, bool* fused = nullptr) {
  if (fused) *fused = false;
  if (o.L != nullptr) {
    if (part) {
      *nparts = hm_apply_dot_parts(*o.L);
      if (fused) *fused = sc != nullptr;
      return hm_launch_apply_A_dot(*o.L, o.jac, o.precision, o.ess, x, y, part, stream, sc, counter);
    }
    return hm_pcg_operator(o.n, nullptr, nullptr, nullptr, o.L, o.jac, o.precision, o.ess, x, y, stream);
  }
  int rc = hm_pcg_operator(o.n, o.indptr, o.indices, o.vals, nullptr, nullptr, HM_FP64, o.ess, x, y, stream);
  if (rc || !part) return rc;
  *nparts = kReduceBlocks;
  k_dot_partial_t<double><<<kReduceBlocks, kReduceThreads, 0, S_(stream)>>>(o.n, x, y, part);
  return ok_or_cuda();
}

int op_apply(const PcgOp& o, const float* x, float* y, double* part, int64_t* nparts, void* stream,
             double* sc = nullptr, unsigned* counter = nullptr, bool* fused = nullptr) {
  if (part) *nparts = hm_apply_dot_parts(*o.L);
  if (fused) *fused = part != nullptr && sc != nullptr;
  return hm_launch_apply_A32_dot(*o.L, o.jac, o.ess, x, y, part, stream, sc, counter);
}

// `count` PCG iterations (operator + fused p.q, alpha, update with r.z and r.r, beta,
// direction); nothing in it synchronises with the host
// cnt: two counters (zero between uses) for the reductions the producing kernels finish
template <typename T>
int pcg_batch(const PcgOp& o, const double* diag, T* x, T* r, T* z, T* p, T* q, double* pq_part,
              double* sc, double* part, unsigned* cnt, int count, cudaStream_t s) {
  int64_t np = 0;
  for (int j = 0; j < count; ++j) {
    bool fused = false;
    const int rc = op_apply(o, p, q, pq_part, &np, (void*)s, sc, cnt, &fused);
    if (rc) return rc;
    if (!fused) k_pcg_alpha<<<1, 1024, 0, s>>>(pq_part, np, sc);
    k_pcg_update<T><<<kReduceBlocks, kReduceThreads, 0, s>>>(o.n, sc, x, r, z, p, q, diag, part,
                                                               cnt + 1);
    k_pcg_pupdate<T><<<kReduceBlocks, kReduceThreads, 0, s>>>(o.n, sc, z, p);
  }
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

}  // namespace

// A full batch of iterations captured once as a CUDA graph and replayed (a solve plan
// owns one per precision); partial batches, and streams that cannot be captured (the
// legacy default stream), launch directly.
struct HmBatchGraph {
  cudaGraphExec_t exec = nullptr;
  ~HmBatchGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

namespace {

template <typename F>
int run_batch(HmBatchGraph* g, bool full, cudaStream_t s, F&& launch) {
  if (g == nullptr || s == nullptr || !full) return launch();
  if (g->exec == nullptr) {
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HM_ERR_CUDA;
    const int rc = launch();
    const cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (rc != HM_OK || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      (void)cudaGetLastError();
      return rc != HM_OK ? rc : HM_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      g->exec = nullptr;
      return HM_ERR_CUDA;
    }
  }
  return cudaGraphLaunch(g->exec, s) == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

// Jacobi-PCG on vectors of type T from initial guess x; work holds r, z, p, q (T), the
// p.q partials (n doubles), the scalars and the partials.  Returns HM_OK / HM_ERR_NOCONV.
template <typename T>
int pcg_run(const PcgOp& o, const double* diag, const T* b, T* x, double rtol, int maxiter,
            int check_every, double* wd, T* wt, int* iterations, double* relres, void* stream,
            HmBatchGraph* graph = nullptr) {
  const int64_t n = o.n;
  cudaStream_t s = S_(stream);
  T* r = wt;
  T* z = wt + n;
  T* p = wt + 2 * n;
  T* q = wt + 3 * n;
  double* pq_part = wd;
  double* sc = wd + pq_slots(n);
  double* part = sc + SC_N;
  unsigned* cnt = reinterpret_cast<unsigned*>(part + 3 * kReduceBlocks);
  if (check_every <= 0) check_every = 1;
  if (cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), S_(stream)) != cudaSuccess) return HM_ERR_CUDA;
  int rc;
  // x = b on the Dirichlet nodes: every residual and direction is then zero there, which
  // the lattice operator's direction products rely on
  if constexpr (std::is_same<T, double>::value)
    if (o.L && (rc = hm_launch_ess_take_b(*o.L, o.ess, b, x, stream))) return rc;
  int64_t nparts = 0;
  rc = op_apply(o, x, q, nullptr, &nparts, stream);
  if (rc) return rc;
  k_pcg_init<T><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, b, q, diag, r, z, p, part);
  k_pcg_init_final<<<1, 1024, 0, s>>>(part, sc, rtol);
  double host[SC_N];
  int it = 0;
  for (;;) {
    if (cudaMemcpyAsync(host, sc, sizeof(host), cudaMemcpyDeviceToHost, s) != cudaSuccess) return HM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HM_ERR_CUDA;
    if (host[SC_CONV] >= 0.0 || it >= maxiter) break;
    const int count = it + check_every < maxiter ? check_every : maxiter - it;
    rc = run_batch(graph, count == check_every, s, [&] {
      return pcg_batch<T>(o, diag, x, r, z, p, q, pq_part, sc, part, cnt, count, s);
    });
    if (rc) return rc;
    it += count;
  }
  const bool conv = host[SC_CONV] >= 0.0;
  if (iterations) *iterations = conv ? (int)host[SC_CONV] : it;
  if (relres) *relres = host[SC_BB] > 0.0 ? std::sqrt(host[SC_RR] / host[SC_BB]) : 0.0;
  return conv ? HM_OK : HM_ERR_NOCONV;
}

}  // namespace

extern "C" int hm_pcg_impl(int64_t n, const int32_t* indptr, const int32_t* indices,
                           const double* vals, const hm::Lattice* L, const void* quad,
                           int precision, const uint8_t* ess, const double* diag, const double* b,
                           double* x, double rtol, int maxiter, int check_every, void* work,
                           int* iterations, double* relres, void* stream) {
  if (n <= 0 || !diag || !b || !x || !work || maxiter < 0) return HM_ERR_ARG;
  PcgOp o{n, indptr, indices, vals, L, const_cast<void*>(quad), precision, ess};
  double* w = static_cast<double*>(work);
  return pcg_run<double>(o, diag, b, x, rtol, maxiter, check_every, w + 4 * n, w, iterations,
                         relres, stream);
}

int hm_mg_vcycle(hm_mg* mg, const double* r, double* z, void* stream);
// the V-cycle is symmetric only to rounding (FP32): its CG takes the flexible step
bool hm_mg_flexible(const hm_mg* mg);
const double* hm_mg_level0_diag(const hm_mg* mg);
void* hm_mg_jac(const hm_mg* mg);
const uint8_t* hm_mg_ess(const hm_mg* mg);
const hm::Lattice* hm_mg_lattice(const hm_mg* mg);

namespace {
// PCG preconditioned by a multigrid V-cycle (the operator and diagonal are the MG's
// level 0); work as for hm_pcg.  x is the initial guess.
int pcg_mg_run(hm_mg* mg, const double* b, double* x, double rtol, int maxiter, int check_every,
               void* work, int* iterations, double* relres, void* stream, HmBatchGraph* graph) {
  const hm::Lattice* L = hm_mg_lattice(mg);
  if (!L || !hm_mg_jac(mg)) return HM_ERR_ARG;
  const int64_t n = L->ndof;
  cudaStream_t s = S_(stream);
  PcgOp o{n, nullptr, nullptr, nullptr, L, hm_mg_jac(mg), HM_FP64, hm_mg_ess(mg)};
  double* w = static_cast<double*>(work);
  double* r = w;
  double* z = w + n;
  double* p = w + 2 * n;
  double* q = w + 3 * n;
  double* pq_part = w + 4 * n;
  double* sc = pq_part + pq_slots(n);
  double* part = sc + SC_N;
  unsigned* cnt = reinterpret_cast<unsigned*>(part + 3 * kReduceBlocks);
  if (check_every <= 0) check_every = 1;
  if (cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), s) != cudaSuccess) return HM_ERR_CUDA;
  int rc = hm_launch_ess_take_b(*L, o.ess, b, x, stream);   // as in pcg_run
  if (rc) return rc;
  int64_t np = 0;
  rc = op_apply(o, x, q, nullptr, &np, stream);
  if (rc) return rc;
  k_pcg_mg_init<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, b, q, r, part);
  if ((rc = hm_mg_vcycle(mg, r, z, stream))) return rc;
  k_dot_partial_t<double><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, r, z, part);
  k_pcg_init_final<<<1, 1024, 0, s>>>(part, sc, rtol);
  if (cudaMemcpyAsync(p, z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return HM_ERR_CUDA;
  double host[SC_N];
  int it = 0;
  const int flex = hm_mg_flexible(mg) ? 1 : 0;
  // with the FP32 cycle: r.r at each check; the solve stops (HM_ERR_NOCONV) once, past
  // iteration 24, twelve iterations no longer halve the residual -- the cycle's rounding,
  // relative to the smooth part of its correction, then swamps the rest (high contrast)
  std::vector<double> hist;
  const int back = (12 + check_every - 1) / check_every;
  bool stalled = false;
  for (;;) {
    if (cudaMemcpyAsync(host, sc, sizeof(host), cudaMemcpyDeviceToHost, s) != cudaSuccess) return HM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HM_ERR_CUDA;
    if (host[SC_CONV] >= 0.0 || it >= maxiter) break;
    if (flex) {
      hist.push_back(host[SC_RR]);
      if (it >= 24 && (int)hist.size() > back &&
          host[SC_RR] > 0.25 * hist[hist.size() - 1 - back]) {
        stalled = true;
        break;
      }
    }
    const int count = it + check_every < maxiter ? check_every : maxiter - it;
    rc = run_batch(graph, count == check_every, s, [&]() -> int {
      for (int j = 0; j < count; ++j) {
        bool fused = false;
        int e = op_apply(o, p, q, pq_part, &np, (void*)s, sc, cnt, &fused);
        if (e) return e;
        if (!fused) k_pcg_alpha<<<1, 1024, 0, s>>>(pq_part, np, sc);
        k_pcg_update_rr<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, sc, x, r, p, q, part,
                                                                 flex ? z : nullptr);
        if ((e = hm_mg_vcycle(mg, r, z, (void*)s))) return e;
        k_pcg_rz_beta<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, r, z, part, cnt + 1, sc, flex);
        k_pcg_pupdate<double><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, sc, z, p);
      }
      return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
    });
    if (rc) return rc;
    it += count;
  }
  const bool conv = !stalled && host[SC_CONV] >= 0.0;
  if (iterations) *iterations = conv ? (int)host[SC_CONV] : it;
  if (relres) *relres = host[SC_BB] > 0.0 ? std::sqrt(host[SC_RR] / host[SC_BB]) : 0.0;
  return conv ? HM_OK : HM_ERR_NOCONV;
}
}  // namespace

extern "C" int hm_pcg_mg(hm_mg* mg, const double* b, double* x, double rtol, int maxiter,
                         int check_every, void* work, int* iterations, double* relres,
                         void* stream) {
  if (!mg || !b || !x || !work || maxiter < 0) return HM_ERR_ARG;
  return pcg_mg_run(mg, b, x, rtol, maxiter, check_every, work, iterations, relres, stream,
                    nullptr);
}

extern "C" int64_t hm_pcg_mixed_workspace_bytes(int64_t n) {
  // FP64: r, t, the p.q partials (at most one per node), scalars, partials, b.b;
  // FP32: x, r, z, p, q of the single-precision recurrence
  return (int64_t)sizeof(double) * (4 * n + pq_slots(n) + SC_N + 3 * (int64_t)kReduceBlocks + 8) +
         (int64_t)sizeof(float) * (5 * n + 16);
}

// Conjugate gradients with reliable updates (Sleijpen & van der Vorst, 1996): the
// recurrence runs in FP32 (vectors and the FP32 matrix-free operator, sums in FP64) on
// a system scaled by the residual norm s; when its residual has fallen by `delta` since
// the last anchor, or it claims convergence, the correction is added to the FP64 x,
// the true residual b - A64 x replaces the recurrence's (rescaled; the search direction
// is kept), and the true residual decides convergence.  Goal and stall test follow the
// reference's refined solves (modeling/PDEVariationalProblem.py:1236-1237, :1299): a
// residual that no longer halves between anchors is at its rounding floor; it counts as
// converged within 10 rtol.
namespace {
int pcg_mixed_run(const hm::Lattice* L, void* jac64, void* jac32, const uint8_t* ess,
                  const double* diag, const double* b, double* x, double rtol, double delta,
                  int max_updates, int maxiter, int check_every, void* work, int* iterations,
                  int* updates, double* relres, void* stream, HmBatchGraph* graph) {
  if (!L || !jac64 || !jac32 || !diag || !b || !x || !work || max_updates <= 0 || maxiter < 0 ||
      !(delta > 0.0 && delta < 1.0) || !(rtol >= 0.0))
    return HM_ERR_ARG;
  const int64_t n = L->ndof;
  cudaStream_t s = S_(stream);
  double* w = static_cast<double*>(work);
  double* r64 = w;
  double* t64 = w + n;
  double* pq_part = w + 4 * n;     // (w + 2n .. 4n: the FP64 finish's z and p)
  double* sc = pq_part + pq_slots(n);
  double* part = sc + SC_N;
  double* bbp = part + 3 * kReduceBlocks;
  unsigned* cnt = reinterpret_cast<unsigned*>(bbp + 1);
  float* f32 = reinterpret_cast<float*>(bbp + 8);
  float* x32 = f32;
  float* r32 = f32 + n;
  float* z32 = f32 + 2 * n;
  float* p32 = f32 + 3 * n;
  float* q32 = f32 + 4 * n;
  PcgOp o32{n, nullptr, nullptr, nullptr, L, jac32, HM_FP32, ess};
  PcgOp o64{n, nullptr, nullptr, nullptr, L, jac64, HM_FP64, ess};
  if (check_every <= 0) check_every = 1;
  double h[SC_N];
  auto read = [&]() -> int {
    if (cudaMemcpyAsync(h, sc, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return HM_ERR_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? HM_OK : HM_ERR_CUDA;
  };
  // the anchor: [x += s x32; t = A64 x]; r = b - t; new scale; FP32 r, z, p from r (p
  // restarted as z on the first anchor and on a restart)
  auto anchor = [&](bool first, bool restart) -> int {
    int64_t np = 0;
    if (!first) {
      k_mx_accum<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, sc, x32, x);
      const int rc = op_apply(o64, x, t64, nullptr, &np, stream);
      if (rc) return rc;
    }
    // first: x is b on the Dirichlet nodes and 0 elsewhere, so r = b off them, 0 on them
    k_residual64<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, b, first ? nullptr : t64,
                                                          first ? ess : nullptr, r64, part);
    k_mx_scale<<<1, 1024, 0, s>>>(part, sc);
    if (first && cudaMemcpyAsync(bbp, sc + SC_TRUE, sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return HM_ERR_CUDA;
    k_mx_anchor<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, r64, diag, sc, (first || restart) ? 1 : 0,
                                                         r32, z32, p32, part);
    k_mx_anchor_final<<<1, 1024, 0, s>>>(part, sc, bbp, rtol);
    if (cudaGetLastError() != cudaSuccess) return HM_ERR_CUDA;
    return read();
  };
  if (cudaMemsetAsync(sc, 0, sizeof(double) * SC_N, s) != cudaSuccess ||
      cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), s) != cudaSuccess ||
      cudaMemsetAsync(x, 0, sizeof(double) * n, s) != cudaSuccess ||
      cudaMemsetAsync(x32, 0, sizeof(float) * n, s) != cudaSuccess)
    return HM_ERR_CUDA;
  int rc = hm_launch_ess_take_b(*L, ess, b, x, stream);
  if (rc) return rc;
  rc = anchor(true, true);
  if (rc) return rc;
  const double bb = h[SC_TRUE];
  const double tol2 = rtol * rtol * bb, goal2 = 100.0 * tol2;
  double tr = bb, prev = bb;
  int it = 0, nup = 0, stalls = 0, last_anchor = 0;
  bool conv = tr <= tol2;
  while (!conv) {
    const int count = it + check_every < maxiter ? check_every : maxiter - it;
    rc = run_batch(graph, count == check_every, s, [&] {
      return pcg_batch<float>(o32, diag, x32, r32, z32, p32, q32, pq_part, sc, part, cnt, count, s);
    });
    if (rc) return rc;
    it += count;
    if ((rc = read())) return rc;
    const bool claim = h[SC_CONV] >= 0.0;
    // a recurrence that has grown above its anchor's residual, or has not fallen by
    // delta in 2000 iterations, has lost its way in single precision: restart it
    const bool lost = !(h[SC_RR] <= 1.0) || it - last_anchor > 2000;
    if (!claim && !lost && h[SC_RR] > delta * delta && it < maxiter) continue;
    if ((rc = anchor(false, lost))) return rc;
    last_anchor = it;
    ++nup;
    tr = h[SC_TRUE];
    if (tr <= tol2) { conv = true; break; }
    const bool stalled = tr > 0.25 * prev;
    stalls = stalled ? stalls + 1 : 0;
    prev = tr;
    if ((stalled && claim) || stalls >= 2 || it >= maxiter || nup >= max_updates) {
      conv = tr <= goal2;
      break;
    }
  }
  if (!conv && it < maxiter) {
    // single precision cannot carry this solve (its residual stalls above the goal, or
    // the anchors run out): finish it in FP64 from the current x, as the reference's
    // refined solves do (_solve_in_double, modeling/PDEVariationalProblem.py:1329-1360)
    int its64 = 0;
    double rr64 = 0.0;
    const int rc64 = pcg_run<double>(o64, diag, b, x, rtol, maxiter - it, check_every, pq_part,
                                     w, &its64, &rr64, stream);
    if (rc64 != HM_OK && rc64 != HM_ERR_NOCONV) return rc64;
    if (iterations) *iterations = it + its64;
    if (updates) *updates = nup;
    if (relres) *relres = rr64;
    return rc64;
  }
  if (iterations) *iterations = it;
  if (updates) *updates = nup;
  if (relres) *relres = bb > 0.0 ? std::sqrt(tr / bb) : 0.0;
  return conv ? HM_OK : HM_ERR_NOCONV;
}
}  // namespace

extern "C" int hm_pcg_mixed_impl(const hm::Lattice* L, void* jac64, void* jac32, const uint8_t* ess,
                                 const double* diag, const double* b, double* x, double rtol,
                                 double delta, int max_updates, int maxiter, int check_every,
                                 void* work, int* iterations, int* updates, double* relres,
                                 void* stream) {
  return pcg_mixed_run(L, jac64, jac32, ess, diag, b, x, rtol, delta, max_updates, maxiter,
                       check_every, work, iterations, updates, relres, stream, nullptr);
}

// ------------------------------------------------------------------ solve plans
struct hm_pcg_plan {
  hm::Lattice L;
  void* jac64;
  void* jac32;          // NULL: an FP64 solve
  const uint8_t* ess;
  const double* diag;
  double* b;
  double* x;
  void* work;
  int check_every;
  hm_mg* mg;            // non-NULL: MG-preconditioned FP64 solves
  HmBatchGraph graph;
};

extern "C" int hm_pcg_plan_create(const hm_lattice* h, void* jac64, void* jac32,
                                  const uint8_t* ess, const double* diag, double* b, double* x,
                                  void* work, int check_every, hm_pcg_plan** plan) {
  const hm::Lattice* L = hm_lattice_geometry(h);
  if (!L || !jac64 || !diag || !b || !x || !work || !plan || check_every <= 0) return HM_ERR_ARG;
  hm_pcg_plan* p = new (std::nothrow) hm_pcg_plan();
  if (!p) return HM_ERR_NOMEM;
  p->L = *L;
  p->jac64 = jac64;
  p->jac32 = jac32;
  p->ess = ess;
  p->diag = diag;
  p->b = b;
  p->x = x;
  p->work = work;
  p->check_every = check_every;
  p->mg = nullptr;
  *plan = p;
  return HM_OK;
}

int hm_plan_buffers(const hm_pcg_plan* p, double** b, double** x) {
  if (!p || !b || !x) return HM_ERR_ARG;
  *b = p->b;
  *x = p->x;
  return HM_OK;
}

extern "C" int hm_pcg_plan_set_mg(hm_pcg_plan* p, hm_mg* mg) {
  if (!p || (mg && p->jac32 != nullptr)) return HM_ERR_ARG;
  if (p->graph.exec) {
    cudaGraphExecDestroy(p->graph.exec);
    p->graph.exec = nullptr;
  }
  p->mg = mg;
  return HM_OK;
}

extern "C" int hm_pcg_plan_solve(hm_pcg_plan* p, double rtol, double delta, int max_updates,
                                 int maxiter, int* iterations, int* updates, double* relres,
                                 void* stream) {
  if (!p || maxiter < 0) return HM_ERR_ARG;
  if (p->mg != nullptr) {
    if (updates) *updates = 0;
    if (cudaMemsetAsync(p->x, 0, sizeof(double) * p->L.ndof, S_(stream)) != cudaSuccess)
      return HM_ERR_CUDA;
    return pcg_mg_run(p->mg, p->b, p->x, rtol, maxiter, p->check_every, p->work, iterations,
                      relres, stream, &p->graph);
  }
  if (p->jac32 != nullptr)
    return pcg_mixed_run(&p->L, p->jac64, p->jac32, p->ess, p->diag, p->b, p->x, rtol, delta,
                         max_updates, maxiter, p->check_every, p->work, iterations, updates,
                         relres, stream, &p->graph);
  const int64_t n = p->L.ndof;
  cudaStream_t s = S_(stream);
  if (cudaMemsetAsync(p->x, 0, sizeof(double) * n, s) != cudaSuccess) return HM_ERR_CUDA;
  PcgOp o{n, nullptr, nullptr, nullptr, &p->L, p->jac64, HM_FP64, p->ess};
  double* w = static_cast<double*>(p->work);
  if (updates) *updates = 0;
  return pcg_run<double>(o, p->diag, p->b, p->x, rtol, maxiter, p->check_every, w + 4 * n, w,
                         iterations, relres, stream, &p->graph);
}

extern "C" int hm_pcg_plan_destroy(hm_pcg_plan* p) {
  delete p;
  return HM_OK;
}

// ------------------------------------------------------------------- solve groups
// Several FP64 solve plans of one lattice size solved together: every plan's iteration
// batch is one branch of a single CUDA graph (one launch runs the batches of all
// plans, concurrently on the device), and one host synchronisation per batch reads
// every plan's convergence.  Each branch launches exactly the kernels its plan launches
// alone, on its own buffers, and a converged plan's iterate is frozen (its step length
// is zero), so every result is the one the plan gives solved alone, bit for bit.
struct hm_pcg_group {
  std::vector<hm_pcg_plan*> plans;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec = nullptr;
  int check_every = 1;
  ~hm_pcg_group() {
    if (exec) cudaGraphExecDestroy(exec);
    for (auto e : join) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    for (auto s : side) cudaStreamDestroy(s);
  }
};

namespace {
struct PlanBufs {
  double *r, *z, *p, *q, *pq_part, *sc, *part;
  unsigned* cnt;
};
PlanBufs plan_bufs(const hm_pcg_plan* pl) {
  const int64_t n = pl->L.ndof;
  double* w = static_cast<double*>(pl->work);
  PlanBufs b;
  b.r = w; b.z = w + n; b.p = w + 2 * n; b.q = w + 3 * n;
  b.pq_part = w + 4 * n;
  b.sc = b.pq_part + pq_slots(n);
  b.part = b.sc + SC_N;
  b.cnt = reinterpret_cast<unsigned*>(b.part + 3 * kReduceBlocks);
  return b;
}

// a plan's solve up to its first convergence check (x from zero), as its own solve does
int group_init(hm_pcg_plan* pl, double rtol, cudaStream_t s) {
  const int64_t n = pl->L.ndof;
  const PlanBufs B = plan_bufs(pl);
  PcgOp o{n, nullptr, nullptr, nullptr, &pl->L, pl->jac64, HM_FP64, pl->ess};
  if (cudaMemsetAsync(pl->x, 0, sizeof(double) * n, s) != cudaSuccess ||
      cudaMemsetAsync(B.cnt, 0, 2 * sizeof(unsigned), s) != cudaSuccess)
    return HM_ERR_CUDA;
  int rc = hm_launch_ess_take_b(pl->L, o.ess, pl->b, pl->x, (void*)s);
  if (rc) return rc;
  int64_t np = 0;
  if ((rc = op_apply(o, pl->x, B.q, nullptr, &np, (void*)s))) return rc;
  if (pl->mg != nullptr) {
    k_pcg_mg_init<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, pl->b, B.q, B.r, B.part);
    if ((rc = hm_mg_vcycle(pl->mg, B.r, B.z, (void*)s))) return rc;
    k_dot_partial_t<double><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, B.r, B.z, B.part);
    k_pcg_init_final<<<1, 1024, 0, s>>>(B.part, B.sc, rtol);
    if (cudaMemcpyAsync(B.p, B.z, sizeof(double) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return HM_ERR_CUDA;
  } else {
    k_pcg_init<double><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, pl->b, B.q, pl->diag, B.r, B.z,
                                                               B.p, B.part);
    k_pcg_init_final<<<1, 1024, 0, s>>>(B.part, B.sc, rtol);
  }
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

// `count` iterations of a plan, the same launches as its own solve's batches
int group_batch(hm_pcg_plan* pl, int count, cudaStream_t s) {
  const int64_t n = pl->L.ndof;
  const PlanBufs B = plan_bufs(pl);
  PcgOp o{n, nullptr, nullptr, nullptr, &pl->L, pl->jac64, HM_FP64, pl->ess};
  if (pl->mg == nullptr)
    return pcg_batch<double>(o, pl->diag, pl->x, B.r, B.z, B.p, B.q, B.pq_part, B.sc, B.part,
                             B.cnt, count, s);
  int64_t np = 0;
  for (int j = 0; j < count; ++j) {
    bool fused = false;
    int e = op_apply(o, B.p, B.q, B.pq_part, &np, (void*)s, B.sc, B.cnt, &fused);
    if (e) return e;
    if (!fused) k_pcg_alpha<<<1, 1024, 0, s>>>(B.pq_part, np, B.sc);
    const int flex = hm_mg_flexible(pl->mg) ? 1 : 0;
    k_pcg_update_rr<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, B.sc, pl->x, B.r, B.p, B.q, B.part,
                                                             flex ? B.z : nullptr);
    if ((e = hm_mg_vcycle(pl->mg, B.r, B.z, (void*)s))) return e;
    k_pcg_rz_beta<<<kReduceBlocks, kReduceThreads, 0, s>>>(n, B.r, B.z, B.part, B.cnt + 1, B.sc, flex);
    k_pcg_pupdate<double><<<kReduceBlocks, kReduceThreads, 0, s>>>(n, B.sc, B.z, B.p);
  }
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
}  // namespace

extern "C" int hm_pcg_group_create(hm_pcg_plan** plans, int count, hm_pcg_group** out) {
  if (!plans || count < 1 || count > 64 || !out) return HM_ERR_ARG;
  for (int i = 0; i < count; ++i) {
    if (!plans[i] || plans[i]->jac32 != nullptr) return HM_ERR_ARG;   // FP64 plans only
    if (plans[i]->check_every != plans[0]->check_every) return HM_ERR_ARG;
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return HM_ERR_ARG;
  }
  hm_pcg_group* g = new (std::nothrow) hm_pcg_group();
  if (!g) return HM_ERR_NOMEM;
  g->plans.assign(plans, plans + count);
  g->check_every = plans[0]->check_every;
  if (cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming) != cudaSuccess) {
    delete g;
    return HM_ERR_CUDA;
  }
  for (int i = 0; i < count; ++i) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      delete g;
      return HM_ERR_CUDA;
    }
    g->side.push_back(st);
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      delete g;
      return HM_ERR_CUDA;
    }
    g->join.push_back(ev);
  }
  *out = g;
  return HM_OK;
}

extern "C" int hm_pcg_group_destroy(hm_pcg_group* g) {
  delete g;
  return HM_OK;
}

extern "C" int hm_pcg_group_solve(hm_pcg_group* g, double rtol, int maxiter, int* iterations,
                                  double* relres, void* stream) {
  if (!g || maxiter < 0 || !(rtol >= 0.0)) return HM_ERR_ARG;
  cudaStream_t s = S_(stream);
  const int k = (int)g->plans.size();
  int rc;
  for (int i = 0; i < k; ++i)
    if ((rc = group_init(g->plans[i], rtol, s))) return rc;
  std::vector<double> host((size_t)k * SC_N);
  int it = 0;
  bool all = false;
  for (;;) {
    for (int i = 0; i < k; ++i)
      if (cudaMemcpyAsync(&host[(size_t)i * SC_N], plan_bufs(g->plans[i]).sc, SC_N * sizeof(double),
                          cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return HM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HM_ERR_CUDA;
    all = true;
    for (int i = 0; i < k; ++i) all = all && host[(size_t)i * SC_N + SC_CONV] >= 0.0;
    if (all || it >= maxiter) break;
    const int count = it + g->check_every < maxiter ? g->check_every : maxiter - it;
    if (s == nullptr || count != g->check_every) {
      for (int i = 0; i < k; ++i)
        if ((rc = group_batch(g->plans[i], count, s))) return rc;
    } else {
      if (g->exec == nullptr) {
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return HM_ERR_CUDA;
        int crc = cudaEventRecord(g->fork, s) == cudaSuccess ? HM_OK : HM_ERR_CUDA;
        for (int i = 0; i < k && crc == HM_OK; ++i) {
          if (cudaStreamWaitEvent(g->side[i], g->fork, 0) != cudaSuccess) { crc = HM_ERR_CUDA; break; }
          crc = group_batch(g->plans[i], count, g->side[i]);
          if (crc == HM_OK && (cudaEventRecord(g->join[i], g->side[i]) != cudaSuccess ||
                               cudaStreamWaitEvent(s, g->join[i], 0) != cudaSuccess))
            crc = HM_ERR_CUDA;
        }
        const cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (crc != HM_OK || e != cudaSuccess) {
          if (graph) cudaGraphDestroy(graph);
          (void)cudaGetLastError();
          return crc != HM_OK ? crc : HM_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&g->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
          g->exec = nullptr;
          return HM_ERR_CUDA;
        }
      }
      if (cudaGraphLaunch(g->exec, s) != cudaSuccess) return HM_ERR_CUDA;
    }
    it += count;
  }
  for (int i = 0; i < k; ++i) {
    const double* h = &host[(size_t)i * SC_N];
    const bool conv = h[SC_CONV] >= 0.0;
    if (iterations) iterations[i] = conv ? (int)h[SC_CONV] : it;
    if (relres) relres[i] = h[SC_BB] > 0.0 ? std::sqrt(h[SC_RR] / h[SC_BB]) : 0.0;
  }
  return all ? HM_OK : HM_ERR_NOCONV;
}
