// Pointwise observation operator of the Q2 lattice and a deterministic CSR transpose
// (sm_100a).
//
// B: row o holds the 27 Q2 basis values at target o, in the element that contains it
// (the reference's PointwiseObservation._build, modeling/pointwiseObservation.py:94-170,
// which locates each target with MFEM FindPoints and evaluates the element's shape
// functions there).  On the uniform lattice the element is floor(x / h) per axis
// (clamped to the last element for targets on the far face) and the shape functions are
// products of the three 1D quadratic Lagrange polynomials on the nodes 0, 1/2, 1.  The
// arithmetic is written with explicit round-to-nearest operations, so no contraction
// changes a value: the rows equal a host evaluation of the same formulas bit for bit.
//
// B^T (the adjoint source and W_uu = B^T B / sigma^2 of misfit.py:65-110) comes from a
// general transpose: integer counts per column, an exclusive scan, a fill through
// per-column cursors, and a sort of each transposed row by source row, so that the
// result does not depend on the order the atomics resolved in.
#include <cmath>

#include "hm_common.cuh"
#include "hm_internal.h"

namespace hm {
namespace {

constexpr int kScanBlock = 1024;

// 1D quadratic Lagrange values at t (nodes 0, 1/2, 1): 2(t - 1/2)(t - 1), -4t(t - 1),
// 2t(t - 1/2)
__device__ __forceinline__ void lagrange3_rn(double t, double (&b)[3]) {
  const double tm1 = __dsub_rn(t, 1.0), tmh = __dsub_rn(t, 0.5);
  b[0] = __dmul_rn(__dmul_rn(2.0, tmh), tm1);
  b[1] = __dmul_rn(__dmul_rn(-4.0, t), tm1);
  b[2] = __dmul_rn(__dmul_rn(2.0, t), tmh);
}

// one thread per target: its element, its 27 columns (ascending) and values; targets
// outside the box (beyond a relative 1e-12 of an element) or not finite set *bad
__global__ void k_obs_rows(Lattice L, const double* __restrict__ pts, int64_t npts,
                           int32_t* __restrict__ indptr, int32_t* __restrict__ indices,
                           double* __restrict__ vals, unsigned* __restrict__ bad) {
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o == 0) indptr[npts] = (int32_t)(27 * npts);
  if (o >= npts) return;
  indptr[o] = (int32_t)(27 * o);
  const double h[3] = {L.hx, L.hy, L.hz};
  const int ne[3] = {L.nx, L.ny, L.nz};
  double b[3][3];
  int e[3];
  bool out = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double x = pts[3 * o + d];
    const double s = __ddiv_rn(x, h[d]);
    if (!(s >= -1e-12 && s <= (double)ne[d] + 1e-12)) out = true;
    double f = floor(s);
    f = f < 0.0 ? 0.0 : (f > (double)(ne[d] - 1) ? (double)(ne[d] - 1) : f);
    e[d] = out ? 0 : (int)f;
    lagrange3_rn(__dsub_rn(s, f), b[d]);
  }
  if (out) atomicOr(bad, 1u);
  int32_t* col = indices + 27 * o;
  double* val = vals + 27 * o;
#pragma unroll
  for (int a = 0; a < 27; ++a) {
    const int a1 = a % 3, a2 = (a / 3) % 3, a3 = a / 9;
    col[a] = (int32_t)((2 * e[0] + a1) + (int64_t)L.Nx * ((2 * e[1] + a2) + (int64_t)L.Ny * (2 * e[2] + a3)));
    val[a] = out ? 0.0 : __dmul_rn(__dmul_rn(b[0][a1], b[1][a2]), b[2][a3]);
  }
}

__global__ void k_count_cols(int64_t nnz, const int32_t* __restrict__ indices, int32_t ncol,
                             int32_t* __restrict__ count, unsigned* __restrict__ bad) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int32_t c = indices[k];
  if (c < 0 || c >= ncol) { atomicOr(bad, 1u); return; }
  atomicAdd(count + c, 1);
}

// exclusive scan of n counts in blocks of kScanBlock; block totals to tot
__global__ void __launch_bounds__(kScanBlock) k_scan_blocks(int64_t n, const int32_t* __restrict__ in,
                                                           int32_t* __restrict__ out,
                                                           int64_t* __restrict__ tot) {
  __shared__ int64_t sh[kScanBlock];
  const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  const int64_t v = i < n ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int d = 1; d < kScanBlock; d <<= 1) {
    const int64_t t = threadIdx.x >= (unsigned)d ? sh[threadIdx.x - d] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = (int32_t)(sh[threadIdx.x] - v);
  if (threadIdx.x == kScanBlock - 1) tot[blockIdx.x] = sh[threadIdx.x];
}
// exclusive scan of the block totals (one block, looping); the grand total to out[n]
__global__ void __launch_bounds__(kScanBlock) k_scan_totals(int64_t nb, int64_t* __restrict__ tot,
                                                           int32_t* __restrict__ out, int64_t n) {
  __shared__ int64_t sh[kScanBlock];
  int64_t carry = 0;
  for (int64_t base = 0; base < nb; base += kScanBlock) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = i < nb ? tot[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int d = 1; d < kScanBlock; d <<= 1) {
      const int64_t t = threadIdx.x >= (unsigned)d ? sh[threadIdx.x - d] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) tot[i] = carry + sh[threadIdx.x] - v;
    const int64_t blocksum = sh[kScanBlock - 1];
    __syncthreads();
    carry += blocksum;
  }
  if (threadIdx.x == 0) out[n] = (int32_t)carry;
}
__global__ void k_scan_add(int64_t n, const int64_t* __restrict__ tot, int32_t* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = (int32_t)(out[i] + tot[i / kScanBlock]);
}

// one thread per source row: its entries to their columns' next free places (entries
// outside [0, nnz), columns outside [0, ncol) or beyond a column's count set *bad and are
// skipped)
__global__ void k_fill_t(int64_t nrow, int64_t nnz, int32_t ncol, const int32_t* __restrict__ indptr,
                         const int32_t* __restrict__ indices, const double* __restrict__ vals,
                         const int32_t* __restrict__ tindptr, int32_t* __restrict__ cursor,
                         int32_t* __restrict__ tindices, double* __restrict__ tvals,
                         unsigned* __restrict__ bad) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nrow) return;
  const int32_t lo = indptr[r], hi = indptr[r + 1];
  if (lo < 0 || hi < lo || hi > nnz) { atomicOr(bad, 1u); return; }
  for (int32_t k = lo; k < hi; ++k) {
    const int32_t c = indices[k];
    if (c < 0 || c >= ncol) continue;   // counted as bad already
    const int32_t pos = tindptr[c] + atomicAdd(cursor + c, 1);
    if (pos >= tindptr[c + 1]) { atomicOr(bad, 1u); continue; }
    tindices[pos] = (int32_t)r;
    tvals[pos] = vals[k];
  }
}
// one thread per transposed row: insertion sort by source row (rows are short)
__global__ void k_sort_rows(int64_t ncol, const int32_t* __restrict__ tindptr,
                            int32_t* __restrict__ tindices, double* __restrict__ tvals) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const int32_t lo = tindptr[c], hi = tindptr[c + 1];
  for (int32_t i = lo + 1; i < hi; ++i) {
    const int32_t key = tindices[i];
    const double v = tvals[i];
    int32_t j = i - 1;
    while (j >= lo && tindices[j] > key) {
      tindices[j + 1] = tindices[j];
      tvals[j + 1] = tvals[j];
      --j;
    }
    tindices[j + 1] = key;
    tvals[j + 1] = v;
  }
}

inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline int blocks_of(int64_t n, int t) { return (int)((n + t - 1) / t); }

int read_flag(unsigned* flag, cudaStream_t s, unsigned* host) {
  if (cudaMemcpyAsync(host, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return HM_ERR_CUDA;
  return HM_OK;
}

}  // namespace
}  // namespace hm

using namespace hm;

extern "C" int64_t hm_lattice_observation_workspace_bytes(int64_t npts) {
  (void)npts;
  return 256;
}

extern "C" int hm_lattice_observation(const hm_lattice* h, const double* d_points, int64_t npts,
                                      int32_t* d_indptr, int32_t* d_indices, double* d_vals,
                                      void* d_work, void* stream) {
  if (!h || npts < 0 || !d_indptr || (npts > 0 && (!d_points || !d_indices || !d_vals)) || !d_work)
    return HM_ERR_ARG;
  if (27 * npts > (int64_t)INT32_MAX) return HM_ERR_RANGE;
  const Lattice& L = *hm_lattice_geometry(h);
  cudaStream_t s = S_(stream);
  unsigned* bad = static_cast<unsigned*>(d_work);
  if (cudaMemsetAsync(bad, 0, sizeof(unsigned), s) != cudaSuccess) return HM_ERR_CUDA;
  k_obs_rows<<<blocks_of(npts + 1, 128), 128, 0, s>>>(L, d_points, npts, d_indptr, d_indices,
                                                      d_vals, bad);
  if (cudaGetLastError() != cudaSuccess) return HM_ERR_CUDA;
  unsigned flag = 0;
  const int rc = read_flag(bad, s, &flag);
  if (rc) return rc;
  return flag ? HM_ERR_RANGE : HM_OK;
}

extern "C" int64_t hm_csr_transpose_workspace_bytes(int64_t ncol) {
  const int64_t nb = (ncol + 1 + kScanBlock - 1) / kScanBlock;
  return 256 + 4 * (ncol + 1) + 8 * nb + 64;
}

extern "C" int hm_csr_transpose(int64_t nrow, int64_t ncol, int64_t nnz, const int32_t* d_indptr,
                                const int32_t* d_indices, const double* d_vals,
                                int32_t* d_tindptr, int32_t* d_tindices, double* d_tvals,
                                void* d_work, void* stream) {
  if (nrow < 0 || ncol < 0 || nnz < 0 || ncol > (int64_t)INT32_MAX || nnz > (int64_t)INT32_MAX ||
      !d_indptr || !d_tindptr || !d_work || (nnz > 0 && (!d_indices || !d_vals || !d_tindices || !d_tvals)))
    return HM_ERR_ARG;
  cudaStream_t s = S_(stream);
  unsigned char* w = static_cast<unsigned char*>(d_work);
  unsigned* bad = reinterpret_cast<unsigned*>(w);
  int32_t* count = reinterpret_cast<int32_t*>(w + 256);
  const int64_t nb = (ncol + 1 + kScanBlock - 1) / kScanBlock;
  int64_t* tot = reinterpret_cast<int64_t*>(
      w + ((256 + 4 * (ncol + 1) + 7) / 8) * 8);
  if (cudaMemsetAsync(bad, 0, sizeof(unsigned), s) != cudaSuccess ||
      cudaMemsetAsync(count, 0, sizeof(int32_t) * (ncol + 1), s) != cudaSuccess)
    return HM_ERR_CUDA;
  if (nnz > 0) k_count_cols<<<blocks_of(nnz, 256), 256, 0, s>>>(nnz, d_indices, (int32_t)ncol, count, bad);
  // exclusive scan of the ncol counts (the last slot stays 0); the total to tindptr[ncol]
  k_scan_blocks<<<(int)nb, kScanBlock, 0, s>>>(ncol, count, d_tindptr, tot);
  k_scan_totals<<<1, kScanBlock, 0, s>>>(nb, tot, d_tindptr, ncol);
  if (ncol > 0) k_scan_add<<<blocks_of(ncol, 256), 256, 0, s>>>(ncol, tot, d_tindptr);
  if (cudaMemsetAsync(count, 0, sizeof(int32_t) * (ncol + 1), s) != cudaSuccess) return HM_ERR_CUDA;
  if (nrow > 0)
    k_fill_t<<<blocks_of(nrow, 256), 256, 0, s>>>(nrow, nnz, (int32_t)ncol, d_indptr, d_indices,
                                                  d_vals, d_tindptr, count, d_tindices, d_tvals,
                                                  bad);
  if (ncol > 0) k_sort_rows<<<blocks_of(ncol, 256), 256, 0, s>>>(ncol, d_tindptr, d_tindices, d_tvals);
  if (cudaGetLastError() != cudaSuccess) return HM_ERR_CUDA;
  unsigned flag = 0;
  const int rc = read_flag(bad, s, &flag);
  if (rc) return rc;
  return flag ? HM_ERR_RANGE : HM_OK;
}
