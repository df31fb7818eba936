// The lattice path on a caller's own dof numbering, and the element-matrix export.
//
// The fused kernels number the Q2 dofs lexicographically on the node lattice.  A caller
// whose space numbers them otherwise (MFEM: vertices, then edges, faces and interiors,
// with its own element-local order) keeps its numbering through three pieces:
//   hm_lattice_dof_permutation  (host)   its element dof table -> perm[lattice node]
//   hm_lattice_caller_map       (device) for each entry of ITS CSR pattern (the arrays
//                                        hm_pattern_build gives for its table) the
//                                        position of the same (row, column) in the
//                                        lattice pattern
//   hm_gather_f64               (device) dst[i] = src[idx[i]]: vectors in and out
//                                        (idx = perm, or its inverse) and block values
//                                        out (idx = that map), coalesced writes, each
//                                        entry written once (deterministic)
// and hm_lattice_element_blocks writes the (27 x 27) element matrices of a point in a
// caller-chosen element-local order, the debug export of QuadratureKernel.
// element_matrices (hippymfem/fem/kernel.py:1964-2068).
#include <vector>

#include "hm_common.cuh"
#include "hm_internal.h"

namespace hm {

// ------------------------------------------------------------- caller position map
// One warp per lattice row n: row r = perm[n] of the caller's pattern must hold the
// same number of columns, its diagonal first; each lattice entry (n, c) finds its
// caller column perm[c] by a binary search of the ascending part of row r.
__global__ void k_caller_map(Lattice L, const int32_t* __restrict__ perm,
                             const int32_t* __restrict__ cindptr,
                             const int32_t* __restrict__ cindices, int32_t* __restrict__ src_pos,
                             uint32_t* __restrict__ status) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= L.ndof) return;
  const int i = (int)(row % L.Nx), j = (int)((row / L.Nx) % L.Ny), k = (int)(row / ((int64_t)L.Nx * L.Ny));
  const int n1 = stencil_n(i, L.Nx), n2 = stencil_n(j, L.Ny), n3 = stencil_n(k, L.Nz);
  const int lo1 = stencil_lo(i), lo2 = stencil_lo(j), lo3 = stencil_lo(k);
  const int kd = ((k - lo3) * n2 + (j - lo2)) * n1 + (i - lo1);
  const int len = n1 * n2 * n3;
  const int64_t lbase = row_start(L, i, j, k);
  const int32_t r = perm[row];
  if (r < 0 || r >= L.ndof) {
    if (lane == 0) atomicOr(status, HM_STATUS_RANGE);
    return;
  }
  const int32_t cb = cindptr[r], ce = cindptr[r + 1];
  if (ce - cb != len || cindices[cb] != r) {
    if (lane == 0) atomicOr(status, HM_STATUS_RANGE);
    return;
  }
  for (int pos = lane; pos < len; pos += 32) {
    const int rank = pos == 0 ? kd : (pos <= kd ? pos - 1 : pos);
    const int k1 = rank % n1, t = rank / n1, k2 = t % n2, k3 = t / n2;
    const int64_t c = (lo1 + k1) + (int64_t)L.Nx * ((lo2 + k2) + (int64_t)L.Ny * (lo3 + k3));
    const int32_t cc = perm[c];
    int32_t at = -1;
    if (cc == r) {
      at = cb;
    } else {
      int32_t a = cb + 1, b = ce;          // ascending columns in [a, b)
      while (a < b) {
        const int32_t mid = a + ((b - a) >> 1);
        if (cindices[mid] < cc) a = mid + 1;
        else b = mid;
      }
      if (a < ce && cindices[a] == cc) at = a;
    }
    if (at < 0) {
      atomicOr(status, HM_STATUS_RANGE);
      continue;
    }
    src_pos[at] = (int32_t)(lbase + pos);
  }
}

__global__ void k_gather_f64(int64_t n, const int32_t* __restrict__ idx, const double* __restrict__ src,
                             double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = __ldg(src + __ldg(idx + i));
}

// ------------------------------------------------------------ element matrices
// One CTA per element: the 216 pointwise values of the element and the tables of the
// 27 basis functions at the 27 points in shared memory, then each (a, b) entry as its
// 27-point sum (rows: test dof a, columns: trial dof b, as kernel.py:1704-1710):
//   A(a, b)   = sum_q D grad phi_a . grad phi_b
//   C(a, b)   = sum_q (E . grad phi_a) psi_b      (E = D grad u)
//   Wum(a, b) = sum_q (F . grad phi_a) psi_b      (F = D grad p)
//   Wmm(a, b) = sum_q W psi_a psi_b               (W = D grad u . grad p)
// written at [element][local[a]][local[b]].
struct LocalOrder { int32_t v[27]; };

template <typename real>
__global__ void __launch_bounds__(256) k_element_blocks(Lattice L, const real* __restrict__ quad,
                                                        int64_t e0, LocalOrder local,
                                                        double* oA, double* oC, double* oWum,
                                                        double* oWmm) {
  __shared__ double sq[216];
  __shared__ double nb[27][27];        // [q][a]
  __shared__ double gd[3][27][27];     // [axis][q][a], physical (1/h included)
  __shared__ int32_t loc[27];
  const int tid = threadIdx.x;
  const int64_t e = e0 + blockIdx.x;
  for (int t = tid; t < 216; t += blockDim.x) sq[t] = (double)quad[e * 216 + t];
  if (tid < 27) loc[tid] = local.v[tid];
  const double ih[3] = {1.0 / L.hx, 1.0 / L.hy, 1.0 / L.hz};
  for (int t = tid; t < 729; t += blockDim.x) {
    const int q = t / 27, a = t % 27;
    const int q1 = q % 3, q2 = (q / 3) % 3, q3 = q / 9;
    const int a1 = a % 3, a2 = (a / 3) % 3, a3 = a / 9;
    const double b1 = bq(q1, a1), b2 = bq(q2, a2), b3 = bq(q3, a3);
    nb[q][a] = b1 * b2 * b3;
    gd[0][q][a] = dbq(q1, a1) * b2 * b3 * ih[0];
    gd[1][q][a] = b1 * dbq(q2, a2) * b3 * ih[1];
    gd[2][q][a] = b1 * b2 * dbq(q3, a3) * ih[2];
  }
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * 729;
  for (int t = tid; t < 729; t += blockDim.x) {
    const int a = t / 27, b = t % 27;
    double sA = 0.0, sC = 0.0, sU = 0.0, sM = 0.0;
#pragma unroll 3
    for (int q = 0; q < 27; ++q) {
      const double ga0 = gd[0][q][a], ga1 = gd[1][q][a], ga2 = gd[2][q][a];
      const double nbq = nb[q][b];
      sA = fma(sq[q], ga0 * gd[0][q][b] + ga1 * gd[1][q][b] + ga2 * gd[2][q][b], sA);
      sC = fma(sq[27 + q] * ga0 + sq[54 + q] * ga1 + sq[81 + q] * ga2, nbq, sC);
      sU = fma(sq[108 + q] * ga0 + sq[135 + q] * ga1 + sq[162 + q] * ga2, nbq, sU);
      sM = fma(sq[189 + q] * nb[q][a], nbq, sM);
    }
    const int64_t o = base + (int64_t)loc[a] * 27 + loc[b];
    if (oA) oA[o] = sA;
    if (oC) oC[o] = sC;
    if (oWum) oWum[o] = sU;
    if (oWmm) oWmm[o] = sM;
  }
}

}  // namespace hm

using namespace hm;

namespace {
inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline int blocks_for(int64_t n, int per) { return (int)((n + per - 1) / per); }

// lattice node of element-local dof a of element e
inline int64_t lattice_node(const Lattice& L, int64_t e, int a) {
  const int64_t ex = e % L.nx, ey = (e / L.nx) % L.ny, ez = e / ((int64_t)L.nx * L.ny);
  return (2 * ex + a % 3) + (int64_t)L.Nx * ((2 * ey + (a / 3) % 3) + (int64_t)L.Ny * (2 * ez + a / 9));
}
}  // namespace

extern "C" int hm_lattice_dof_permutation(const hm_lattice* h, const int64_t* cdofs,
                                          const int32_t* local, int32_t* perm) {
  if (!h || !cdofs || !perm) return HM_ERR_ARG;
  const Lattice& L = *hm_lattice_geometry(h);
  int slot_of[27];
  bool used[27] = {false};
  for (int a = 0; a < 27; ++a) {
    slot_of[a] = local ? local[a] : a;
    if (slot_of[a] < 0 || slot_of[a] >= 27 || used[slot_of[a]]) return HM_ERR_ARG;
    used[slot_of[a]] = true;
  }
  for (int64_t n = 0; n < L.ndof; ++n) perm[n] = -1;
  for (int64_t e = 0; e < L.ne; ++e)
    for (int a = 0; a < 27; ++a) {
      const int64_t c = cdofs[e * 27 + slot_of[a]];
      if (c < 0 || c >= L.ndof) return HM_ERR_RANGE;
      int32_t& p = perm[lattice_node(L, e, a)];
      if (p == -1) p = (int32_t)c;
      else if (p != (int32_t)c) return HM_ERR_ARG;     // two dofs at one node
    }
  // a bijection: every node numbered (each lies in an element) and no dof used twice
  std::vector<char> seen(L.ndof, 0);
  for (int64_t n = 0; n < L.ndof; ++n) {
    if (perm[n] < 0 || seen[perm[n]]) return HM_ERR_ARG;
    seen[perm[n]] = 1;
  }
  return HM_OK;
}

extern "C" int hm_lattice_caller_map(const hm_lattice* h, const int32_t* d_perm,
                                     const int32_t* d_cindptr, const int32_t* d_cindices,
                                     int32_t* d_src_pos, uint32_t* d_status, void* stream) {
  if (!h || !d_perm || !d_cindptr || !d_cindices || !d_src_pos || !d_status) return HM_ERR_ARG;
  const Lattice& L = *hm_lattice_geometry(h);
  k_caller_map<<<blocks_for(L.ndof * 32, 256), 256, 0, S_(stream)>>>(L, d_perm, d_cindptr,
                                                                    d_cindices, d_src_pos, d_status);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

extern "C" int hm_gather_f64(int64_t n, const int32_t* d_idx, const double* d_src, double* d_dst,
                             void* stream) {
  if (n < 0 || (n > 0 && (!d_idx || !d_src || !d_dst)) || d_src == d_dst) return HM_ERR_ARG;
  if (n == 0) return HM_OK;
  const int64_t want = (n + 255) / 256;
  const int grid = (int)(want < 148 * 16 ? want : 148 * 16);
  k_gather_f64<<<grid, 256, 0, S_(stream)>>>(n, d_idx, d_src, d_dst);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

extern "C" int hm_lattice_element_blocks(const hm_lattice* h, const void* d_quad, int precision,
                                         int64_t e0, int64_t count, const int32_t* local,
                                         double* d_A, double* d_C, double* d_Wum, double* d_Wmm,
                                         void* stream) {
  if (!h || !d_quad) return HM_ERR_ARG;
  if (precision != HM_FP64 && precision != HM_FP32) return HM_ERR_ARG;
  const Lattice& L = *hm_lattice_geometry(h);
  if (e0 < 0 || count < 0 || e0 + count > L.ne || count > INT32_MAX) return HM_ERR_ARG;
  LocalOrder lo;
  bool used[27] = {false};
  for (int a = 0; a < 27; ++a) {
    lo.v[a] = local ? local[a] : a;
    if (lo.v[a] < 0 || lo.v[a] >= 27 || used[lo.v[a]]) return HM_ERR_ARG;
    used[lo.v[a]] = true;
  }
  if (count == 0 || !(d_A || d_C || d_Wum || d_Wmm)) return HM_OK;
  if (precision == HM_FP32)
    k_element_blocks<float><<<(int)count, 256, 0, S_(stream)>>>(L, (const float*)d_quad, e0, lo,
                                                                d_A, d_C, d_Wum, d_Wmm);
  else
    k_element_blocks<double><<<(int)count, 256, 0, S_(stream)>>>(L, (const double*)d_quad, e0, lo,
                                                                 d_A, d_C, d_Wum, d_Wmm);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
