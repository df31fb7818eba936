// Shared definitions of the hippymfem_b200 kernels: status codes, the Q2 / 3-point
// Gauss tables and the structured-lattice geometry.
//
// The element is MFEM's Q2 H1 hexahedron (Lagrange nodes 0, 1/2, 1 along each axis),
// integrated with the 3x3x3 Gauss-Legendre rule in MFEM's tensor order (point (i,j,k)
// at i + 3 (j + 3 k)); the reference tabulates the same N / G tables in
// hippymfem/fem/elementbatch.py:509-525.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/hippymfem_b200.h"

#define HM_HD __host__ __device__ __forceinline__

namespace hm {

// ------------------------------------------------------------------ 1D Q2 at Gauss
// sqrt(3/5)/2 = sqrt(0.15): the Gauss points on [0, 1] are 1/2 - s, 1/2, 1/2 + s.
constexpr double kS = 0.3872983346207417;

// B(q, a): Lagrange basis a in {0, 1, 2} at Gauss point q in {0, 1, 2}.
HM_HD constexpr double bq(int q, int a) {
  return q == 1 ? (a == 1 ? 1.0 : 0.0)
       : a == 1 ? 0.4
       : ((q == 0) == (a == 0)) ? 0.3 + kS : 0.3 - kS;
}
// dB(q, a): derivative of basis a at Gauss point q.
HM_HD constexpr double dbq(int q, int a) {
  return q == 1 ? (a == 0 ? -1.0 : a == 1 ? 0.0 : 1.0)
       : a == 1 ? (q == 0 ? 8.0 * kS : -8.0 * kS)
       : a == 0 ? (q == 0 ? -1.0 - 4.0 * kS : -1.0 + 4.0 * kS)
                : (q == 0 ? 1.0 - 4.0 * kS : 1.0 + 4.0 * kS);
}
// Gauss weight on [0, 1].
HM_HD constexpr double wq(int q) { return q == 1 ? 8.0 / 18.0 : 5.0 / 18.0; }

// ------------------------------------------------------- tile of 4 x 4 x 4 rows
// A tile owns node rows 4t .. 4t+3 along each axis.  Its halo'd elements are
// 2t-1, 2t, 2t+1 (local l = 0, 1, 2), whose nodes are 4t-2 .. 4t+4 (local s = 0..6)
// and whose quadrature points are local g = 3 l + q (0..8).  Owned row r is local
// node s = r + 2.  Along one axis, row r couples to the columns of its stencil:
//   r = 0 (vertex 4t):   s' = 0..4     r = 1 (mid):   s' = 2..4
//   r = 2 (vertex 4t+2): s' = 2..6     r = 3 (mid):   s' = 4..6
// giving 16 ordered 1D pairs p = (row, column).  A pair's support is the quadrature
// points of the elements that hold both nodes: 6 points for a vertex with itself,
// 3 otherwise.
HM_HD constexpr int row_pair_base(int r) { return r == 0 ? 0 : r == 1 ? 5 : r == 2 ? 8 : 13; }
HM_HD constexpr int row_stencil(int r) { return (r & 1) ? 3 : 5; }
HM_HD constexpr int row_col_start(int r) { return r == 0 ? 0 : r == 3 ? 4 : 2; }
HM_HD constexpr int pair_row_of(int p) { return p < 5 ? 0 : p < 8 ? 1 : p < 13 ? 2 : 3; }
HM_HD constexpr int pair_s(int p) { return pair_row_of(p) + 2; }
HM_HD constexpr int pair_c(int p) { return row_col_start(pair_row_of(p)) + (p - row_pair_base(pair_row_of(p))); }
// the first element holding both nodes of a pair: the left element of the upper node
HM_HD constexpr int lo_elem(int s, int c) {
  return ((s < c ? c : s) - 1) / 2;
}
HM_HD constexpr bool both_vertex_same(int s, int c) { return s == c && (s & 1) == 0; }
HM_HD constexpr int pair_g0(int p) {
  return both_vertex_same(pair_s(p), pair_c(p)) ? 3 * (pair_s(p) / 2 - 1)
                                                : 3 * lo_elem(pair_s(p), pair_c(p));
}
HM_HD constexpr int pair_cnt(int p) { return both_vertex_same(pair_s(p), pair_c(p)) ? 6 : 3; }

// 1D pair tables: M = B(row) B(col), K = B'(row) B'(col), R = B'(row) B(col),
// C = B(row) B'(col), at the t-th support point of pair p.
enum Tab { TM = 0, TK = 1, TR = 2, TC = 3 };
HM_HD constexpr double pair_coef(int tab, int p, int t) {
  return tab == TM ? bq((pair_g0(p) + t) % 3, pair_s(p) - 2 * ((pair_g0(p) + t) / 3)) *
                         bq((pair_g0(p) + t) % 3, pair_c(p) - 2 * ((pair_g0(p) + t) / 3))
       : tab == TK ? dbq((pair_g0(p) + t) % 3, pair_s(p) - 2 * ((pair_g0(p) + t) / 3)) *
                         dbq((pair_g0(p) + t) % 3, pair_c(p) - 2 * ((pair_g0(p) + t) / 3))
       : tab == TR ? dbq((pair_g0(p) + t) % 3, pair_s(p) - 2 * ((pair_g0(p) + t) / 3)) *
                         bq((pair_g0(p) + t) % 3, pair_c(p) - 2 * ((pair_g0(p) + t) / 3))
                   : bq((pair_g0(p) + t) % 3, pair_s(p) - 2 * ((pair_g0(p) + t) / 3)) *
                         dbq((pair_g0(p) + t) % 3, pair_c(p) - 2 * ((pair_g0(p) + t) / 3));
}

// Single-index (vector) tables for owned row r: support and B / B' of its node.
HM_HD constexpr int vrow_g0(int r) { return (r & 1) ? 3 * ((r + 1) / 2) : 3 * (r / 2); }
HM_HD constexpr int vrow_cnt(int r) { return (r & 1) ? 3 : 6; }
enum VTab { VB = 0, VD = 1 };
HM_HD constexpr double vrow_coef(int tab, int r, int t) {
  return tab == VB ? bq((vrow_g0(r) + t) % 3, r + 2 - 2 * ((vrow_g0(r) + t) / 3))
                   : dbq((vrow_g0(r) + t) % 3, r + 2 - 2 * ((vrow_g0(r) + t) / 3));
}

// ------------------------------------------------------------------ lattice
struct Lattice {
  int nx, ny, nz;      // elements per axis
  int Nx, Ny, Nz;      // nodes per axis (2 n + 1)
  int tx, ty, tz;      // tiles per axis (ceil(N / 4))
  double hx, hy, hz;   // element sizes
  int64_t ne, ndof;
};

// 1D stencil of node i on an axis of N nodes: [lo, lo + n)
HM_HD int stencil_lo(int i) { return (i & 1) ? i - 1 : (i >= 2 ? i - 2 : 0); }
HM_HD int stencil_n(int i, int N) {
  if (i & 1) return 3;
  const int lo = i >= 2 ? i - 2 : 0;
  const int hi = i + 2 <= N - 1 ? i + 2 : N - 1;
  return hi - lo + 1;
}
// number of 1D (row, column) pairs of the rows before node i
HM_HD int64_t stencil_prefix(int i, int N) {
  // vertex rows 2k (k >= 1, not last) hold 5, mid rows 3, the first and last vertex 3
  // (when N >= 3); C(2k) = 8k - 2 for k >= 1
  if (i == 0) return 0;
  const int k = i / 2;
  const int64_t even = k >= 1 ? 8 * (int64_t)k - 2 : 0;
  return (i & 1) ? even + stencil_n(2 * k, N) : even;
}
// CSR offset of row (i, j, k) of the lattice pattern (rows in node order)
HM_HD int64_t row_start(const Lattice& L, int i, int j, int k) {
  const int64_t T1 = stencil_prefix(L.Nx, L.Nx), T2 = stencil_prefix(L.Ny, L.Ny);
  return stencil_prefix(k, L.Nz) * T1 * T2 +
         (int64_t)stencil_n(k, L.Nz) *
             (stencil_prefix(j, L.Ny) * T1 + (int64_t)stencil_n(j, L.Ny) * stencil_prefix(i, L.Nx));
}

// ------------------------------------------------------------ PCG device scalars
// (shared by the solver and the operator kernels that finish a CG step's reductions)
enum { SC_RZ = 0, SC_PQ, SC_ALPHA, SC_BETA, SC_RR, SC_BB, SC_TOL2, SC_CONV, SC_TMP0, SC_TMP1,
       SC_TMP2, SC_IT, SC_N };

#ifdef __CUDACC__
// sum over the block (valid in thread 0); every thread of the block must call it
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
  return t;
}

// After thread 0 of every block has written its partial: true in the block that
// finishes last (block-uniform).  The partials it then reads are complete; the
// counter is reset by that block.  Which block is last does not change any result:
// it sums the partials in a fixed order.
__device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  return last;
}

// alpha = r.z / p.q from the p.q partials (the last block of the product)
__device__ __forceinline__ void finish_alpha(const double* part, unsigned nparts, double* sc,
                                             unsigned* counter, double* sh) {
  double t = 0.0;
  for (unsigned b = threadIdx.x; b < nparts; b += blockDim.x) t += __ldcg(part + b);
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    sc[SC_PQ] = t;
    const double a = sc[SC_RZ] / t;
    sc[SC_ALPHA] = (sc[SC_CONV] >= 0.0 || t == 0.0 || !isfinite(a)) ? 0.0 : a;
    *counter = 0u;
  }
}
#endif

}  // namespace hm
