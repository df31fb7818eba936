// Constant-exact single-precision blocks: the mixed-precision route of the reference's
// element kernel, consistent_block (hippymfem/fem/kernel.py:1503-1571).
//
// Each element matrix is contracted in single precision (FP32 pointwise data, FP32
// basis tables, FP32 sums) and then corrected, in FP64, by one rank-one term per side
// so that its products with the element's constants are the double-precision ones
// (the FP64 "tangents" along the constants, here single-index contractions against the
// FP64 sums of the basis tables):
//   d(a) = rs64(a) - sum_b K(a, b),   e(b) = cs64(b) - sum_a K(a, b)
//   two-sided (C, Wum):  K' = K + d(a)/27 + e(b)/27 - (sum d)/729
//   symmetric (A, Wmm):  K  = (K + K^T)/2 first, K' = K + (d(a) + d(b))/27 - (sum d)/729,
//                        both triangles taken from the upper one (symmetric to the bit)
// (the reference's K + Dj V + V^T Di^T - V^T (V Dj) V with V = 1/sqrt(27) [1 ... 1]).
// The corrected element matrices are then assembled into the lattice pattern by a
// gather: every CSR entry sums its (at most 8) element contributions in a fixed element
// order, so the assembly is deterministic and symmetric blocks stay symmetric to the
// bit; the folded elimination of the fused kernel follows.  Not the fast path (the
// fused FP64 and FP32 assemblies are): the route of the precision study, where the
// single-precision error of the C block's cancelling entries would otherwise stand.
#include "hm_common.cuh"
#include "hm_internal.h"

namespace hm {

enum { CB_A = 0, CB_C = 1, CB_WUM = 2, CB_WMM = 3 };

// One CTA per element: the corrected (27 x 27) matrix of block `blk` into out[e][729]
__global__ void __launch_bounds__(256) k_consistent_elements(Lattice L, const double* __restrict__ quad,
                                                             int blk, double* __restrict__ out) {
  __shared__ float n32[27][27], g32[3][27][27];     // [q][a] FP32 tables (physical gradients)
  __shared__ double s0[27], s1[3][27];              // FP64 sums over the basis at each point
  __shared__ double q64[216];
  __shared__ float q32[216];
  __shared__ double K[27][28];
  __shared__ double rs[27], cs[27], d[27], e[27];
  __shared__ double dsum;
  const int tid = threadIdx.x;
  const int64_t el = blockIdx.x;
  for (int t = tid; t < 216; t += blockDim.x) {
    const double v = quad[el * 216 + t];
    q64[t] = v;
    q32[t] = (float)v;
  }
  const double ih[3] = {1.0 / L.hx, 1.0 / L.hy, 1.0 / L.hz};
  for (int t = tid; t < 729; t += blockDim.x) {
    const int q = t / 27, a = t % 27;
    const int q1 = q % 3, q2 = (q / 3) % 3, q3 = q / 9;
    const int a1 = a % 3, a2 = (a / 3) % 3, a3 = a / 9;
    const double b1 = bq(q1, a1), b2 = bq(q2, a2), b3 = bq(q3, a3);
    n32[q][a] = (float)(b1 * b2 * b3);
    g32[0][q][a] = (float)(dbq(q1, a1) * b2 * b3 * ih[0]);
    g32[1][q][a] = (float)(b1 * dbq(q2, a2) * b3 * ih[1]);
    g32[2][q][a] = (float)(b1 * b2 * dbq(q3, a3) * ih[2]);
  }
  if (tid < 27) {
    // FP64 sums over the 27 basis functions at point q (1 and 0 up to rounding)
    const int q = tid, q1 = q % 3, q2 = (q / 3) % 3, q3 = q / 9;
    double s = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int a = 0; a < 27; ++a) {
      const int a1 = a % 3, a2 = (a / 3) % 3, a3 = a / 9;
      const double b1 = bq(q1, a1), b2 = bq(q2, a2), b3 = bq(q3, a3);
      s += b1 * b2 * b3;
      sx += dbq(q1, a1) * b2 * b3 * ih[0];
      sy += b1 * dbq(q2, a2) * b3 * ih[1];
      sz += b1 * b2 * dbq(q3, a3) * ih[2];
    }
    s0[q] = s; s1[0][q] = sx; s1[1][q] = sy; s1[2][q] = sz;
  }
  __syncthreads();
  // the single-precision element matrix
  for (int t = tid; t < 729; t += blockDim.x) {
    const int a = t / 27, b = t % 27;
    float acc = 0.0f;
    for (int q = 0; q < 27; ++q) {
      float v;
      if (blk == CB_A) {
        v = q32[q] * (g32[0][q][a] * g32[0][q][b] + g32[1][q][a] * g32[1][q][b] +
                      g32[2][q][a] * g32[2][q][b]);
      } else if (blk == CB_WMM) {
        v = q32[189 + q] * n32[q][a] * n32[q][b];
      } else {
        const int f = blk == CB_C ? 27 : 108;       // E (C) or F (Wum)
        v = (q32[f + q] * g32[0][q][a] + q32[f + 27 + q] * g32[1][q][a] +
             q32[f + 54 + q] * g32[2][q][a]) * n32[q][b];
      }
      acc += v;
    }
    K[a][b] = (double)acc;
  }
  // the FP64 tangents along the constants: row sums rs(a) = sum_b K64(a, b), column
  // sums cs(b) = sum_a K64(a, b), by single-index contractions
  if (tid < 54) {
    const int a = tid % 27;
    const bool col = tid >= 27;
    double acc = 0.0;
    for (int q = 0; q < 27; ++q) {
      const int q1 = q % 3, q2 = (q / 3) % 3, q3 = q / 9;
      const int a1 = a % 3, a2 = (a / 3) % 3, a3 = a / 9;
      const double b1 = bq(q1, a1), b2 = bq(q2, a2), b3 = bq(q3, a3);
      const double nq = b1 * b2 * b3;
      const double gq[3] = {dbq(q1, a1) * b2 * b3 * ih[0], b1 * dbq(q2, a2) * b3 * ih[1],
                            b1 * b2 * dbq(q3, a3) * ih[2]};
      double v;
      if (blk == CB_A) {
        v = q64[q] * (gq[0] * s1[0][q] + gq[1] * s1[1][q] + gq[2] * s1[2][q]);
      } else if (blk == CB_WMM) {
        v = q64[189 + q] * nq * s0[q];
      } else {
        const int f = blk == CB_C ? 27 : 108;
        // rows: (E . grad phi_a) sum_b psi_b; columns: (E . sum_a grad phi_a) psi_b
        v = col ? (q64[f + q] * s1[0][q] + q64[f + 27 + q] * s1[1][q] + q64[f + 54 + q] * s1[2][q]) * nq
                : (q64[f + q] * gq[0] + q64[f + 27 + q] * gq[1] + q64[f + 54 + q] * gq[2]) * s0[q];
      }
      acc += v;
    }
    if (col) cs[a] = acc;
    else rs[a] = acc;
  }
  __syncthreads();
  const bool sym = blk == CB_A || blk == CB_WMM;
  if (sym) {
    for (int t = tid; t < 729; t += blockDim.x) {
      const int a = t / 27, b = t % 27;
      if (a < b) {
        const double v = 0.5 * (K[a][b] + K[b][a]);
        K[a][b] = v;
        K[b][a] = v;
      }
    }
    __syncthreads();
  }
  if (tid < 54) {
    const int a = tid % 27;
    double s = 0.0;
    if (tid < 27) {
      for (int b = 0; b < 27; ++b) s += K[a][b];
      d[a] = rs[a] - s;
    } else {
      for (int b = 0; b < 27; ++b) s += K[b][a];
      e[a] = cs[a] - s;
    }
  }
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int a = 0; a < 27; ++a) s += d[a];
    dsum = s;
  }
  __syncthreads();
  double* o = out + el * 729;
  for (int t = tid; t < 729; t += blockDim.x) {
    const int a = t / 27, b = t % 27;
    double v;
    if (sym) {
      const int lo = a < b ? a : b, hi = a < b ? b : a;   // from the upper triangle
      v = K[lo][hi] + (d[lo] + d[hi]) / 27.0 - dsum / 729.0;
    } else {
      v = K[a][b] + d[a] / 27.0 + e[b] / 27.0 - dsum / 729.0;
    }
    o[t] = v;
  }
}

// the elements holding both node x and node y along one axis of n elements: [lo, hi]
__device__ __forceinline__ void common_elems(int x, int y, int n, int& lo, int& hi) {
  const int mx = x > y ? x : y, mn = x < y ? x : y;
  lo = (mx - 1) / 2;
  if (lo < 0) lo = 0;
  hi = mn / 2;
  if (hi > n - 1) hi = n - 1;
}

// One warp per lattice row: each CSR entry the sum of its element contributions
// (elements ascending), then the block's elimination policy
__global__ void k_consistent_assemble(Lattice L, const double* __restrict__ Ke, int blk,
                                      const uint8_t* __restrict__ ess, double* __restrict__ vals) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= L.ndof) return;
  const int i = (int)(row % L.Nx), j = (int)((row / L.Nx) % L.Ny), k = (int)(row / ((int64_t)L.Nx * L.Ny));
  const int n1 = stencil_n(i, L.Nx), n2 = stencil_n(j, L.Ny), n3 = stencil_n(k, L.Nz);
  const int lo1 = stencil_lo(i), lo2 = stencil_lo(j), lo3 = stencil_lo(k);
  const int kd = ((k - lo3) * n2 + (j - lo2)) * n1 + (i - lo1);
  const int len = n1 * n2 * n3;
  const int64_t base = row_start(L, i, j, k);
  const bool rfix = ess != nullptr && ess[row];
  for (int pos = lane; pos < len; pos += 32) {
    const int rank = pos == 0 ? kd : (pos <= kd ? pos - 1 : pos);
    const int k1 = rank % n1, t = rank / n1, k2 = t % n2, k3 = t / n2;
    const int ci = lo1 + k1, cj = lo2 + k2, ck = lo3 + k3;
    int a0, a1, b0, b1, c0, c1;
    common_elems(i, ci, L.nx, a0, a1);
    common_elems(j, cj, L.ny, b0, b1);
    common_elems(k, ck, L.nz, c0, c1);
    double acc = 0.0;
    for (int ez = c0; ez <= c1; ++ez)
      for (int ey = b0; ey <= b1; ++ey)
        for (int ex = a0; ex <= a1; ++ex) {
          const int64_t e = ex + (int64_t)L.nx * (ey + (int64_t)L.ny * ez);
          const int ra = (i - 2 * ex) + 3 * (j - 2 * ey) + 9 * (k - 2 * ez);
          const int cb = (ci - 2 * ex) + 3 * (cj - 2 * ey) + 9 * (ck - 2 * ez);
          acc += Ke[e * 729 + ra * 27 + cb];
        }
    if (ess != nullptr) {
      const int64_t col = ci + (int64_t)L.Nx * (cj + (int64_t)L.Ny * ck);
      if (blk == CB_A) {
        if (rfix || ess[col]) acc = (rfix && col == row) ? 1.0 : 0.0;
      } else if (blk != CB_WMM && rfix) {
        acc = 0.0;
      }
    }
    vals[base + pos] = acc;
  }
}

}  // namespace hm

using namespace hm;

extern "C" int64_t hm_lattice_consistent_workspace_bytes(const hm_lattice* h) {
  if (!h) return 0;
  return 8 * 729 * hm_lattice_geometry(h)->ne;
}

extern "C" int hm_lattice_assemble_consistent(const hm_lattice* h, const double* d_quad,
                                              const uint8_t* d_ess, double* d_vals_A,
                                              double* d_vals_C, double* d_vals_Wum,
                                              double* d_vals_Wmm, void* d_work, void* stream) {
  if (!h || !d_quad || !d_work) return HM_ERR_ARG;
  const Lattice& L = *hm_lattice_geometry(h);
  if (L.ne > INT32_MAX) return HM_ERR_UNSUPPORTED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  double* outs[4] = {d_vals_A, d_vals_C, d_vals_Wum, d_vals_Wmm};
  double* Ke = static_cast<double*>(d_work);
  for (int b = 0; b < 4; ++b) {
    if (!outs[b]) continue;
    k_consistent_elements<<<(int)L.ne, 256, 0, s>>>(L, d_quad, b, Ke);
    const int64_t threads = L.ndof * 32;
    k_consistent_assemble<<<(int)((threads + 255) / 256), 256, 0, s>>>(L, Ke, b, d_ess, outs[b]);
    if (cudaGetLastError() != cudaSuccess) return HM_ERR_CUDA;
  }
  return HM_OK;
}
