// Structured-lattice kernels of the Q2 log-conductivity path (sm_100a).
//
//   k_pattern_*     the CSR graph (diagonal first), the entry->slot map and the
//                   transpose map of a Q2 x Q2 block, arithmetically
//   k_quad          pointwise data D, E = D grad u, F = D grad p, W = D grad u.grad p
//   k_elem_apply,   the matrix-free Jacobian apply
//   k_node_gather
// (the fused assembly k_tile_assemble is in hm_tile.cu)
#include <cstdio>

#include "hm_common.cuh"
#include "hm_internal.h"

namespace hm {

// =============================================================== pattern kernels
__device__ __forceinline__ void node_of(int64_t n, const Lattice& L, int& i, int& j, int& k) {
  i = (int)(n % L.Nx);
  const int64_t t = n / L.Nx;
  j = (int)(t % L.Ny);
  k = (int)(t / L.Ny);
}

// CSR position of column (ci, cj, ck) within row (i, j, k): diagonal first, the rest
// ascending (ascending lexicographic node number = z, then y, then x rank)
__device__ __forceinline__ int pos_in_row(const Lattice& L, int i, int j, int k, int ci,
                                          int cj, int ck) {
  const int n1 = stencil_n(i, L.Nx), n2 = stencil_n(j, L.Ny);
  const int rank = ((ck - stencil_lo(k)) * n2 + (cj - stencil_lo(j))) * n1 + (ci - stencil_lo(i));
  const int kd = ((k - stencil_lo(k)) * n2 + (j - stencil_lo(j))) * n1 + (i - stencil_lo(i));
  return rank == kd ? 0 : (rank < kd ? rank + 1 : rank);
}

__global__ void k_pattern_indptr(Lattice L, int32_t* __restrict__ indptr) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n > L.ndof) return;
  if (n == L.ndof) {
    indptr[n] = (int32_t)(stencil_prefix(L.Nx, L.Nx) * stencil_prefix(L.Ny, L.Ny) *
                          stencil_prefix(L.Nz, L.Nz));
    return;
  }
  int i, j, k;
  node_of(n, L, i, j, k);
  indptr[n] = (int32_t)row_start(L, i, j, k);
}

// one warp per row: the row's columns in CSR order
__global__ void k_pattern_indices(Lattice L, const int32_t* __restrict__ indptr,
                                  int32_t* __restrict__ indices) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= L.ndof) return;
  int i, j, k;
  node_of(row, L, i, j, k);
  const int n1 = stencil_n(i, L.Nx), n2 = stencil_n(j, L.Ny), n3 = stencil_n(k, L.Nz);
  const int lo1 = stencil_lo(i), lo2 = stencil_lo(j), lo3 = stencil_lo(k);
  const int kd = ((k - lo3) * n2 + (j - lo2)) * n1 + (i - lo1);
  const int len = n1 * n2 * n3;
  const int64_t base = indptr[row];
  for (int pos = lane; pos < len; pos += 32) {
    const int rank = pos == 0 ? kd : (pos <= kd ? pos - 1 : pos);
    const int k1 = rank % n1, t = rank / n1, k2 = t % n2, k3 = t / n2;
    indices[base + pos] = (int32_t)((lo1 + k1) + (int64_t)L.Nx * ((lo2 + k2) + (int64_t)L.Ny * (lo3 + k3)));
  }
}

// entry k = (e*27 + a)*27 + b -> CSR position (patternbuild.build_tables' slot)
__global__ void k_pattern_slot(Lattice L, int32_t* __restrict__ slot) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= L.ne * 729) return;
  const int b = (int)(k % 27);
  const int a = (int)((k / 27) % 27);
  const int64_t e = k / 729;
  const int ex = (int)(e % L.nx), ey = (int)((e / L.nx) % L.ny), ez = (int)(e / ((int64_t)L.nx * L.ny));
  const int i = 2 * ex + a % 3, j = 2 * ey + (a / 3) % 3, kk = 2 * ez + a / 9;
  const int ci = 2 * ex + b % 3, cj = 2 * ey + (b / 3) % 3, ck = 2 * ez + b / 9;
  slot[k] = (int32_t)(row_start(L, i, j, kk) + pos_in_row(L, i, j, kk, ci, cj, ck));
}

// tpos[s] = CSR position of (col, row) for entry s = (row, col)
__global__ void k_pattern_tpos(Lattice L, const int32_t* __restrict__ indptr,
                               int32_t* __restrict__ tpos) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= L.ndof) return;
  int i, j, k;
  node_of(row, L, i, j, k);
  const int n1 = stencil_n(i, L.Nx), n2 = stencil_n(j, L.Ny), n3 = stencil_n(k, L.Nz);
  const int lo1 = stencil_lo(i), lo2 = stencil_lo(j), lo3 = stencil_lo(k);
  const int kd = ((k - lo3) * n2 + (j - lo2)) * n1 + (i - lo1);
  const int len = n1 * n2 * n3;
  const int64_t base = indptr[row];
  for (int pos = lane; pos < len; pos += 32) {
    const int rank = pos == 0 ? kd : (pos <= kd ? pos - 1 : pos);
    const int k1 = rank % n1, t = rank / n1, k2 = t % n2, k3 = t / n2;
    const int ci = lo1 + k1, cj = lo2 + k2, ck = lo3 + k3;
    tpos[base + pos] = (int32_t)(row_start(L, ci, cj, ck) + pos_in_row(L, ci, cj, ck, i, j, k));
  }
}

// ============================================================ quadrature data
// One thread per (element, Gauss point), 8 elements per 216-thread block.  Layout:
// quad[e][c][q], c = 0 D, 1-3 E, 4-6 F, 7 W (each element's 216 values contiguous).
// With mhat, D = w|J| e^m mhat: the data of the directional derivative along mhat
// (the second-order products of the assembled vectors, with f = 0).
template <typename real>
__global__ void __launch_bounds__(216) k_quad(Lattice L, const double* __restrict__ u,
                                              const double* __restrict__ m,
                                              const double* __restrict__ p,
                                              const double* __restrict__ mhat,
                                              real* __restrict__ quad,
                                              uint32_t* __restrict__ status) {
  __shared__ real sv[8][4][27];
  const int le = threadIdx.x / 27, q = threadIdx.x % 27;
  const int64_t e = blockIdx.x * 8LL + le;
  const bool live = e < L.ne;
  if (live) {
    const int ex = (int)(e % L.nx), ey = (int)((e / L.nx) % L.ny), ez = (int)(e / ((int64_t)L.nx * L.ny));
    const int a = q;
    const int64_t node = (2 * ex + a % 3) + (int64_t)L.Nx * ((2 * ey + (a / 3) % 3) + (int64_t)L.Ny * (2 * ez + a / 9));
    sv[le][0][a] = (real)u[node];
    sv[le][1][a] = (real)m[node];
    sv[le][2][a] = (real)p[node];
    if (mhat) sv[le][3][a] = (real)mhat[node];
  }
  __syncthreads();
  if (!live) return;
  const int q1 = q % 3, q2 = (q / 3) % 3, q3 = q / 9;
  real b1[3], b2[3], b3[3], d1[3], d2[3], d3[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    b1[a] = (real)bq(q1, a); b2[a] = (real)bq(q2, a); b3[a] = (real)bq(q3, a);
    d1[a] = (real)dbq(q1, a); d2[a] = (real)dbq(q2, a); d3[a] = (real)dbq(q3, a);
  }
  real val[3], gx[3], gy[3], gz[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const real* x = sv[le][f];
    real vb = 0, vx = 0, vy = 0, vz = 0;
#pragma unroll
    for (int a3 = 0; a3 < 3; ++a3) {
      real sbb = 0, sdb = 0, sbd = 0;
#pragma unroll
      for (int a2 = 0; a2 < 3; ++a2) {
        real xb = 0, xd = 0;
#pragma unroll
        for (int a1 = 0; a1 < 3; ++a1) {
          xb = fma(b1[a1], x[a1 + 3 * a2 + 9 * a3], xb);
          xd = fma(d1[a1], x[a1 + 3 * a2 + 9 * a3], xd);
        }
        sbb = fma(b2[a2], xb, sbb);
        sdb = fma(b2[a2], xd, sdb);
        sbd = fma(d2[a2], xb, sbd);
      }
      vb = fma(b3[a3], sbb, vb);
      vx = fma(b3[a3], sdb, vx);
      vy = fma(b3[a3], sbd, vy);
      vz = fma(d3[a3], sbb, vz);
    }
    val[f] = vb;
    gx[f] = vx / (real)L.hx;
    gy[f] = vy / (real)L.hy;
    gz[f] = vz / (real)L.hz;
  }
  const real wdet = (real)(wq(q1) * wq(q2) * wq(q3) * L.hx * L.hy * L.hz);
  real D = wdet * exp(val[1]);
  if (mhat) {
    // mhat at the point (value only)
    const real* x = sv[le][3];
    real vb = 0;
#pragma unroll
    for (int a3 = 0; a3 < 3; ++a3) {
      real sbb = 0;
#pragma unroll
      for (int a2 = 0; a2 < 3; ++a2) {
        real xb = 0;
#pragma unroll
        for (int a1 = 0; a1 < 3; ++a1) xb = fma(b1[a1], x[a1 + 3 * a2 + 9 * a3], xb);
        sbb = fma(b2[a2], xb, sbb);
      }
      vb = fma(b3[a3], sbb, vb);
    }
    D *= vb;
  }
  const real E[3] = {D * gx[0], D * gy[0], D * gz[0]};
  const real F[3] = {D * gx[2], D * gy[2], D * gz[2]};
  const real W = D * (gx[0] * gx[2] + gy[0] * gy[2] + gz[0] * gz[2]);
  real* out = quad + e * 216;
  out[q] = D;
  out[27 + q] = E[0]; out[54 + q] = E[1]; out[81 + q] = E[2];
  out[108 + q] = F[0]; out[135 + q] = F[1]; out[162 + q] = F[2];
  out[189 + q] = W;
  const bool finite = isfinite(D) && isfinite(E[0]) && isfinite(E[1]) && isfinite(E[2]) &&
                      isfinite(F[0]) && isfinite(F[1]) && isfinite(F[2]) && isfinite(W);
  if (!finite) atomicOr(status, HM_STATUS_NONFINITE);
}

// ====================================================== matrix-free Jacobian apply
// y = A(D) x in two deterministic passes:
//   k_elem_apply   three threads per element, thread t owning Gauss slice q3 = t:
//                  x at the element's nodes -> gradients at the slice's 9 points (sum
//                  factorisation in registers) -> flux D grad x / h^2 -> back to the
//                  element's nodes; the three slices' contributions are combined with
//                  warp shuffles and y_e written in SoA layout Ye[a][e]
//   k_node_gather  one thread per node: the sum of its <= 8 element contributions in a
//                  fixed order; y = x on Dirichlet nodes (the Jacobian's elimination,
//                  x zeroed there on input)
// D is kept in SoA layout Dq[q][e] (hm_lattice_jacobian_prepare), so both passes read
// and write coalesced.

template <typename src, typename real>
__global__ void k_extract_D(Lattice L, const src* __restrict__ quad, real* __restrict__ Dq) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= L.ne * 27) return;
  const int64_t e = i / 27;
  const int q = (int)(i - e * 27);
  Dq[(int64_t)q * L.ne + e] = (real)quad[e * 216 + q];
}

// B(q, a) and B'(q, a) for a run-time point index q (a compile-time)
template <typename real>
__device__ __forceinline__ real bq_rt(int q, int a) {
  return q == 0 ? (real)bq(0, a) : q == 1 ? (real)bq(1, a) : (real)bq(2, a);
}
template <typename real>
__device__ __forceinline__ real dbq_rt(int q, int a) {
  return q == 0 ? (real)dbq(0, a) : q == 1 ? (real)dbq(1, a) : (real)dbq(2, a);
}

// ESS: zero x on the Dirichlet nodes on the fly (callers whose x is already zero there
// -- every vector inside the lattice solves -- skip the markers).  CHEB: the input is the
// first Chebyshev direction d = b idiag / theta of a smoother started from zero, formed
// on the fly from b (xin), the reciprocal Jacobi diagonal (cdiag) and theta = cheb[0].
template <typename real, typename vec, bool ESS = true, bool CHEB = false>
__global__ void __launch_bounds__(256, 2)
    k_elem_apply(Lattice L, const real* __restrict__ Dq, const uint8_t* __restrict__ ess,
                 const vec* __restrict__ xin, real* __restrict__ Ye,
                 const double* __restrict__ cdiag = nullptr, const double* __restrict__ cheb = nullptr) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int k = lane / 3, t = lane - 3 * k;                 // element slot, Gauss slice
  const int64_t e = warp * 10 + k;
  const bool live = lane < 30 && e < L.ne;
  // 32-bit decode (the lattice keeps every index below 2^31)
  const unsigned ec = live ? (unsigned)e : 0u;
  const unsigned exy = ec / (unsigned)L.nx;
  const int ex = (int)(ec - exy * (unsigned)L.nx);
  const int ez = (int)(exy / (unsigned)L.ny), ey = (int)(exy - (unsigned)ez * (unsigned)L.ny);
  const unsigned n0 = (unsigned)(2 * ex) + (unsigned)L.Nx * ((unsigned)(2 * ey) + (unsigned)L.Ny * (unsigned)(2 * ez));
  const unsigned nsy = (unsigned)L.Nx, nsz = (unsigned)L.Nx * (unsigned)L.Ny;
  const double inv_theta = CHEB ? 1.0 / __ldg(cheb) : 0.0;
  // z interpolation onto slice t, one node plane a3 at a time: Xb[a2][a1], Xd[a2][a1]
  real Xb[9], Xd[9];
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3) {
    const real b3 = bq_rt<real>(t, a3), d3 = dbq_rt<real>(t, a3);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const unsigned n = n0 + (unsigned)(i % 3) + nsy * (unsigned)(i / 3) + nsz * (unsigned)a3;
      real xv = (real)0;
      if (live) {
        if constexpr (CHEB) xv = (real)__dmul_rn(inv_theta * (double)__ldg(xin + n), __ldg(cdiag + n));
        else xv = (real)__ldg(xin + n);
      }
      const bool fixed = ESS && ess != nullptr && live && __ldg(ess + n) != 0;
      const real x = fixed ? (real)0 : xv;
      Xb[i] = a3 == 0 ? b3 * x : fma(b3, x, Xb[i]);
      Xd[i] = a3 == 0 ? d3 * x : fma(d3, x, Xd[i]);
    }
  }
  const real sx = (real)(1.0 / (L.hx * L.hx)), sy = (real)(1.0 / (L.hy * L.hy)),
             sz = (real)(1.0 / (L.hz * L.hz));
  // gradients and fluxes at the slice's points, folded straight back along x:
  // Z0[a1][q2] = sum_q1 B'(q1,a1) Fx,  Z1 = sum B Fy,  Z2 = sum B Fz
  real Z0[9], Z1[9], Z2[9];
#pragma unroll
  for (int q2 = 0; q2 < 3; ++q2) {
    real bb[3], db[3], bd[3];
#pragma unroll
    for (int a1 = 0; a1 < 3; ++a1) {
      bb[a1] = (real)bq(q2, 0) * Xb[a1] + (real)bq(q2, 1) * Xb[a1 + 3] + (real)bq(q2, 2) * Xb[a1 + 6];
      db[a1] = (real)dbq(q2, 0) * Xb[a1] + (real)dbq(q2, 1) * Xb[a1 + 3] + (real)dbq(q2, 2) * Xb[a1 + 6];
      bd[a1] = (real)bq(q2, 0) * Xd[a1] + (real)bq(q2, 1) * Xd[a1 + 3] + (real)bq(q2, 2) * Xd[a1 + 6];
    }
#pragma unroll
    for (int a1 = 0; a1 < 3; ++a1) { Z0[a1 * 3 + q2] = 0; Z1[a1 * 3 + q2] = 0; Z2[a1 * 3 + q2] = 0; }
#pragma unroll
    for (int q1 = 0; q1 < 3; ++q1) {
      const real gx = (real)dbq(q1, 0) * bb[0] + (real)dbq(q1, 1) * bb[1] + (real)dbq(q1, 2) * bb[2];
      const real gy = (real)bq(q1, 0) * db[0] + (real)bq(q1, 1) * db[1] + (real)bq(q1, 2) * db[2];
      const real gz = (real)bq(q1, 0) * bd[0] + (real)bq(q1, 1) * bd[1] + (real)bq(q1, 2) * bd[2];
      const real d = live ? Dq[(int64_t)(q1 + 3 * q2 + 9 * t) * L.ne + ec] : (real)0;  // coalesced in e
      const real fx = d * gx * sx, fy = d * gy * sy, fz = d * gz * sz;
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
        Z0[a1 * 3 + q2] = fma((real)dbq(q1, a1), fx, Z0[a1 * 3 + q2]);
        Z1[a1 * 3 + q2] = fma((real)bq(q1, a1), fy, Z1[a1 * 3 + q2]);
        Z2[a1 * 3 + q2] = fma((real)bq(q1, a1), fz, Z2[a1 * 3 + q2]);
      }
    }
  }
  // back along y: UB[a2][a1] = sum_q2 B(q2,a2) Z0 + B'(q2,a2) Z1,  UD = sum_q2 B(q2,a2) Z2
  real UB[9], UD[9];
#pragma unroll
  for (int a2 = 0; a2 < 3; ++a2)
#pragma unroll
    for (int a1 = 0; a1 < 3; ++a1) {
      real ub = 0, ud = 0;
#pragma unroll
      for (int q2 = 0; q2 < 3; ++q2) {
        ub = fma((real)bq(q2, a2), Z0[a1 * 3 + q2], ub);
        ub = fma((real)dbq(q2, a2), Z1[a1 * 3 + q2], ub);
        ud = fma((real)bq(q2, a2), Z2[a1 * 3 + q2], ud);
      }
      UB[a2 * 3 + a1] = ub;
      UD[a2 * 3 + a1] = ud;
    }
  // back along z: thread t owns node plane a3 = t and sums the three slices' parts,
  // slice order 0, 1, 2 (fixed)
  real y[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) y[i] = 0;
  const int base = 3 * k;
#pragma unroll
  for (int src = 0; src < 3; ++src) {
    const real cb = bq_rt<real>(src, 0) * (t == 0) + bq_rt<real>(src, 1) * (t == 1) + bq_rt<real>(src, 2) * (t == 2);
    const real cd = dbq_rt<real>(src, 0) * (t == 0) + dbq_rt<real>(src, 1) * (t == 1) + dbq_rt<real>(src, 2) * (t == 2);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const real ub = __shfl_sync(0xffffffffu, UB[i], base + src);
      const real ud = __shfl_sync(0xffffffffu, UD[i], base + src);
      y[i] = fma(cb, ub, fma(cd, ud, y[i]));
    }
  }
  if (live) {
#pragma unroll
    for (int i = 0; i < 9; ++i) Ye[(int64_t)(i + 9 * t) * L.ne + e] = y[i];
  }
}

// One thread per pair of x-neighbours (2m, 2m+1) of a node row (the row's last node,
// 2n, alone), so that every lane of a warp runs the same loop: node 2m takes element
// m-1 (local a1 = 2) and m (a1 = 0), node 2m+1 element m (a1 = 1); consecutive lanes
// read consecutive elements of each Ye plane.  Per node the contributions are summed
// over (z, y, x) element pairs with the lower element first, a fixed order.  With part
// != nullptr each block also writes its partial sum of dotw . y (the p.q of a CG step).
__device__ __forceinline__ void axis_elems(int i, int nel, int& e0, int& a0, int& cnt) {
  if (i & 1) { e0 = i >> 1; a0 = 1; cnt = 1; }
  else if (i == 0) { e0 = 0; a0 = 0; cnt = 1; }
  else if ((i >> 1) >= nel) { e0 = (i >> 1) - 1; a0 = 2; cnt = 1; }
  else { e0 = (i >> 1) - 1; a0 = 2; cnt = 2; }   // elements i/2-1 (a=2), i/2 (a=0)
}

// OUT selects what is written for each node's product y (FP64 only for OUT != 0), with
// c.b the smoother's right-hand side, c.diag the reciprocal of the Jacobi diagonal,
// theta = c.cheb[0]:
//   0  yout = y
//   1  the first smoothing step from zero (the input was d = b c.diag / theta):
//      c.r = b - y, c.x = d
//   2  one smoothing step from c.x (the input): c.x += (b - y) c.diag / theta, in place,
//      or into c.z (FP64) when given (this pass reads no x but the Dirichlet nodes' own)
//   3  as 1 with d already in c.x (the input): c.r = b - y
// c.r and c.x are in the vector type V (the updates are formed in FP64 and rounded once)
template <typename V>
struct ChebOutT {
  const double* b;
  const double* diag;
  const double* cheb;
  V* r;
  V* x;
  double* z;
};
using ChebOut = ChebOutT<double>;
template <typename real, typename vec, int OUT = 0>
__global__ void __launch_bounds__(256)
    k_node_gather(Lattice L, const real* __restrict__ Ye, const uint8_t* __restrict__ ess,
                  const vec* __restrict__ xin, vec* __restrict__ yout,
                  const vec* __restrict__ dotw, double* __restrict__ part,
                  double* __restrict__ sc, unsigned* __restrict__ counter, ChebOutT<vec> c = {},
                  const uint32_t* __restrict__ skip = nullptr) {
  if (skip != nullptr && *skip != 0u) return;    // the whole launch stands down
  const unsigned per_row = (unsigned)L.nx + 1u;                  // pairs + the last node
  const unsigned rows = (unsigned)L.Ny * (unsigned)L.Nz;
  const unsigned task = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = task < rows * per_row;
  const unsigned row = live ? task / per_row : 0u;
  const unsigned m = live ? task - row * per_row : 0u;
  const unsigned iz = row / (unsigned)L.Ny, iy = row - iz * (unsigned)L.Ny;
  const bool last = m == (unsigned)L.nx;                          // node 2n alone
  const unsigned n0 = row * (unsigned)L.Nx + 2u * m;              // node 2m
  double dot = 0.0;
  if (live) {
    int ey0, ay0, cy, ez0, az0, cz;
    axis_elems((int)iy, L.ny, ey0, ay0, cy);
    axis_elems((int)iz, L.nz, ez0, az0, cz);
    const unsigned ne = (unsigned)L.ne, nx = (unsigned)L.nx;
    const bool f0 = ess != nullptr && ess[n0];
    const bool f1 = !last && ess != nullptr && ess[n0 + 1];
    // every contribution is loaded before any is added (all twelve loads in flight at
    // once), then summed in the fixed order (z, y element pairs, lower element first)
    real v[4][3];
#pragma unroll
    for (int c3 = 0; c3 < 2; ++c3)
#pragma unroll
      for (int c2 = 0; c2 < 2; ++c2) {
        const int c = 2 * c3 + c2;
        const bool on = c3 < cz && c2 < cy;
        const unsigned a23 = 3u * (unsigned)(c2 ? 0 : ay0) + 9u * (unsigned)(c3 ? 0 : az0);
        const unsigned erow = nx * ((unsigned)(ey0 + c2) + (unsigned)L.ny * (unsigned)(ez0 + c3));
        // node 2m: element m-1 (a1 = 2) then element m (a1 = 0); node 2m+1: element m
        v[c][0] = (on && m > 0) ? Ye[(size_t)(2u + a23) * ne + erow + m - 1u] : (real)0;
        v[c][1] = (on && !last) ? Ye[(size_t)a23 * ne + erow + m] : (real)0;
        v[c][2] = (on && !last) ? Ye[(size_t)(1u + a23) * ne + erow + m] : (real)0;
      }
    real acc0 = 0, acc1 = 0;
#pragma unroll
    for (int c3 = 0; c3 < 2; ++c3)
#pragma unroll
      for (int c2 = 0; c2 < 2; ++c2) {
        const int c = 2 * c3 + c2;
        if (c3 < cz && c2 < cy) {
          if (m > 0) acc0 += v[c][0];
          if (!last) {
            acc0 += v[c][1];
            acc1 += v[c][2];
          }
        }
      }
    if constexpr (OUT == 0) {
      const double y0 = f0 ? (double)xin[n0] : (double)acc0;
      yout[n0] = (vec)y0;
      if (dotw) dot = (double)dotw[n0] * y0;
      if (!last) {
        const double y1 = f1 ? (double)xin[n0 + 1] : (double)acc1;
        yout[n0 + 1] = (vec)y1;
        if (dotw) dot = fma((double)dotw[n0 + 1], y1, dot);
      }
    } else {
      const double inv_theta = 1.0 / c.cheb[0];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (h == 1 && last) break;
        const unsigned nn = n0 + (unsigned)h;
        const bool fx = h ? f1 : f0;
        const double acc = (double)(h ? acc1 : acc0);
        const double bn = c.b[nn];
        if constexpr (OUT == 1) {
          const double d = __dmul_rn(inv_theta * bn, c.diag[nn]);
          const double y = fx ? (double)(vec)d : acc;
          c.r[nn] = (vec)(bn - y);
          c.x[nn] = (vec)d;
        } else if constexpr (OUT == 3) {
          const double y = fx ? (double)c.x[nn] : acc;
          c.r[nn] = (vec)(bn - y);
        } else {
          const double xn = (double)c.x[nn];
          const double y = fx ? xn : acc;
          // the update rounded on its own before the add, as the step-by-step smoother
          const double xnew = xn + __dmul_rn(inv_theta * (bn - y), c.diag[nn]);
          if (c.z != nullptr) c.z[nn] = xnew;
          else c.x[nn] = (vec)xnew;
        }
      }
    }
  }
  if (part != nullptr) {
    __shared__ double sh[32];
    double v = dot;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      double t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
    // a CG step: the last block takes alpha from the partials
    if (sc != nullptr && last_block(counter)) finish_alpha(part, gridDim.x, sc, counter, sh);
  }
}

// diagonal of A(D): sum_g D(g) sum_d (d_d phi_n)^2, one thread per node
template <typename real>
__global__ void k_diag_A(Lattice L, const real* __restrict__ quad, const uint8_t* __restrict__ ess,
                         double* __restrict__ diag) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= L.ndof) return;
  const int i = (int)(n % L.Nx), j = (int)((n / L.Nx) % L.Ny), k = (int)(n / ((int64_t)L.Nx * L.Ny));
  if (ess != nullptr && ess[n]) { diag[n] = 1.0; return; }
  const int gi[3] = {i, j, k};
  const int ne[3] = {L.nx, L.ny, L.nz};
  const double h2[3] = {1.0 / (L.hx * L.hx), 1.0 / (L.hy * L.hy), 1.0 / (L.hz * L.hz)};
  // elements touching the node along each axis
  int el0[3], nel[3];
  for (int d = 0; d < 3; ++d) {
    if (gi[d] & 1) { el0[d] = gi[d] / 2; nel[d] = 1; }
    else {
      el0[d] = gi[d] / 2 - 1; nel[d] = 2;
      if (el0[d] < 0) { el0[d] = 0; nel[d] = 1; }
      else if (el0[d] + 1 >= ne[d]) nel[d] = 1;
    }
  }
  double acc = 0.0;
  for (int c3 = 0; c3 < nel[2]; ++c3)
    for (int c2 = 0; c2 < nel[1]; ++c2)
      for (int c1 = 0; c1 < nel[0]; ++c1) {
        const int e1 = el0[0] + c1, e2 = el0[1] + c2, e3 = el0[2] + c3;
        const int a1 = i - 2 * e1, a2 = j - 2 * e2, a3 = k - 2 * e3;
        const real* Dq = quad + (e1 + (int64_t)L.nx * (e2 + (int64_t)L.ny * e3)) * 216;
        // the node's 1D values and derivatives at the three points of each axis, once
        // per element (the products below keep their order)
        double b[3][3], d[3][3];
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          b[0][t] = bq(t, a1); b[1][t] = bq(t, a2); b[2][t] = bq(t, a3);
          d[0][t] = dbq(t, a1); d[1][t] = dbq(t, a2); d[2][t] = dbq(t, a3);
        }
#pragma unroll
        for (int q = 0; q < 27; ++q) {
          const int q1 = q % 3, q2 = (q / 3) % 3, q3 = q / 9;
          const double b1 = b[0][q1], b2 = b[1][q2], b3 = b[2][q3];
          const double d1 = d[0][q1], d2 = d[1][q2], d3 = d[2][q3];
          const double s = d1 * d1 * b2 * b2 * b3 * b3 * h2[0] + b1 * b1 * d2 * d2 * b3 * b3 * h2[1] +
                           b1 * b1 * b2 * b2 * d3 * d3 * h2[2];
          acc += (double)Dq[q] * s;
        }
      }
  diag[n] = acc;
}

}  // namespace hm

// ================================================================= host launchers
using namespace hm;

namespace {
inline int grid1(int64_t n, int block) { return (int)((n + block - 1) / block); }
inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }
// blocks of the gather: one thread per x-pair of every node row
inline int gather_blocks(const Lattice& L) {
  return grid1((int64_t)L.Ny * L.Nz * (L.nx + 1), 256);
}
}

int hm_launch_pattern(const Lattice& L, int32_t* indptr, int32_t* indices, int32_t* slot, void* stream) {
  cudaStream_t s = S_(stream);
  k_pattern_indptr<<<grid1(L.ndof + 1, 256), 256, 0, s>>>(L, indptr);
  if (indices) k_pattern_indices<<<grid1(L.ndof * 32, 256), 256, 0, s>>>(L, indptr, indices);
  if (slot) k_pattern_slot<<<grid1(L.ne * 729, 256), 256, 0, s>>>(L, slot);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

int hm_launch_tpos(const Lattice& L, const int32_t* indptr, int32_t* tpos, void* stream) {
  k_pattern_tpos<<<grid1(L.ndof * 32, 256), 256, 0, S_(stream)>>>(L, indptr, tpos);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

int hm_launch_quad(const Lattice& L, const double* u, const double* m, const double* p,
                   int precision, void* quad, uint32_t* status, void* stream, const double* mhat) {
  const int blocks = grid1(L.ne, 8);
  if (precision == HM_FP32)
    k_quad<float><<<blocks, 216, 0, S_(stream)>>>(L, u, m, p, mhat, (float*)quad, status);
  else
    k_quad<double><<<blocks, 216, 0, S_(stream)>>>(L, u, m, p, mhat, (double*)quad, status);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

int hm_launch_jacobian_prepare(const Lattice& L, const void* quad, int quad_precision, void* jac,
                               int precision, void* stream) {
  const int blocks = grid1(L.ne * 27, 256);
  cudaStream_t s = S_(stream);
  if (quad_precision == HM_FP32) {
    if (precision == HM_FP32) k_extract_D<float, float><<<blocks, 256, 0, s>>>(L, (const float*)quad, (float*)jac);
    else k_extract_D<float, double><<<blocks, 256, 0, s>>>(L, (const float*)quad, (double*)jac);
  } else {
    if (precision == HM_FP32) k_extract_D<double, float><<<blocks, 256, 0, s>>>(L, (const double*)quad, (float*)jac);
    else k_extract_D<double, double><<<blocks, 256, 0, s>>>(L, (const double*)quad, (double*)jac);
  }
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

template <typename real, typename vec>
static int launch_apply_t(const Lattice& L, void* jac, const uint8_t* ess, const vec* x,
                          vec* y, const vec* dotw, double* part, void* stream,
                          double* sc = nullptr, unsigned* counter = nullptr,
                          bool x_zero_on_ess = false) {
  real* Dq = static_cast<real*>(jac);
  real* Ye = Dq + L.ne * 27;
  const int64_t warps = (L.ne + 9) / 10;
  if (x_zero_on_ess)
    k_elem_apply<real, vec, false><<<grid1(warps * 32, 256), 256, 0, S_(stream)>>>(L, Dq, ess, x, Ye);
  else
    k_elem_apply<real, vec, true><<<grid1(warps * 32, 256), 256, 0, S_(stream)>>>(L, Dq, ess, x, Ye);
  k_node_gather<real, vec><<<gather_blocks(L), 256, 0, S_(stream)>>>(
      L, Ye, ess, x, y, dotw, part, part != nullptr ? sc : nullptr, counter);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

// One Chebyshev-Jacobi smoothing step of degree 1 on the lattice operator (FP64, every
// vector zero on the Dirichlet nodes), the operator pass and the vector update fused:
//   from zero:  x = d = b idiag / theta,  r = b - A d          (pre-smoothing)
//   from x:     x += (b - A x) idiag / theta                   (post-smoothing)
// (idiag: the reciprocal of the Jacobi diagonal)
// the same arithmetic as the start / step / finish kernels of the multigrid smoother.
int hm_launch_cheb1_from_zero(const Lattice& L, void* jac, const uint8_t* ess, const double* b,
                              const double* idiag, const double* cheb, double* x, double* r,
                              void* stream) {
  double* Dq = static_cast<double*>(jac);
  double* Ye = Dq + L.ne * 27;
  const int64_t warps = (L.ne + 9) / 10;
  k_elem_apply<double, double, false, true><<<grid1(warps * 32, 256), 256, 0, S_(stream)>>>(
      L, Dq, ess, b, Ye, idiag, cheb);
  ChebOut c{b, idiag, cheb, r, x, nullptr};
  k_node_gather<double, double, 1><<<gather_blocks(L), 256, 0, S_(stream)>>>(
      L, Ye, ess, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
int hm_launch_cheb1_from_x(const Lattice& L, void* jac, const uint8_t* ess, const double* b,
                           const double* idiag, const double* cheb, double* x, void* stream) {
  double* Dq = static_cast<double*>(jac);
  double* Ye = Dq + L.ne * 27;
  const int64_t warps = (L.ne + 9) / 10;
  k_elem_apply<double, double, false><<<grid1(warps * 32, 256), 256, 0, S_(stream)>>>(L, Dq, ess, x, Ye);
  ChebOut c{b, idiag, cheb, nullptr, x, nullptr};
  k_node_gather<double, double, 2><<<gather_blocks(L), 256, 0, S_(stream)>>>(
      L, Ye, ess, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

// the same two steps with the FP32 operator and FP32 level vectors (the multigrid cycle in
// single precision): the first direction d = b idiag / theta is formed in FP64 from the
// FP64 right-hand side, once per node, and rounded to FP32 into x (k_cheb_first32); the
// element pass and the gather then read it from there; the post-smoothing result goes
// to the FP64 z
// d = b idiag / theta rounded to FP32, one thread per node (the FP64 product the FP64
// element pass forms on the fly)
__global__ void k_cheb_first32(int64_t n, const double* __restrict__ b, const double* __restrict__ idiag,
                               const double* __restrict__ cheb, float* __restrict__ d) {
  const double inv_theta = 1.0 / cheb[0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = (float)__dmul_rn(inv_theta * b[i], idiag[i]);
}
int hm_launch_cheb1_from_zero32(const Lattice& L, void* jac32, const uint8_t* ess, const double* b,
                                const double* idiag, const double* cheb, float* x, float* r,
                                void* stream) {
  float* Dq = static_cast<float*>(jac32);
  float* Ye = Dq + L.ne * 27;
  const int64_t warps = (L.ne + 9) / 10;
  k_cheb_first32<<<grid1(L.ndof, 256), 256, 0, S_(stream)>>>(L.ndof, b, idiag, cheb, x);
  k_elem_apply<float, float, false><<<grid1(warps * 32, 256), 256, 0, S_(stream)>>>(L, Dq, ess, x, Ye);
  ChebOutT<float> c{b, idiag, cheb, r, x, nullptr};
  k_node_gather<float, float, 3><<<gather_blocks(L), 256, 0, S_(stream)>>>(
      L, Ye, ess, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
int hm_launch_cheb1_from_x32(const Lattice& L, void* jac32, const uint8_t* ess, const double* b,
                             const double* idiag, const double* cheb, const float* x, double* z,
                             void* stream) {
  float* Dq = static_cast<float*>(jac32);
  float* Ye = Dq + L.ne * 27;
  const int64_t warps = (L.ne + 9) / 10;
  k_elem_apply<float, float, false><<<grid1(warps * 32, 256), 256, 0, S_(stream)>>>(L, Dq, ess, x, Ye);
  ChebOutT<float> c{b, idiag, cheb, nullptr, const_cast<float*>(x), z};
  k_node_gather<float, float, 2><<<gather_blocks(L), 256, 0, S_(stream)>>>(
      L, Ye, ess, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
int hm_launch_apply_A32(const Lattice& L, void* jac32, const uint8_t* ess, const float* x,
                        float* y, bool clean, void* stream) {
  return launch_apply_t<float, float>(L, jac32, ess, x, y, nullptr, nullptr, stream, nullptr,
                                      nullptr, clean);
}

// number of partial sums k_node_gather writes when asked for the fused dot product
int64_t hm_apply_dot_parts(const Lattice& L) { return gather_blocks(L); }

int hm_launch_apply_A(const Lattice& L, void* jac, int precision, const uint8_t* ess,
                      const double* x, double* y, void* stream) {
  if (precision == HM_FP32)
    return launch_apply_t<float, double>(L, jac, ess, x, y, nullptr, nullptr, stream);
  return launch_apply_t<double, double>(L, jac, ess, x, y, nullptr, nullptr, stream);
}

// with sc and counter the gather's last block also takes the CG step's alpha; x must be
// zero on the Dirichlet nodes (the solves keep every search direction so)
int hm_launch_apply_A_dot(const Lattice& L, void* jac, int precision, const uint8_t* ess,
                          const double* x, double* y, double* part, void* stream, double* sc,
                          unsigned* counter) {
  if (precision == HM_FP32)
    return launch_apply_t<float, double>(L, jac, ess, x, y, x, part, stream, sc, counter, true);
  return launch_apply_t<double, double>(L, jac, ess, x, y, x, part, stream, sc, counter, true);
}

// y = A x for an x that is zero on the Dirichlet nodes (FP64 operator)
int hm_launch_apply_A_clean(const Lattice& L, void* jac, const uint8_t* ess, const double* x,
                            double* y, void* stream) {
  return launch_apply_t<double, double>(L, jac, ess, x, y, nullptr, nullptr, stream, nullptr,
                                        nullptr, true);
}

// the FP32 operator on FP32 vectors (the inner solves of the mixed-precision PCG), x zero
// on the Dirichlet nodes
int hm_launch_apply_A32_dot(const Lattice& L, void* jac32, const uint8_t* ess, const float* x,
                            float* y, double* part, void* stream, double* sc, unsigned* counter) {
  return launch_apply_t<float, float>(L, jac32, ess, x, y, part ? x : nullptr, part, stream, sc,
                                      counter, true);
}

// x = b on the Dirichlet nodes (the identity rows of the eliminated operator): after it
// every residual of a solve, and so every search direction, is zero there
__global__ void k_ess_take_b(int64_t n, const uint8_t* __restrict__ ess, const double* __restrict__ b,
                             double* __restrict__ x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n && ess[i]) x[i] = b[i];
}
int hm_launch_ess_take_b(const Lattice& L, const uint8_t* ess, const double* b, double* x,
                         void* stream) {
  if (ess == nullptr) return HM_OK;
  k_ess_take_b<<<grid1(L.ndof, 256), 256, 0, S_(stream)>>>(L.ndof, ess, b, x);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

int hm_launch_diag_A(const Lattice& L, const void* quad, int precision, const uint8_t* ess,
                     double* diag, void* stream) {
  if (precision == HM_FP32)
    k_diag_A<float><<<grid1(L.ndof, 256), 256, 0, S_(stream)>>>(L, (const float*)quad, ess, diag);
  else
    k_diag_A<double><<<grid1(L.ndof, 256), 256, 0, S_(stream)>>>(L, (const double*)quad, ess, diag);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

// ================================================== allocation-free residual / gradient
// A caller that cannot allocate device memory when it needs a residual or a gradient
// (a process whose GPU memory another runtime's pool has already claimed -- JAX/XLA
// preallocates most of the device by default, hypre/MFEM may sit on an Umpire pool --
// or a loop that must not pay for an allocation) gets the assembled vectors through
// hm_lattice_residual_noalloc.  Its one scratch buffer, the pointwise data of the
// lattice's elements, is this fixed array: every GPU that loads the library holds it
// (HM_NOALLOC_MAX_ELEMENTS * 216 doubles, 14.2 MB) until the process exits.
#define HM_NOALLOC_MAX_ELEMENTS 8192
static __device__ __align__(256) double g_noalloc_quad[HM_NOALLOC_MAX_ELEMENTS * 216];

#include <mutex>

namespace {
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[64] = {nullptr};  // device address of g_noalloc_quad, per device
}  // namespace

// The device address of the scratch array on the current device, looked up once per
// device (the array's name is only a host-side stand-in for it).
static int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return HM_ERR_CUDA;
  if (dev < 0 || dev >= 64) return HM_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_addr[dev] == nullptr) {
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_quad) != cudaSuccess || ptr == nullptr) return HM_ERR_CUDA;
    g_noalloc_addr[dev] = ptr;
  }
  *out = g_noalloc_addr[dev];
  return HM_OK;
}

extern "C" int hm_lattice_residual_noalloc(const hm_lattice* h, const double* d_u, const double* d_m,
                                           const double* d_p, double f, const uint8_t* d_ess,
                                           double* d_vec_state, double* d_vec_param,
                                           double* d_vec_adjoint, int zero_ess_vectors,
                                           uint32_t* d_status, void* stream) {
  if (!h || !d_u || !d_m || !d_p || !d_status) return HM_ERR_ARG;
  if (!d_vec_state && !d_vec_param && !d_vec_adjoint) return HM_ERR_ARG;
  const hm::Lattice& L = *hm_lattice_geometry(h);
  if (L.ne > HM_NOALLOC_MAX_ELEMENTS) return HM_ERR_NOMEM;
  void* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  // k_quad overwrites the scratch for every element before the assembly reads it, so
  // nothing is carried over from the previous call
  rc = hm_launch_quad(L, d_u, d_m, d_p, HM_FP64, scratch, d_status, stream);
  if (rc) return rc;
  return hm_launch_assemble(L, scratch, HM_FP64, nullptr, d_ess, f, nullptr, nullptr, nullptr,
                            nullptr, d_vec_state, d_vec_param, d_vec_adjoint, zero_ess_vectors,
                            stream);
}

// ================================================== assembled vectors from the fields
// dR/dp (ADJOINT, with the source -f w|J| phi), dR/du (STATE) and dR/dm (PARAMETER) of the
// point (u, m, p) -- or, with mhat, the second-order products along mhat (D = w|J| e^m
// mhat, f = 0) -- without the pointwise-data intermediate: one pass evaluates the
// fields at the element's 27 points and contracts the element vectors (written in the
// SoA layout Ye[a][e] of the operator), the node gather sums them per node in the fixed
// order.  The vector counterpart of k_quad + the vector phases of the tile assembly.
namespace hm {
template <int NV>
struct VecOut { double* ye[3]; };   // element results: ADJOINT, STATE, PARAMETER (NULL: skip)

// Sum factorisation on the element's 3 x 3 x 3 nodes and points: nodes -> points one
// axis at a time (x, y, z), the pointwise data at the 27 points, then points -> nodes
// (z, y, x) for the three element vectors.  One CTA holds 8 elements, a thread per
// (element, index); every stage reads the previous one's arrays in shared memory.
//   evaluation   X: B u, B' u, B p, B' p, B m, B mhat        (index q1 + 3 a2 + 9 a3)
//                Y: u: BB, BB', B'B;  p: the same;  m, mhat: BB  (q1 + 3 q2 + 9 a3)
//                Z: grad u, grad p, m, mhat at the point      (q1 + 3 q2 + 9 q3)
//   integration  Z: E_x B, E_y B, E_z B' + s B | F_x B, F_y B, F_z B' | W B
//                Y: (.) B, (.) B' + (.) B per vector        (q1 + 3 a2 + 9 a3)
//                X: B' (.) + B (.)                          (a1 + 3 a2 + 9 a3)
// with the 1/h of each derivative folded in at its z sums.
__device__ __forceinline__ double b1d(int q, int a) { return bq(q, a); }
__device__ __forceinline__ double d1d(int q, int a) { return dbq(q, a); }

__global__ void __launch_bounds__(216, 4) k_elem_vectors(Lattice L, const double* __restrict__ u,
                                                      const double* __restrict__ m,
                                                      const double* __restrict__ p,
                                                      const double* __restrict__ mhat, double f,
                                                      VecOut<3> o, uint32_t* __restrict__ status,
                                                      const uint32_t* __restrict__ skip = nullptr) {
  if (skip != nullptr && *skip != 0u) return;    // the whole launch stands down
  // per element: arrays of 27, the element's block padded to 11 (mod 16) doubles, so
  // that the two elements a warp spans fall on different banks
  constexpr int kV = 4 * 27 + 15, kA = 7 * 27 + 14, kB = 8 * 27 + 3;
  __shared__ double sv[8][kV];           // node values u, m, p, mhat
  __shared__ double s1[8][kA];           // evaluation X / integration Z
  __shared__ double s2[8][kB];           // evaluation Y / integration Y
  __shared__ double sp[8][kB];           // E(3), F(3), W, source weight at the points
  const int tid = threadIdx.x, le = tid / 27, i = tid % 27;
  const int c1 = i % 3, c2 = (i / 3) % 3, c3 = i / 9;   // the thread's three indices
  const double ihx = 1.0 / L.hx, ihy = 1.0 / L.hy, ihz = 1.0 / L.hz;
  const double wdet = wq(c1) * wq(c2) * wq(c3) * L.hx * L.hy * L.hz;
  for (int64_t g0 = blockIdx.x * 8LL; g0 < L.ne; g0 += (int64_t)gridDim.x * 8) {
    const int64_t e = g0 + le;
    const bool live = le < 8 && e < L.ne;
    __syncthreads();                      // the previous group's arrays are consumed
    if (live) {
      const int ex = (int)(e % L.nx), ey = (int)((e / L.nx) % L.ny), ez = (int)(e / ((int64_t)L.nx * L.ny));
      const int64_t node = (2 * ex + c1) + (int64_t)L.Nx * ((2 * ey + c2) + (int64_t)L.Ny * (2 * ez + c3));
      sv[le][(0) * 27 + i] = u[node];
      sv[le][(1) * 27 + i] = m[node];
      sv[le][(2) * 27 + i] = p[node];
      sv[le][(3) * 27 + i] = mhat ? mhat[node] : 0.0;
    }
    __syncthreads();
    if (live) {   // X: index (q1 = c1, a2 = c2, a3 = c3), sums over a1
      double r[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
        const int j = a1 + 3 * c2 + 9 * c3;
        const double b = b1d(c1, a1), d = d1d(c1, a1);
        const double vu = sv[le][(0) * 27 + j], vm = sv[le][(1) * 27 + j], vp = sv[le][(2) * 27 + j], vh = sv[le][(3) * 27 + j];
        r[0] = fma(b, vu, r[0]); r[1] = fma(d, vu, r[1]);
        r[2] = fma(b, vp, r[2]); r[3] = fma(d, vp, r[3]);
        r[4] = fma(b, vm, r[4]); r[5] = fma(b, vh, r[5]);
      }
#pragma unroll
      for (int k = 0; k < 6; ++k) s1[le][(k) * 27 + i] = r[k];
    }
    __syncthreads();
    if (live) {   // Y: index (q1 = c1, q2 = c2, a3 = c3), sums over a2
      double r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int a2 = 0; a2 < 3; ++a2) {
        const int j = c1 + 3 * a2 + 9 * c3;
        const double b = b1d(c2, a2), d = d1d(c2, a2);
        const double x0 = s1[le][(0) * 27 + j], x1 = s1[le][(1) * 27 + j], x2 = s1[le][(2) * 27 + j], x3 = s1[le][(3) * 27 + j];
        r[0] = fma(b, x0, r[0]); r[1] = fma(b, x1, r[1]); r[2] = fma(d, x0, r[2]);
        r[3] = fma(b, x2, r[3]); r[4] = fma(b, x3, r[4]); r[5] = fma(d, x2, r[5]);
        r[6] = fma(b, s1[le][(4) * 27 + j], r[6]); r[7] = fma(b, s1[le][(5) * 27 + j], r[7]);
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) s2[le][(k) * 27 + i] = r[k];
    }
    __syncthreads();
    if (live) {   // Z: the point (c1, c2, c3), sums over a3; then the pointwise data
      double gu[3] = {0, 0, 0}, gp[3] = {0, 0, 0}, mv = 0.0, mh = 0.0;
#pragma unroll
      for (int a3 = 0; a3 < 3; ++a3) {
        const int j = c1 + 3 * c2 + 9 * a3;
        const double b = b1d(c3, a3), d = d1d(c3, a3);
        gu[0] = fma(b, s2[le][(1) * 27 + j], gu[0]); gu[1] = fma(b, s2[le][(2) * 27 + j], gu[1]);
        gu[2] = fma(d, s2[le][(0) * 27 + j], gu[2]);
        gp[0] = fma(b, s2[le][(4) * 27 + j], gp[0]); gp[1] = fma(b, s2[le][(5) * 27 + j], gp[1]);
        gp[2] = fma(d, s2[le][(3) * 27 + j], gp[2]);
        mv = fma(b, s2[le][(6) * 27 + j], mv); mh = fma(b, s2[le][(7) * 27 + j], mh);
      }
      gu[0] *= ihx; gu[1] *= ihy; gu[2] *= ihz;
      gp[0] *= ihx; gp[1] *= ihy; gp[2] *= ihz;
      double D = wdet * exp(mv);
      if (mhat) D *= mh;
      const double E0 = D * gu[0], E1 = D * gu[1], E2 = D * gu[2];
      const double F0 = D * gp[0], F1 = D * gp[1], F2 = D * gp[2];
      const double W = D * (gu[0] * gp[0] + gu[1] * gp[1] + gu[2] * gp[2]);
      sp[le][(0) * 27 + i] = E0; sp[le][(1) * 27 + i] = E1; sp[le][(2) * 27 + i] = E2;
      sp[le][(3) * 27 + i] = F0; sp[le][(4) * 27 + i] = F1; sp[le][(5) * 27 + i] = F2;
      sp[le][(6) * 27 + i] = W;
      sp[le][(7) * 27 + i] = mhat ? 0.0 : -f * wdet;
      if (!(isfinite(E0) && isfinite(E1) && isfinite(E2) && isfinite(F0) && isfinite(F1) &&
            isfinite(F2) && isfinite(W)))
        atomicOr(status, HM_STATUS_NONFINITE);
    }
    __syncthreads();
    if (live) {   // integration Z: index (q1 = c1, q2 = c2, a3 = c3), sums over q3
      double r[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int q3 = 0; q3 < 3; ++q3) {
        const int j = c1 + 3 * c2 + 9 * q3;
        const double b = b1d(q3, c3), d = d1d(q3, c3);
        r[0] = fma(b, sp[le][(0) * 27 + j], r[0]);
        r[1] = fma(b, sp[le][(1) * 27 + j], r[1]);
        r[2] = fma(d * ihz, sp[le][(2) * 27 + j], fma(b, sp[le][(7) * 27 + j], r[2]));
        r[3] = fma(b, sp[le][(3) * 27 + j], r[3]);
        r[4] = fma(b, sp[le][(4) * 27 + j], r[4]);
        r[5] = fma(d, sp[le][(5) * 27 + j], r[5]);
        r[6] = fma(b, sp[le][(6) * 27 + j], r[6]);
      }
      s1[le][(0) * 27 + i] = r[0] * ihx; s1[le][(1) * 27 + i] = r[1] * ihy; s1[le][(2) * 27 + i] = r[2];
      s1[le][(3) * 27 + i] = r[3] * ihx; s1[le][(4) * 27 + i] = r[4] * ihy; s1[le][(5) * 27 + i] = r[5] * ihz;
      s1[le][(6) * 27 + i] = r[6];
    }
    __syncthreads();
    if (live) {   // integration Y: index (q1 = c1, a2 = c2, a3 = c3), sums over q2
      double r[5] = {0, 0, 0, 0, 0};
#pragma unroll
      for (int q2 = 0; q2 < 3; ++q2) {
        const int j = c1 + 3 * q2 + 9 * c3;
        const double b = b1d(q2, c2), d = d1d(q2, c2);
        r[0] = fma(b, s1[le][(0) * 27 + j], r[0]);
        r[1] = fma(d, s1[le][(1) * 27 + j], fma(b, s1[le][(2) * 27 + j], r[1]));
        r[2] = fma(b, s1[le][(3) * 27 + j], r[2]);
        r[3] = fma(d, s1[le][(4) * 27 + j], fma(b, s1[le][(5) * 27 + j], r[3]));
        r[4] = fma(b, s1[le][(6) * 27 + j], r[4]);
      }
#pragma unroll
      for (int k = 0; k < 5; ++k) s2[le][(k) * 27 + i] = r[k];
    }
    __syncthreads();
    if (live) {   // integration X: the node (a1 = c1, a2 = c2, a3 = c3), sums over q1
      double ra = 0.0, rs = 0.0, rp = 0.0;
#pragma unroll
      for (int q1 = 0; q1 < 3; ++q1) {
        const int j = q1 + 3 * c2 + 9 * c3;
        const double b = b1d(q1, c1), d = d1d(q1, c1);
        ra = fma(d, s2[le][(0) * 27 + j], fma(b, s2[le][(1) * 27 + j], ra));
        rs = fma(d, s2[le][(2) * 27 + j], fma(b, s2[le][(3) * 27 + j], rs));
        rp = fma(b, s2[le][(4) * 27 + j], rp);
      }
      if (o.ye[0]) o.ye[0][(int64_t)i * L.ne + e] = ra;
      if (o.ye[1]) o.ye[1][(int64_t)i * L.ne + e] = rs;
      if (o.ye[2]) o.ye[2][(int64_t)i * L.ne + e] = rp;
    }
  }
}

__global__ void k_zero_marked(int64_t n, const uint8_t* __restrict__ ess, double* __restrict__ v) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n && ess[i]) v[i] = 0.0;
}

// *same = 0 where (u, m, p) differs from (u0, m0, p0) in any entry (compared as values:
// NaN differs from itself); *same was set nonzero before
__global__ void k_points_compare(int64_t n, const double* __restrict__ u, const double* __restrict__ u0,
                                 const double* __restrict__ m, const double* __restrict__ m0,
                                 const double* __restrict__ p, const double* __restrict__ p0,
                                 uint32_t* __restrict__ same) {
  bool diff = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    diff |= !(u[i] == u0[i]) || !(m[i] == m0[i]) || !(p[i] == p0[i]);
  if (__syncthreads_or(diff) && threadIdx.x == 0) *same = 0u;
}
// out = kept where *same (nonzero), left alone otherwise
__global__ void k_copy_if_same(int64_t n, const uint32_t* __restrict__ same,
                               const double* __restrict__ kept, double* __restrict__ out) {
  if (*same == 0u) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = kept[i];
}
}  // namespace hm

extern "C" int64_t hm_lattice_vectors_workspace_bytes(const hm_lattice* h, int nvectors) {
  if (!h || nvectors < 1 || nvectors > 3) return 0;
  return 8 * 27 * hm_lattice_geometry(h)->ne * (int64_t)nvectors;
}

extern "C" int hm_lattice_vectors(const hm_lattice* h, const double* d_u, const double* d_m,
                                  const double* d_p, const double* d_mhat, double f,
                                  const uint8_t* d_ess, double* d_vec_state, double* d_vec_param,
                                  double* d_vec_adjoint, int zero_ess_vectors, void* d_work,
                                  uint32_t* d_status, void* stream) {
  if (!h || !d_u || !d_m || !d_p || !d_work || !d_status) return HM_ERR_ARG;
  if (!d_vec_state && !d_vec_param && !d_vec_adjoint) return HM_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(d_work) & 7u) != 0) return HM_ERR_ARG;
  const Lattice& L = *hm_lattice_geometry(h);
  cudaStream_t s = S_(stream);
  double* w = static_cast<double*>(d_work);
  VecOut<3> o{};
  double* outs[3] = {d_vec_adjoint, d_vec_state, d_vec_param};
  int k = 0;
  for (int i = 0; i < 3; ++i)
    if (outs[i]) o.ye[i] = w + (int64_t)(k++) * 27 * L.ne;
  const int64_t groups = (L.ne + 7) / 8;
  const int grid = (int)(groups < 148 * 16 ? groups : 148 * 16);
  k_elem_vectors<<<grid, 216, 0, s>>>(L, d_u, d_m, d_p, d_mhat, f, o, d_status);
  for (int i = 0; i < 3; ++i) {
    if (!outs[i]) continue;
    k_node_gather<double, double, 0><<<gather_blocks(L), 256, 0, s>>>(
        L, o.ye[i], nullptr, nullptr, outs[i], nullptr, nullptr, nullptr, nullptr);
    if (zero_ess_vectors && d_ess && i != 2)
      k_zero_marked<<<grid1(L.ndof, 256), 256, 0, s>>>(L.ndof, d_ess, outs[i]);
  }
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

extern "C" int hm_lattice_vectors_at(const hm_lattice* h, const double* d_u, const double* d_m,
                                     const double* d_p, const double* d_u0, const double* d_m0,
                                     const double* d_p0, const double* d_kept_state,
                                     const double* d_kept_param, const double* d_kept_adjoint,
                                     double f, double* d_vec_state, double* d_vec_param,
                                     double* d_vec_adjoint, void* d_work, uint32_t* d_same,
                                     uint32_t* d_status, void* stream) {
  if (!h || !d_u || !d_m || !d_p || !d_u0 || !d_m0 || !d_p0 || !d_work || !d_same || !d_status)
    return HM_ERR_ARG;
  double* outs[3] = {d_vec_adjoint, d_vec_state, d_vec_param};
  const double* kept[3] = {d_kept_adjoint, d_kept_state, d_kept_param};
  if (!outs[0] && !outs[1] && !outs[2]) return HM_ERR_ARG;
  for (int i = 0; i < 3; ++i)
    if (outs[i] && !kept[i]) return HM_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(d_work) & 7u) != 0) return HM_ERR_ARG;
  const Lattice& L = *hm_lattice_geometry(h);
  cudaStream_t s = S_(stream);
  if (cudaMemsetAsync(d_same, 0xff, sizeof(uint32_t), s) != cudaSuccess) return HM_ERR_CUDA;
  const int cgrid = (int)(grid1(L.ndof, 256) < 148 * 8 ? grid1(L.ndof, 256) : 148 * 8);
  k_points_compare<<<cgrid, 256, 0, s>>>(L.ndof, d_u, d_u0, d_m, d_m0, d_p, d_p0, d_same);
  // the vectors from the fields, every launch standing down when the point is the same
  double* w = static_cast<double*>(d_work);
  VecOut<3> o{};
  int k = 0;
  for (int i = 0; i < 3; ++i)
    if (outs[i]) o.ye[i] = w + (int64_t)(k++) * 27 * L.ne;
  const int64_t groups = (L.ne + 7) / 8;
  const int grid = (int)(groups < 148 * 16 ? groups : 148 * 16);
  k_elem_vectors<<<grid, 216, 0, s>>>(L, d_u, d_m, d_p, nullptr, f, o, d_status, d_same);
  for (int i = 0; i < 3; ++i) {
    if (!outs[i]) continue;
    k_node_gather<double, double, 0><<<gather_blocks(L), 256, 0, s>>>(
        L, o.ye[i], nullptr, nullptr, outs[i], nullptr, nullptr, nullptr, nullptr, ChebOut{}, d_same);
    k_copy_if_same<<<cgrid, 256, 0, s>>>(L.ndof, d_same, kept[i], outs[i]);
  }
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

// ======================================================== boundary mass (Robin term)
// beta * int_{boundary} phi_n phi_c ds added to a block's values in the lattice pattern:
// the boundary-integrator term of the prior's operator (modeling/prior.py:941-944).  On
// the box's face x = 0 the integrand is phi_i(0) phi_ci(0) (= 1 for i = ci = 0) times the
// y and z 1D factors, so each entry gains, per face holding both nodes, the product of
// the two in-face 1D assembled mass entries.  One warp per boundary row.
namespace hm {
// 1D assembled Q2 mass entry between nodes i and c on an axis of n elements of size h
// (3-point Gauss, exact for the products): sum over the elements holding both
__device__ __forceinline__ double mass_1d(int i, int c, int n, double h) {
  const int hi = i > c ? i : c, lo = i < c ? i : c;
  if (hi - lo > 2) return 0.0;
  double s = 0.0;
  for (int e = (hi - 1) / 2 < 0 ? 0 : (hi - 1) / 2; e <= lo / 2 && e < n; ++e) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) t += wq(q) * bq(q, i - 2 * e) * bq(q, c - 2 * e);
    s += h * t;
  }
  return s;
}

__global__ void k_boundary_mass(Lattice L, double beta, double* __restrict__ vals) {
  const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= L.ndof) return;
  const int i = (int)(row % L.Nx), j = (int)((row / L.Nx) % L.Ny), k = (int)(row / ((int64_t)L.Nx * L.Ny));
  const bool on[3] = {i == 0 || i == L.Nx - 1, j == 0 || j == L.Ny - 1, k == 0 || k == L.Nz - 1};
  if (!on[0] && !on[1] && !on[2]) return;
  const int n1 = stencil_n(i, L.Nx), n2 = stencil_n(j, L.Ny), n3 = stencil_n(k, L.Nz);
  const int lo1 = stencil_lo(i), lo2 = stencil_lo(j), lo3 = stencil_lo(k);
  const int kd = ((k - lo3) * n2 + (j - lo2)) * n1 + (i - lo1);
  const int len = n1 * n2 * n3;
  const int64_t base = row_start(L, i, j, k);
  for (int pos = lane; pos < len; pos += 32) {
    const int rank = pos == 0 ? kd : (pos <= kd ? pos - 1 : pos);
    const int k1 = rank % n1, t = rank / n1, k2 = t % n2, k3 = t / n2;
    const int c[3] = {lo1 + k1, lo2 + k2, lo3 + k3};
    const int r[3] = {i, j, k};
    double add = 0.0;
    // the faces normal to axis d: the row and the column on the same face
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (!on[d] || c[d] != r[d]) continue;
      const int a = (d + 1) % 3, b = (d + 2) % 3;
      const int na[3] = {L.nx, L.ny, L.nz};
      const double ha[3] = {L.hx, L.hy, L.hz};
      add += mass_1d(r[a], c[a], na[a], ha[a]) * mass_1d(r[b], c[b], na[b], ha[b]);
    }
    if (add != 0.0) vals[base + pos] += beta * add;
  }
}
}  // namespace hm

extern "C" int hm_lattice_add_boundary_mass(const hm_lattice* h, double beta, double* d_vals,
                                            void* stream) {
  if (!h || !d_vals) return HM_ERR_ARG;
  const Lattice& L = *hm_lattice_geometry(h);
  k_boundary_mass<<<grid1(L.ndof * 32, 256), 256, 0, S_(stream)>>>(L, beta, d_vals);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
