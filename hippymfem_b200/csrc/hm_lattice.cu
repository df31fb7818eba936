// Structured-lattice kernels of the Q2 log-conductivity path (sm_100a).
//
//   k_pattern_*     the CSR graph (diagonal first), the entry->slot map and the
//                   transpose map of a Q2 x Q2 block, arithmetically
//   k_quad          pointwise data D, E = D grad u, F = D grad p, W = D grad u.grad p
//   k_tile_assemble the fused assembly: every CSR value of A, C, Wum, Wmm and the
//                   three assembled vectors, each written exactly once
//   k_tile_apply_A  the matrix-free Jacobian apply
//
// The assembly is output-stationary.  On a uniform lattice every block is a sum of
// separable terms over the global quadrature lattice, e.g.
//     A(n, j) = sum_g D(g) sum_d  T_d,x(g_x; n_x, j_x) T_d,y(...) T_d,z(...)
// with 1D pair tables T (B B, B' B', B' B) that vanish unless the row and column
// nodes share an element.  A CTA owns a 4 x 4 x 4 tile of node rows, stages the
// pointwise data of the 3 x 3 x 3 elements around it in shared memory, contracts the
// three axes one after the other (sum factorisation over the tile's 16 ordered 1D
// pairs per axis) and streams the finished rows out in CSR order.  No atomics, no
// colouring, no slot map: every value is summed in registers in a fixed order and
// stored once, so the assembly is bit-reproducible by construction.
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

__device__ __forceinline__ int64_t row_start(const Lattice& L, int i, int j, int k) {
  const int64_t T1 = stencil_prefix(L.Nx, L.Nx), T2 = stencil_prefix(L.Ny, L.Ny);
  return stencil_prefix(k, L.Nz) * T1 * T2 +
         (int64_t)stencil_n(k, L.Nz) *
             (stencil_prefix(j, L.Ny) * T1 + (int64_t)stencil_n(j, L.Ny) * stencil_prefix(i, L.Nx));
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
template <typename real>
__global__ void __launch_bounds__(216) k_quad(Lattice L, const double* __restrict__ u,
                                              const double* __restrict__ m,
                                              const double* __restrict__ p,
                                              real* __restrict__ quad,
                                              uint32_t* __restrict__ status) {
  __shared__ real sv[8][3][27];
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
  const real D = wdet * exp(val[1]);
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

// ================================================================ tile assembly
// Position of every (p1, p2, p3) output of an interior tile (no stencil clipped) in the
// tile's CSR-ordered output: runs (r2, r3) of four consecutive rows r1, each row
// diagonal first and then its columns ascending (z, then y, then x rank).
struct TileTabs {
  uint16_t inv[16][16][16];  // [p3][p2][p1] -> position in the tile output
  uint16_t runoff[17];       // start of run r2 + 4 r3
};
HM_HD constexpr TileTabs make_tile_tabs() {
  TileTabs t{};
  int off = 0;
  for (int run = 0; run < 16; ++run) {
    const int r2 = run & 3, r3 = run >> 2;
    t.runoff[run] = (uint16_t)off;
    const int n2 = row_stencil(r2), n3 = row_stencil(r3);
    const int d2 = (r2 & 1) ? 1 : 2, d3 = (r3 & 1) ? 1 : 2;
    for (int r1 = 0; r1 < 4; ++r1) {
      const int n1 = row_stencil(r1), d1 = (r1 & 1) ? 1 : 2;
      const int kd = (d3 * n2 + d2) * n1 + d1;
      for (int k3 = 0; k3 < n3; ++k3)
        for (int k2 = 0; k2 < n2; ++k2)
          for (int k1 = 0; k1 < n1; ++k1) {
            const int rank = (k3 * n2 + k2) * n1 + k1;
            const int pos = rank == kd ? 0 : (rank < kd ? rank + 1 : rank);
            t.inv[row_pair_base(r3) + k3][row_pair_base(r2) + k2][row_pair_base(r1) + k1] =
                (uint16_t)(off + pos);
          }
      off += n1 * n2 * n3;
    }
  }
  t.runoff[16] = (uint16_t)off;
  return t;
}
__device__ const TileTabs kTileTabs = make_tile_tabs();

// Strides of the stage buffers: the p3 stride is 9 (mod 16) doubles, so the 16 lanes of
// a half-warp (9 consecutive g1 of one p3 and 7 of the next, or 16 p2 of one p3) hit 16
// distinct 8-byte bank pairs.
constexpr int kT1P = 89;    // T1[p3 * kT1P + g2 * 9 + g1]
constexpr int kT2P = 153;   // T2[p3 * kT2P + p2 * 9 + g1]

// O is swizzled: position j lives at j ^ ((j >> 4) & 15), a permutation inside each
// aligned group of 16, so the contiguous copy-out stays conflict-free and the scattered
// stage-3 stores spread over the banks.
HM_HD int oswz(int j) { return j ^ ((j >> 4) & 15); }

template <typename real>
struct TileSmem {
  real W[8][9][9][9];      // pointwise data of the 27 halo'd elements on the 9^3 Gauss lattice
  real T1[16 * kT1P];      // after the z contraction
  real T2[16 * kT2P];      // after the y contraction
  real O[4096];            // the tile's rows of one block, CSR-ordered (run-major), swizzled
  int32_t rowptr[4][4][4]; // CSR offsets of the owned rows [r3][r2][r1]
  int32_t rowoff[4][4][4]; // offsets of the rows in O (tiles with clipped stencils)
  int32_t runoff[17];      // offsets of the runs in O
  uint8_t ess[7][7][7];    // Dirichlet markers of the halo'd nodes [s3][s2][s1]
  int8_t nst[3][4];        // stencil size of each owned row, per axis (0: no row)
  int8_t clip[3][4];       // columns clipped at the low end of that stencil
  int8_t dk[3][4];         // the row's own place in its (clipped) stencil
};

struct TileCtx {
  int t1, t2, t3;      // tile coordinates
  int vl[3];           // bit l set: halo'd element l is inside the mesh, per axis
  bool clipped;        // some owned row has a clipped stencil or lies outside the mesh
  bool has_ess;        // some halo'd node is a Dirichlet node
};

// The stages are instantiated once per 1D table and not inlined: the blocks share
// them, which keeps the kernel's code small enough for the instruction cache.

// stage 1: contract the z axis of one weight with table TZ -> T1
template <int TZ, typename real>
__device__ __noinline__ void stage1(const real* __restrict__ Wc, real* __restrict__ T1) {
  for (int task = threadIdx.x; task < 81; task += blockDim.x) {
    const int g1 = task % 9, g2 = task / 9;
    real w[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) w[l] = Wc[(l * 9 + g2) * 9 + g1];
#pragma unroll
    for (int p = 0; p < 16; ++p) {
      real acc = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t)
        if (t < pair_cnt(p)) acc = fma((real)pair_coef(TZ, p, t), w[pair_g0(p) + t], acc);
      T1[p * kT1P + g2 * 9 + g1] = acc;
    }
  }
}

// stage 2: contract the y axis with table TY -> T2 = scale * ... (+ T2 when acc)
template <int TY, typename real>
__device__ __noinline__ void stage2(const real* __restrict__ T1, real* __restrict__ T2, real scale,
                                    bool acc_in) {
  for (int task = threadIdx.x; task < 144; task += blockDim.x) {
    const int g1 = task % 9, p3 = task / 9;
    real w[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) w[l] = T1[p3 * kT1P + l * 9 + g1];
    real* out = T2 + p3 * kT2P + g1;
#pragma unroll
    for (int p = 0; p < 16; ++p) {
      real acc = 0;
#pragma unroll
      for (int t = 0; t < 6; ++t)
        if (t < pair_cnt(p)) acc = fma((real)pair_coef(TY, p, t), w[pair_g0(p) + t], acc);
      out[p * 9] = acc_in ? fma(scale, acc, out[p * 9]) : scale * acc;
    }
  }
}

enum BlockKind { BK_A = 0, BK_C = 1, BK_WUM = 2, BK_WMM = 3 };
// elimination applied by the last stage 3 of a block
enum Elim { EL_NONE = 0, EL_ROWCOL_DIAG = 1, EL_ROW = 2 };

// Places of outputs (p1 = 0..15, p2, p3) in O for a tile with clipped stencils; -1 if
// the column lies outside the mesh (or the row does).
template <typename real>
__device__ __noinline__ void clipped_positions(const TileSmem<real>& S, int p2, int p3, int* pos) {
  const int r2 = pair_row_of(p2), r3 = pair_row_of(p3);
  const int n2 = S.nst[1][r2], n3 = S.nst[2][r3];
  const int k2 = p2 - row_pair_base(r2) - S.clip[1][r2];
  const int k3 = p3 - row_pair_base(r3) - S.clip[2][r3];
  const bool ok23 = n2 > 0 && n3 > 0 && k2 >= 0 && k2 < n2 && k3 >= 0 && k3 < n3;
#pragma unroll 1
  for (int p1 = 0; p1 < 16; ++p1) {
    const int r1 = pair_row_of(p1);
    const int n1 = S.nst[0][r1];
    const int k1 = p1 - row_pair_base(r1) - S.clip[0][r1];
    if (!ok23 || n1 == 0 || k1 < 0 || k1 >= n1) { pos[p1] = -1; continue; }
    const int rank = (k3 * n2 + k2) * n1 + k1;
    const int kd = (S.dk[2][r3] * n2 + S.dk[1][r2]) * n1 + S.dk[0][r1];
    pos[p1] = S.rowoff[r3][r2][r1] + (rank == kd ? 0 : (rank < kd ? rank + 1 : rank));
  }
}

// stage 3: contract the x axis with table TX and scatter into the CSR-ordered tile
// output O (= or +=); with elim the block's folded elimination is applied:
// EL_ROWCOL_DIAG (A) zeroes rows and columns of Dirichlet nodes and puts 1 on their
// diagonal, EL_ROW (C, Wum) zeroes their rows.
template <int TX, typename real>
__device__ __forceinline__ void stage3_out(TileSmem<real>& S, const TileCtx& c, const real (&w)[9],
                                           int p2, int p3, int p, int at, bool acc_in, int elim,
                                           bool check) {
  real acc = 0;
#pragma unroll
  for (int t = 0; t < 6; ++t)
    if (t < pair_cnt(p)) acc = fma((real)pair_coef(TX, p, t), w[pair_g0(p) + t], acc);
  if (at < 0) return;
  at = oswz(at);
  real v = acc_in ? S.O[at] + acc : acc;
  if (check) {
    const int r2 = pair_row_of(p2), r3 = pair_row_of(p3);
    const bool ress = S.ess[r3 + 2][r2 + 2][pair_row_of(p) + 2] != 0;
    if (elim == EL_ROWCOL_DIAG) {
      const bool cess = S.ess[pair_c(p3)][pair_c(p2)][pair_c(p)] != 0;
      const bool diag = pair_s(p2) == pair_c(p2) && pair_s(p3) == pair_c(p3) && pair_s(p) == pair_c(p);
      if (ress || cess) v = (ress && diag) ? (real)1 : (real)0;
    } else if (ress) {
      v = 0;
    }
  }
  S.O[at] = v;
}

template <int TX, typename real>
__device__ __noinline__ void stage3(TileSmem<real>& S, const TileCtx& c, bool acc_in, int elim) {
  const bool check = elim != EL_NONE && c.has_ess;
  for (int task = threadIdx.x; task < 256; task += blockDim.x) {
    const int p2 = task % 16, p3 = task / 16;
    real w[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) w[l] = S.T2[p3 * kT2P + p2 * 9 + l];
    if (!c.clipped) {
      const uint4* src = reinterpret_cast<const uint4*>(&kTileTabs.inv[p3][p2][0]);
      const uint4 a = __ldg(src), b = __ldg(src + 1);
      const uint32_t wv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int p = 0; p < 16; ++p)
        stage3_out<TX>(S, c, w, p2, p3, p, (int)((wv[p >> 1] >> (16 * (p & 1))) & 0xffffu), acc_in,
                       elim, check);
    } else {
      int pos[16];
      clipped_positions(S, p2, p3, pos);
#pragma unroll
      for (int p = 0; p < 16; ++p) stage3_out<TX>(S, c, w, p2, p3, p, pos[p], acc_in, elim, check);
    }
  }
}

// The separable terms of each block; terms that share the x table form one stage-3
// group, and each group's y/z partial sums are added before the x contraction:
//   A   = K.M.M/hx^2 (D)  +  M.[K.M/hy^2 + M.K/hz^2] (D)
//   C   = R.M.M/hx (Ex)   +  M.[R.M/hy (Ey) + M.R/hz (Ez)]
//   Wum = C with F in place of E
//   Wmm = M.M.M (W)
// (tables as x.y.z; the weights carry w|J| and the physical gradients)
template <typename real>
__device__ __forceinline__ void tile_block(int blk, TileSmem<real>& S, const Lattice& L,
                                           const TileCtx& c) {
  real* T1 = S.T1;
  real* T2 = S.T2;
  if (blk == BK_A) {
    const real* D = &S.W[0][0][0][0];
    stage1<TM>(D, T1); __syncthreads();
    stage2<TM>(T1, T2, (real)(1.0 / (L.hx * L.hx)), false); __syncthreads();
    stage3<TK>(S, c, false, EL_NONE); __syncthreads();
    stage2<TK>(T1, T2, (real)(1.0 / (L.hy * L.hy)), false); __syncthreads();
    stage1<TK>(D, T1); __syncthreads();
    stage2<TM>(T1, T2, (real)(1.0 / (L.hz * L.hz)), true); __syncthreads();
    stage3<TM>(S, c, true, EL_ROWCOL_DIAG); __syncthreads();
  } else if (blk == BK_C || blk == BK_WUM) {
    const int c0 = blk == BK_C ? 1 : 4;
    const real* Gx = &S.W[c0][0][0][0];
    const real* Gy = &S.W[c0 + 1][0][0][0];
    const real* Gz = &S.W[c0 + 2][0][0][0];
    stage1<TM>(Gx, T1); __syncthreads();
    stage2<TM>(T1, T2, (real)(1.0 / L.hx), false); __syncthreads();
    stage3<TR>(S, c, false, EL_NONE); __syncthreads();
    stage1<TM>(Gy, T1); __syncthreads();
    stage2<TR>(T1, T2, (real)(1.0 / L.hy), false); __syncthreads();
    stage1<TR>(Gz, T1); __syncthreads();
    stage2<TM>(T1, T2, (real)(1.0 / L.hz), true); __syncthreads();
    stage3<TM>(S, c, true, EL_ROW); __syncthreads();
  } else {
    const real* Wq = &S.W[7][0][0][0];
    stage1<TM>(Wq, T1); __syncthreads();
    stage2<TM>(T1, T2, (real)1.0, false); __syncthreads();
    stage3<TM>(S, c, false, EL_NONE); __syncthreads();
  }
}

// Stream the tile's rows of one block out: each run of four consecutive rows is one
// contiguous stretch of the CSR values and of O; a warp copies a run, lanes on
// consecutive positions.
template <typename real>
__device__ __forceinline__ void tile_write(const TileSmem<real>& S, const TileCtx& c,
                                           double* __restrict__ vals) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarp = blockDim.x >> 5;
  for (int run = warp; run < 16; run += nwarp) {
    const int r2 = run & 3, r3 = run >> 2;
    const int a = c.clipped ? S.runoff[run] : (int)kTileTabs.runoff[run];
    const int b = c.clipped ? S.runoff[run + 1] : (int)kTileTabs.runoff[run + 1];
    if (b <= a) continue;
    double* dst = vals + (int64_t)S.rowptr[r3][r2][0];
    for (int j = lane; j < b - a; j += 32) dst[j] = (double)S.O[oswz(a + j)];
  }
}

// ------------------------------------------------------------ assembled vectors
// dR/dp = sum_g E.grad phi - f w|J| phi,  dR/du = sum_g F.grad phi,  dR/dm = sum_g W psi,
// by the same sum factorisation with single-index tables of the owned rows.
template <int TZ, typename real>
__device__ __forceinline__ void vstage1(const real* __restrict__ Wc, real* __restrict__ U1,
                                        int task, bool wdet, const Lattice& L, const TileCtx& c) {
  const int g1 = task % 9, g2 = task / 9;
  real w[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) {
    if (wdet) {
      const bool in = ((c.vl[0] >> (g1 / 3)) & 1) && ((c.vl[1] >> (g2 / 3)) & 1) && ((c.vl[2] >> (l / 3)) & 1);
      w[l] = in ? (real)(wq(g1 % 3) * wq(g2 % 3) * wq(l % 3) * L.hx * L.hy * L.hz) : (real)0;
    } else {
      w[l] = Wc[(l * 9 + g2) * 9 + g1];
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(TZ, r, t), w[vrow_g0(r) + t], acc);
    U1[(r * 9 + g2) * 9 + g1] = acc;
  }
}

template <int TY, typename real>
__device__ __forceinline__ void vstage2(const real* __restrict__ U1, real* __restrict__ U2, int task) {
  const int g1 = task % 9, r3 = task / 9;
  real w[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) w[l] = U1[(r3 * 9 + l) * 9 + g1];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(TY, r, t), w[vrow_g0(r) + t], acc);
    U2[(r3 * 4 + r) * 9 + g1] = acc;
  }
}

template <int TX, typename real>
__device__ __forceinline__ void vstage3(const real* __restrict__ U2, real (&y)[4], int r2, int r3, real scale) {
  real w[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) w[l] = U2[(r3 * 4 + r2) * 9 + l];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(TX, r, t), w[vrow_g0(r) + t], acc);
    y[r] = fma(scale, acc, y[r]);
  }
}

// the 8 vector terms: (weight, x/y/z tables); term 3 is the source (w|J|, scaled -f)
struct VTerm { int w, tx, ty, tz; };
__device__ __constant__ VTerm c_vterms[8] = {
    {1, VD, VB, VB}, {2, VB, VD, VB}, {3, VB, VB, VD}, {-1, VB, VB, VB},   // dR/dp
    {4, VD, VB, VB}, {5, VB, VD, VB}, {6, VB, VB, VD},                     // dR/du
    {7, VB, VB, VB}};                                                       // dR/dm

template <typename real>
__device__ __forceinline__ void tile_vectors(TileSmem<real>& S, const Lattice& L, const TileCtx& c,
                                             double f, double* __restrict__ vstate,
                                             double* __restrict__ vparam,
                                             double* __restrict__ vadj, bool zero_ess) {
  real* U1 = S.T1;            // 8 terms x [4][9][9]  (spans T1 and T2)
  real* U2 = &S.O[0];         // 8 terms x [4][4][9]
  const int tid = threadIdx.x;
  for (int task = tid; task < 8 * 81; task += blockDim.x) {
    const int term = task / 81, tt = task % 81;
    const VTerm vt = c_vterms[term];
    const real* Wc = vt.w >= 0 ? &S.W[vt.w][0][0][0] : nullptr;
    real* out = U1 + term * 324;
    if (vt.tz == VB) vstage1<VB>(Wc, out, tt, vt.w < 0, L, c);
    else vstage1<VD>(Wc, out, tt, vt.w < 0, L, c);
  }
  __syncthreads();
  for (int task = tid; task < 8 * 36; task += blockDim.x) {
    const int term = task / 36, tt = task % 36;
    const VTerm vt = c_vterms[term];
    if (vt.ty == VB) vstage2<VB>(U1 + term * 324, U2 + term * 144, tt);
    else vstage2<VD>(U1 + term * 324, U2 + term * 144, tt);
  }
  __syncthreads();
  // 3 slots x 16 (r2, r3): each sums its terms over r1
  if (tid < 48) {
    const int slot = tid / 16, r2 = tid % 4, r3 = (tid / 4) % 4;
    real y[4] = {0, 0, 0, 0};
    const int t0 = slot == 0 ? 0 : slot == 1 ? 4 : 7;
    const int t1 = slot == 0 ? 4 : slot == 1 ? 7 : 8;
    const real sc[3] = {(real)(1.0 / L.hx), (real)(1.0 / L.hy), (real)(1.0 / L.hz)};
    for (int term = t0; term < t1; ++term) {
      const VTerm vt = c_vterms[term];
      const real scale = term == 3 ? (real)(-f) : term == 7 ? (real)1 : sc[(term - t0) % 3];
      if (vt.tx == VB) vstage3<VB>(U2 + term * 144, y, r2, r3, scale);
      else vstage3<VD>(U2 + term * 144, y, r2, r3, scale);
    }
    double* dst = slot == 0 ? vadj : slot == 1 ? vstate : vparam;
    const int gy = 4 * c.t2 + r2, gz = 4 * c.t3 + r3;
    if (dst != nullptr && gy < L.Ny && gz < L.Nz) {
#pragma unroll
      for (int r1 = 0; r1 < 4; ++r1) {
        const int gx = 4 * c.t1 + r1;
        if (gx >= L.Nx) continue;
        double v = (double)y[r1];
        if (zero_ess && slot != 2 && S.ess[r3 + 2][r2 + 2][r1 + 2]) v = 0.0;
        dst[gx + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)] = v;
      }
    }
  }
}

template <typename real>
__device__ __forceinline__ void tile_load(TileSmem<real>& S, const Lattice& L, TileCtx& c,
                                          const real* __restrict__ quad,
                                          const uint8_t* __restrict__ ess,
                                          const int32_t* __restrict__ indptr) {
  const int tid = threadIdx.x;
  c.t1 = blockIdx.x; c.t2 = blockIdx.y; c.t3 = blockIdx.z;
  const int tt[3] = {c.t1, c.t2, c.t3};
  const int eb[3] = {2 * c.t1 - 1, 2 * c.t2 - 1, 2 * c.t3 - 1};
  const int ne[3] = {L.nx, L.ny, L.nz};
  const int Nn[3] = {L.Nx, L.Ny, L.Nz};
  bool clipped = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c.vl[d] = 0;
#pragma unroll
    for (int l = 0; l < 3; ++l)
      if (eb[d] + l >= 0 && eb[d] + l < ne[d]) c.vl[d] |= 1 << l;
    // the first tile clips row 0's stencil; the last holds the last node (clipped) and
    // may hold rows outside the mesh
    clipped |= tt[d] == 0 || 4 * tt[d] + 4 > Nn[d] - 1;
  }
  c.clipped = clipped;
  // pointwise data: thread (component, point) walks the 27 halo'd elements
  if (tid < 216) {
    const int q = tid % 27, comp = tid / 27;
    real* dst = &S.W[comp][q / 9][(q / 3) % 3][q % 3];
    const int64_t sy = L.nx, sz = (int64_t)L.nx * L.ny;
    const int64_t e0 = eb[0] + sy * eb[1] + sz * eb[2];
    real v[27];
#pragma unroll
    for (int l = 0; l < 27; ++l) {
      const int l1 = l % 3, l2 = (l / 3) % 3, l3 = l / 9;
      const bool in = ((c.vl[0] >> l1) & 1) && ((c.vl[1] >> l2) & 1) && ((c.vl[2] >> l3) & 1);
      v[l] = in ? quad[(e0 + l1 + sy * l2 + sz * l3) * 216 + tid] : (real)0;
    }
#pragma unroll
    for (int l = 0; l < 27; ++l) dst[(3 * (l / 9)) * 81 + (3 * ((l / 3) % 3)) * 9 + 3 * (l % 3)] = v[l];
  }
  int any = 0;
  for (int i = tid; i < 343; i += blockDim.x) {
    const int s1 = i % 7, s2 = (i / 7) % 7, s3 = i / 49;
    const int gx = 4 * c.t1 - 2 + s1, gy = 4 * c.t2 - 2 + s2, gz = 4 * c.t3 - 2 + s3;
    uint8_t m = 0;
    if (ess != nullptr && gx >= 0 && gx < L.Nx && gy >= 0 && gy < L.Ny && gz >= 0 && gz < L.Nz)
      m = ess[gx + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)];
    S.ess[s3][s2][s1] = m;
    any |= m;
  }
  if (indptr != nullptr && tid < 64) {
    const int r1 = tid % 4, r2 = (tid / 4) % 4, r3 = tid / 16;
    const int gx = 4 * c.t1 + r1, gy = 4 * c.t2 + r2, gz = 4 * c.t3 + r3;
    int32_t v = 0;
    if (gx < L.Nx && gy < L.Ny && gz < L.Nz) v = indptr[gx + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)];
    S.rowptr[r3][r2][r1] = v;
  }
  if (clipped && tid < 12) {
    // per axis and owned row: clipped stencil size, low-end clip, own place
    const int d = tid / 4, r = tid % 4;
    const int g = 4 * tt[d] + r;
    if (g < Nn[d]) {
      const int lo = stencil_lo(g);
      S.nst[d][r] = (int8_t)stencil_n(g, Nn[d]);
      S.clip[d][r] = (int8_t)(lo - (4 * tt[d] - 2 + row_col_start(r)));
      S.dk[d][r] = (int8_t)(g - lo);
    } else {
      S.nst[d][r] = 0; S.clip[d][r] = 0; S.dk[d][r] = 0;
    }
  }
  c.has_ess = __syncthreads_or(any) != 0;
  if (clipped && tid < 16) {
    // O layout of a clipped tile: run r2 + 4 r3, rows r1 inside, clipped lengths
    const int r2 = tid & 3, r3 = tid >> 2;
    int off = 0;
    for (int run = 0; run < tid; ++run) {
      const int a2 = run & 3, a3 = run >> 2;
      for (int r1 = 0; r1 < 4; ++r1) off += S.nst[0][r1] * S.nst[1][a2] * S.nst[2][a3];
    }
    S.runoff[tid] = off;
    for (int r1 = 0; r1 < 4; ++r1) {
      S.rowoff[r3][r2][r1] = off;
      off += S.nst[0][r1] * S.nst[1][r2] * S.nst[2][r3];
    }
    if (tid == 15) S.runoff[16] = off;
  }
  __syncthreads();
}

struct AssembleOut {
  double* vals[4];
  double* vec_state;
  double* vec_param;
  double* vec_adj;
  double f;
  int zero_ess;
};

// The fused assembly: one CTA per tile of 4 x 4 x 4 node rows, all pointwise data of
// the 27 halo'd elements resident, the blocks one after the other, each streamed out
// as soon as it is complete, then the vectors.
template <typename real>
__global__ void __launch_bounds__(256, 2)
    k_tile_assemble(Lattice L, const real* __restrict__ quad, const uint8_t* __restrict__ ess,
                    const int32_t* __restrict__ indptr, AssembleOut o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem<real>& S = *reinterpret_cast<TileSmem<real>*>(smem_raw);
  TileCtx c;
  tile_load(S, L, c, quad, ess, indptr);
#pragma unroll 1
  for (int blk = 0; blk < 4; ++blk) {
    if (o.vals[blk] == nullptr) continue;
    tile_block(blk, S, L, c);
    tile_write(S, c, o.vals[blk]);
  }
  if (o.vec_state || o.vec_param || o.vec_adj) {
    __syncthreads();
    tile_vectors(S, L, c, o.f, o.vec_state, o.vec_param, o.vec_adj, o.zero_ess != 0);
  }
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

template <typename real, typename vec>
__global__ void __launch_bounds__(256, 2)
    k_elem_apply(Lattice L, const real* __restrict__ Dq, const uint8_t* __restrict__ ess,
                 const vec* __restrict__ xin, real* __restrict__ Ye) {
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
  // z interpolation onto slice t, one node plane a3 at a time: Xb[a2][a1], Xd[a2][a1]
  real Xb[9], Xd[9];
#pragma unroll
  for (int a3 = 0; a3 < 3; ++a3) {
    const real b3 = bq_rt<real>(t, a3), d3 = dbq_rt<real>(t, a3);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const unsigned n = n0 + (unsigned)(i % 3) + nsy * (unsigned)(i / 3) + nsz * (unsigned)a3;
      const real xv = live ? (real)__ldg(xin + n) : (real)0;
      const bool fixed = ess != nullptr && live && __ldg(ess + n) != 0;
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

// One thread per node; with part != nullptr each block also
// writes its partial sum of dotw . y (the p.q of a CG step), in a fixed order.
template <typename real, typename vec>
__global__ void __launch_bounds__(256)
    k_node_gather(Lattice L, const real* __restrict__ Ye, const uint8_t* __restrict__ ess,
                  const vec* __restrict__ xin, vec* __restrict__ yout,
                  const vec* __restrict__ dotw, double* __restrict__ part) {
  const unsigned n = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = n < (unsigned)L.ndof;
  const unsigned nxy = n / (unsigned)L.Nx;
  const int ix = (int)(n - nxy * (unsigned)L.Nx);
  const int iz = (int)(nxy / (unsigned)L.Ny), iy = (int)(nxy - (unsigned)iz * (unsigned)L.Ny);
  double yv = 0.0;
  if (live) {
    if (ess != nullptr && ess[n]) {
      yv = xin[n];
    } else {
      const int gi[3] = {ix, iy, iz};
      const int nel[3] = {L.nx, L.ny, L.nz};
      // per axis: up to two (element, local index) pairs
      int e0[3], a0[3], cnt[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int i = gi[d];
        if (i & 1) { e0[d] = i >> 1; a0[d] = 1; cnt[d] = 1; }
        else if (i == 0) { e0[d] = 0; a0[d] = 0; cnt[d] = 1; }
        else if ((i >> 1) >= nel[d]) { e0[d] = (i >> 1) - 1; a0[d] = 2; cnt[d] = 1; }
        else { e0[d] = (i >> 1) - 1; a0[d] = 2; cnt[d] = 2; }   // elements i/2-1 (a=2), i/2 (a=0)
      }
      const unsigned ne = (unsigned)L.ne;
      real acc = 0;
      for (int c3 = 0; c3 < cnt[2]; ++c3)
        for (int c2 = 0; c2 < cnt[1]; ++c2)
          for (int c1 = 0; c1 < cnt[0]; ++c1) {
            const unsigned ex = e0[0] + c1, ey = e0[1] + c2, ez = e0[2] + c3;
            const unsigned a1 = c1 ? 0 : a0[0], a2 = c2 ? 0 : a0[1], a3 = c3 ? 0 : a0[2];
            const unsigned e = ex + (unsigned)L.nx * (ey + (unsigned)L.ny * ez);
            acc += Ye[(size_t)(a1 + 3 * a2 + 9 * a3) * ne + e];
          }
      yv = (double)acc;
    }
    yout[n] = (vec)yv;
  }
  if (part != nullptr) {
    __shared__ double sh[32];
    double v = live ? (double)dotw[n] * yv : 0.0;
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
        for (int q = 0; q < 27; ++q) {
          const int q1 = q % 3, q2 = (q / 3) % 3, q3 = q / 9;
          const double b1 = bq(q1, a1), b2 = bq(q2, a2), b3 = bq(q3, a3);
          const double d1 = dbq(q1, a1), d2 = dbq(q2, a2), d3 = dbq(q3, a3);
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
                   int precision, void* quad, uint32_t* status, void* stream) {
  const int blocks = grid1(L.ne, 8);
  if (precision == HM_FP32)
    k_quad<float><<<blocks, 216, 0, S_(stream)>>>(L, u, m, p, (float*)quad, status);
  else
    k_quad<double><<<blocks, 216, 0, S_(stream)>>>(L, u, m, p, (double*)quad, status);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

template <typename real>
static int launch_assemble_t(const Lattice& L, const void* quad, const int32_t* indptr,
                             const uint8_t* ess, const AssembleOut& o, void* stream) {
  const size_t smem = sizeof(TileSmem<real>);
  static bool configured[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !configured[dev]) {
    if (cudaFuncSetAttribute(k_tile_assemble<real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return HM_ERR_CUDA;
    configured[dev] = true;
  }
  dim3 grid(L.tx, L.ty, L.tz);
  k_tile_assemble<real><<<grid, 256, smem, S_(stream)>>>(L, (const real*)quad, ess, indptr, o);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

int hm_launch_assemble(const Lattice& L, const void* quad, int precision, const int32_t* indptr,
                       const uint8_t* ess, double f, double* vA, double* vC, double* vWum,
                       double* vWmm, double* vs, double* vp, double* va, int zero_ess, void* stream) {
  AssembleOut o;
  o.vals[0] = vA; o.vals[1] = vC; o.vals[2] = vWum; o.vals[3] = vWmm;
  o.vec_state = vs; o.vec_param = vp; o.vec_adj = va; o.f = f; o.zero_ess = zero_ess;
  if (precision == HM_FP32) return launch_assemble_t<float>(L, quad, indptr, ess, o, stream);
  return launch_assemble_t<double>(L, quad, indptr, ess, o, stream);
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
                          vec* y, const vec* dotw, double* part, void* stream) {
  real* Dq = static_cast<real*>(jac);
  real* Ye = Dq + L.ne * 27;
  const int64_t warps = (L.ne + 9) / 10;
  k_elem_apply<real, vec><<<grid1(warps * 32, 256), 256, 0, S_(stream)>>>(L, Dq, ess, x, Ye);
  k_node_gather<real, vec><<<grid1(L.ndof, 256), 256, 0, S_(stream)>>>(L, Ye, ess, x, y, dotw, part);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

// number of partial sums k_node_gather writes when asked for the fused dot product
int64_t hm_apply_dot_parts(const Lattice& L) { return grid1(L.ndof, 256); }

int hm_launch_apply_A(const Lattice& L, void* jac, int precision, const uint8_t* ess,
                      const double* x, double* y, void* stream) {
  if (precision == HM_FP32)
    return launch_apply_t<float, double>(L, jac, ess, x, y, nullptr, nullptr, stream);
  return launch_apply_t<double, double>(L, jac, ess, x, y, nullptr, nullptr, stream);
}

int hm_launch_apply_A_dot(const Lattice& L, void* jac, int precision, const uint8_t* ess,
                          const double* x, double* y, double* part, void* stream) {
  if (precision == HM_FP32) return launch_apply_t<float, double>(L, jac, ess, x, y, x, part, stream);
  return launch_apply_t<double, double>(L, jac, ess, x, y, x, part, stream);
}

// the FP32 operator on FP32 vectors (the inner solves of the mixed-precision PCG)
int hm_launch_apply_A32_dot(const Lattice& L, void* jac32, const uint8_t* ess, const float* x,
                            float* y, double* part, void* stream) {
  return launch_apply_t<float, float>(L, jac32, ess, x, y, part ? x : nullptr, part, stream);
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
