// The fused assembly of the Q2 log-conductivity blocks on the structured lattice
// (sm_100a): every CSR value of A, C, Wum, Wmm and the three assembled vectors, each
// written exactly once.
//
// Output-stationary.  On a uniform lattice every block is a sum of separable terms over
// the global quadrature lattice, e.g.
//     A(n, j) = sum_g D(g) sum_d  T_d,x(g_x; n_x, j_x) T_d,y(...) T_d,z(...)
// with 1D pair tables T (B B, B' B', B' B) that vanish unless the row and column nodes
// share an element.  A CTA owns a 4 x 4 x 4 tile of node rows and the 3 x 3 x 3
// elements around it.  The tile works through four phases, one per block; a phase's
// pointwise fields (D | Ex Ey Ez | Fx Fy Fz | W) arrive by one TMA copy into one of two
// shared buffers (elements outside the mesh come back as zeros), the next phase's copy
// in flight meanwhile.  Each phase contracts z, then y (the terms that share an x table
// summed here), then x, and writes its values into the tile's CSR-ordered image, which
// the warps stream out row run by row run.  No atomics, no colouring, no slot map:
// every value is summed in registers in a fixed order and stored once, so the
// assembly is bit-reproducible by construction.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "hm_common.cuh"
#include "hm_internal.h"

namespace hm {

// the library's own device status word (hm_device_status)
__device__ unsigned int g_device_status = 0;

// ------------------------------------------------------------------ tile tables
// Position of every (p1, p2, p3) output of an interior tile (no stencil clipped) in the
// tile's CSR-ordered image: runs (r2, r3) of four consecutive rows r1, each row
// diagonal first and then its columns ascending (z, then y, then x rank).
struct TileTabs {
  uint16_t inv[16][16][16];  // [p3][p2][p1] -> position in the tile image
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

// Geometry of the field buffers.  A phase's TMA box is [ez 3][ey 3][ex 3][BI] reals:
// BI consecutive reals of each element's 216 (8 fields x 27 points) from x0 on, which
// covers the phase's (up to) three fields; x0 keeps the copy 16-byte aligned and the
// fields start `off` reals into each element's row.
template <typename real> struct TileCfg;
template <> struct TileCfg<double> { static constexpr int BI = 82, AL = 2; };
template <> struct TileCfg<float> { static constexpr int BI = 84, AL = 4; };

enum Phase { PH_A = 0, PH_C = 1, PH_WUM = 2, PH_WMM = 3 };
HM_HD constexpr int phase_c0(int ph) { return ph == PH_A ? 0 : ph == PH_C ? 1 : ph == PH_WUM ? 4 : 7; }
template <typename real> HM_HD constexpr int phase_x0(int ph) {
  return (phase_c0(ph) * 27 / TileCfg<real>::AL) * TileCfg<real>::AL;
}
template <typename real> HM_HD constexpr int phase_off(int ph) {
  return phase_c0(ph) * 27 - phase_x0<real>(ph);
}

// Strides of the stage buffers: the p3 stride is 9 (mod 16) reals, so the 16 lanes of
// a half-warp (9 consecutive g1 of one p3 and 7 of the next) hit 16 distinct banks.
constexpr int kT1P = 89;    // T1[p3 * kT1P + g2 * 9 + g1]
constexpr int kT2P = 153;   // T2[p3 * kT2P + p2 * 9 + g1]
constexpr int kImage = 4096;  // reals of a tile image; position kImage is the sink

template <typename real>
struct TileSmem {
  static constexpr int kBuf = ((27 * TileCfg<real>::BI * (int)sizeof(real) + 127) / 128) * 128;
  unsigned char wbuf[2][kBuf];   // the two field buffers (TMA destinations)
  real T1[3][16 * kT1P];         // z-contracted; the tile image (kImage + 1) aliases it
  real T2[2][16 * kT2P];         // y-contracted; the vector scratch aliases it
  unsigned long long mbar[2];    // completion of the two buffers' copies
  int32_t rowptr[16];            // CSR offset of row (0, r2, r3), [r2 + 4 r3]
  int32_t runoff[17];            // image offsets of the runs (clipped tiles)
  int32_t rowoff[64];            // image offsets of the rows (clipped tiles)
  uint8_t ess[7][7][7];          // Dirichlet markers of the halo'd nodes [s3][s2][s1]
  int8_t nst[3][4];              // stencil size of each owned row, per axis (0: no row)
  int8_t clip[3][4];             // columns clipped at the low end of that stencil
  int8_t dk[3][4];               // the row's own place in its (clipped) stencil
};
static_assert(sizeof(TileSmem<double>) <= 113 * 1024, "two CTAs per SM");
static_assert(16 * kT1P * 3 >= kImage + 1, "the image fits in T1");

// ------------------------------------------------------------- TMA + mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// a bounded wait: false if the copy has not landed after ~2^20 polls
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, uint32_t parity) {
  for (int i = 0; i < (1 << 20); ++i)
    if (mbar_try_wait(b, parity)) return true;
  return false;
}
// one thread: the phase's fields of the tile's 27 elements into a buffer
template <typename real>
__device__ __forceinline__ void issue_fields(const CUtensorMap* tmap, TileSmem<real>& S, int buf,
                                             int ph, int e1, int e2, int e3) {
  constexpr uint32_t bytes = 27u * TileCfg<real>::BI * sizeof(real);
  unsigned long long* b = &S.mbar[buf];
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(S.wbuf[buf])),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(phase_x0<real>(ph)), "r"(e1), "r"(e2), "r"(e3),
      "r"(smem_u32(b))
      : "memory");
}

// ------------------------------------------------------------ 1D contractions
// sum over pair p's support of table TAB times the window w (zero coefficients skipped)
template <int TAB, int P, typename real>
__device__ __forceinline__ real pchain(const real (&w)[9]) {
  real acc = (real)pair_coef(TAB, P, 0) * w[pair_g0(P)];
#pragma unroll
  for (int t = 1; t < 6; ++t)
    if (t < pair_cnt(P) && pair_coef(TAB, P, t) != 0.0)
      acc = fma((real)pair_coef(TAB, P, t), w[pair_g0(P) + t], acc);
  return acc;
}
template <int TAB, int P, typename real>
__device__ __forceinline__ real pchain_acc(const real (&w)[9], real acc) {
#pragma unroll
  for (int t = 0; t < 6; ++t)
    if (t < pair_cnt(P) && pair_coef(TAB, P, t) != 0.0)
      acc = fma((real)pair_coef(TAB, P, t), w[pair_g0(P) + t], acc);
  return acc;
}
template <int TAB, int P>
HM_HD constexpr bool pair_first_nonzero() { return pair_coef(TAB, P, 0) != 0.0; }

// z: 9 points of a (g1, g2) column of one field -> T1[p3] (16 outputs)
template <int TZ, int BI, typename real, int P = 0>
__device__ __forceinline__ void z_outputs(const real (&w)[9], real* __restrict__ t1) {
  if constexpr (P < 16) {
    t1[P * kT1P] = pchain<TZ, P>(w);
    z_outputs<TZ, BI, real, P + 1>(w, t1);
  }
}
template <int TZ, int BI, typename real>
__device__ __forceinline__ void z_task(const real* __restrict__ col, real* __restrict__ t1) {
  real w[9];
#pragma unroll
  for (int g = 0; g < 9; ++g) w[g] = col[(g / 3) * 9 * BI + (g % 3) * 9];
  z_outputs<TZ, BI>(w, t1);
}

// y: 9 points of a (g1, p3) column of T1 -> T2[p3][p2] (16 outputs), scaled
template <int TY, typename real, int P = 0>
__device__ __forceinline__ void y_outputs(const real (&w)[9], real* __restrict__ t2, real s) {
  if constexpr (P < 16) {
    t2[P * 9] = s * pchain<TY, P>(w);
    y_outputs<TY, real, P + 1>(w, t2, s);
  }
}
template <int TY, typename real>
__device__ __forceinline__ void y_task(const real* __restrict__ col, real* __restrict__ t2, real s) {
  real w[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) w[l] = col[l * 9];
  y_outputs<TY>(w, t2, s);
}
// y of two terms summed: s1 TY1(col1) + s2 TY2(col2)
template <int TY1, int TY2, typename real, int P = 0>
__device__ __forceinline__ void y2_outputs(const real (&w1)[9], const real (&w2)[9],
                                           real* __restrict__ t2, real s1, real s2) {
  if constexpr (P < 16) {
    t2[P * 9] = fma(s2, pchain<TY2, P>(w2), s1 * pchain<TY1, P>(w1));
    y2_outputs<TY1, TY2, real, P + 1>(w1, w2, t2, s1, s2);
  }
}
template <int TY1, int TY2, typename real>
__device__ __forceinline__ void y2_task(const real* __restrict__ col1, const real* __restrict__ col2,
                                        real* __restrict__ t2, real s1, real s2) {
  real w1[9], w2[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) { w1[l] = col1[l * 9]; w2[l] = col2[l * 9]; }
  y2_outputs<TY1, TY2>(w1, w2, t2, s1, s2);
}

// x: a (p2, p3) row of T2 (one or two terms) -> 16 values of the image at the byte
// offsets pk (two 16-bit offsets per word); with ESS the elimination masks apply.
template <int TX1, int TX2, bool TWO, bool ESS, typename real, int P = 0>
__device__ __forceinline__ void x_outputs(const real (&w1)[9], const real (&w2)[9],
                                          unsigned char* __restrict__ img, const uint32_t (&pk)[8],
                                          uint32_t zmask, uint32_t omask) {
  if constexpr (P < 16) {
    real v = pchain<TX1, P>(w1);
    if constexpr (TWO) v = pchain_acc<TX2, P>(w2, v);
    if constexpr (ESS) {
      if ((zmask >> P) & 1u) v = ((omask >> P) & 1u) ? (real)1 : (real)0;
    }
    const uint32_t off = (P & 1) ? (pk[P >> 1] >> 16) : (pk[P >> 1] & 0xffffu);
    *reinterpret_cast<real*>(img + off) = v;
    x_outputs<TX1, TX2, TWO, ESS, real, P + 1>(w1, w2, img, pk, zmask, omask);
  }
}
template <int TX1, int TX2, bool TWO, typename real>
__device__ __forceinline__ void x_task(const real* __restrict__ row1, const real* __restrict__ row2,
                                       unsigned char* __restrict__ img, const uint32_t (&pk)[8],
                                       bool ess, uint32_t zmask, uint32_t omask) {
  real w1[9], w2[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) {
    w1[l] = row1[l];
    w2[l] = TWO ? row2[l] : (real)0;
  }
  if (ess) x_outputs<TX1, TX2, TWO, true>(w1, w2, img, pk, zmask, omask);
  else x_outputs<TX1, TX2, TWO, false>(w1, w2, img, pk, zmask, omask);
}

// ------------------------------------------------------------ vector stages
// dR/dp = sum_g E.grad phi - f w|J| phi,  dR/du = sum_g F.grad phi,  dR/dm = sum_g W psi,
// by the same sum factorisation with single-index tables of the owned rows.
// Terms of a phase: (field or -1 for the weights alone, x/y/z tables)
struct VTerm { int f, tx, ty, tz; };
HM_HD constexpr int phase_nterms(int ph) { return ph == PH_C ? 4 : ph == PH_WUM ? 3 : ph == PH_WMM ? 1 : 0; }
HM_HD constexpr VTerm phase_term(int ph, int j) {
  return ph == PH_WMM ? VTerm{0, VB, VB, VB}
       : j == 0 ? VTerm{0, VD, VB, VB}
       : j == 1 ? VTerm{1, VB, VD, VB}
       : j == 2 ? VTerm{2, VB, VB, VD}
                : VTerm{-1, VB, VB, VB};
}

template <int TZ, typename real>
__device__ __forceinline__ void v1_task(const real (&w)[9], real* __restrict__ u1) {
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(TZ, r, t), w[vrow_g0(r) + t], acc);
    u1[r * 81] = acc;
  }
}
template <int TY, typename real>
__device__ __forceinline__ void v2_task(const real* __restrict__ u1, real* __restrict__ u2) {
  real w[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) w[l] = u1[l * 9];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(TY, r, t), w[vrow_g0(r) + t], acc);
    u2[r * 9] = acc;
  }
}
template <int TX, typename real>
__device__ __forceinline__ void v3_task(const real* __restrict__ u2, real (&y)[4], real scale) {
  real w[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) w[l] = u2[l];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(TX, r, t), w[vrow_g0(r) + t], acc);
    y[r] = fma(scale, acc, y[r]);
  }
}

struct AssembleOut {
  double* vals[4];
  double* vec_state;
  double* vec_param;
  double* vec_adj;
  double f;
  int zero_ess;
};

// ------------------------------------------------------------ the kernel
template <typename real>
__global__ void __launch_bounds__(256, 2)
    k_tile_assemble(const __grid_constant__ CUtensorMap tmap, Lattice L,
                    const uint8_t* __restrict__ ess, const int32_t* __restrict__ indptr,
                    AssembleOut o) {
  constexpr int BI = TileCfg<real>::BI;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  TileSmem<real>& S = *reinterpret_cast<TileSmem<real>*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t1 = blockIdx.x, t2 = blockIdx.y, t3 = blockIdx.z;
  const int e1 = 2 * t1 - 1, e2 = 2 * t2 - 1, e3 = 2 * t3 - 1;   // first halo'd element

  // the phases with work: a block, or a vector that its fields carry
  const uint32_t pm = (o.vals[0] != nullptr ? 1u : 0u) |
                      ((o.vals[1] != nullptr || o.vec_adj != nullptr) ? 2u : 0u) |
                      ((o.vals[2] != nullptr || o.vec_state != nullptr) ? 4u : 0u) |
                      ((o.vals[3] != nullptr || o.vec_param != nullptr) ? 8u : 0u);
  auto next_phase = [&](int b) -> int {
    const uint32_t rest = pm & ~((2u << b) - 1u);
    return rest ? __ffs(rest) - 1 : -1;
  };
  if (tid == 0) {
    mbar_init(&S.mbar[0], 1);
    mbar_init(&S.mbar[1], 1);
    fence_mbar_init();
    fence_proxy_async();
    const int f0 = pm ? __ffs(pm) - 1 : -1;
    const int f1 = f0 >= 0 ? next_phase(f0) : -1;
    if (f0 >= 0) issue_fields(&tmap, S, 0, f0, e1, e2, e3);
    if (f1 >= 0) issue_fields(&tmap, S, 1, f1, e1, e2, e3);
  }

  // ---- tile setup: Dirichlet markers of the halo, row pointers, clipped stencils
  const int Nn[3] = {L.Nx, L.Ny, L.Nz};
  const int tt[3] = {t1, t2, t3};
  bool clipped = false;
  int vl[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int ne = d == 0 ? L.nx : d == 1 ? L.ny : L.nz;
    vl[d] = 0;
#pragma unroll
    for (int l = 0; l < 3; ++l)
      if (2 * tt[d] - 1 + l >= 0 && 2 * tt[d] - 1 + l < ne) vl[d] |= 1 << l;
    // the first tile clips row 0's stencil; the last holds the last node (clipped)
    // and may hold rows outside the mesh
    clipped |= tt[d] == 0 || 4 * tt[d] + 4 > Nn[d] - 1;
  }
  int any = 0;
  for (int i = tid; i < 343; i += 256) {
    const int s1 = i % 7, s2 = (i / 7) % 7, s3 = i / 49;
    const int gx = 4 * t1 - 2 + s1, gy = 4 * t2 - 2 + s2, gz = 4 * t3 - 2 + s3;
    uint8_t m = 0;
    if (ess != nullptr && gx >= 0 && gx < L.Nx && gy >= 0 && gy < L.Ny && gz >= 0 && gz < L.Nz)
      m = ess[gx + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)];
    S.ess[s3][s2][s1] = m;
    any |= m;
  }
  if (indptr != nullptr && tid < 16) {
    const int r2 = tid & 3, r3 = tid >> 2;
    const int gy = 4 * t2 + r2, gz = 4 * t3 + r3;
    S.rowptr[tid] = (gy < L.Ny && gz < L.Nz) ? indptr[4 * t1 + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)] : 0;
  }
  if (clipped && tid < 12) {
    const int d = tid / 4, r = tid % 4;
    const int td = d == 0 ? t1 : d == 1 ? t2 : t3;
    const int Nd = d == 0 ? L.Nx : d == 1 ? L.Ny : L.Nz;
    const int g = 4 * td + r;
    if (g < Nd) {
      const int lo = stencil_lo(g);
      S.nst[d][r] = (int8_t)stencil_n(g, Nd);
      S.clip[d][r] = (int8_t)(lo - (4 * td - 2 + row_col_start(r)));
      S.dk[d][r] = (int8_t)(g - lo);
    } else {
      S.nst[d][r] = 0; S.clip[d][r] = 0; S.dk[d][r] = 0;
    }
  }
  const bool has_ess = __syncthreads_or(any) != 0;
  if (clipped && tid < 16) {
    // image layout of a clipped tile: run r2 + 4 r3, its rows r1, clipped lengths
    const int r2 = tid & 3, r3 = tid >> 2;
    int off = 0;
    for (int run = 0; run < tid; ++run)
      for (int r1 = 0; r1 < 4; ++r1) off += S.nst[0][r1] * S.nst[1][run & 3] * S.nst[2][run >> 2];
    S.runoff[tid] = off;
    for (int r1 = 0; r1 < 4; ++r1) {
      S.rowoff[tid * 4 + r1] = off;
      off += S.nst[0][r1] * S.nst[1][r2] * S.nst[2][r3];
    }
    if (tid == 15) S.runoff[16] = off;
  }
  __syncthreads();

  // ---- this thread's x task (p2, p3): image byte offsets and elimination masks
  const int xp2 = tid & 15, xp3 = tid >> 4;
  uint32_t pk[8];
  {
    if (!clipped) {
      const uint4* src = reinterpret_cast<const uint4*>(&kTileTabs.inv[xp3][xp2][0]);
      const uint4 a = __ldg(src), b = __ldg(src + 1);
      const uint32_t v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
      for (int i = 0; i < 8; ++i) pk[i] = v[i] * (uint32_t)sizeof(real);   // both halves < 2^13
    } else {
      const int r2 = pair_row_of(xp2), r3 = pair_row_of(xp3);
      const int n2 = S.nst[1][r2], n3 = S.nst[2][r3];
      const int k2 = xp2 - row_pair_base(r2) - S.clip[1][r2];
      const int k3 = xp3 - row_pair_base(r3) - S.clip[2][r3];
      const bool ok23 = n2 > 0 && n3 > 0 && k2 >= 0 && k2 < n2 && k3 >= 0 && k3 < n3;
#pragma unroll
      for (int i = 0; i < 8; ++i) pk[i] = 0;
#pragma unroll
      for (int p1 = 0; p1 < 16; ++p1) {
        const int r1 = pair_row_of(p1);
        const int n1 = S.nst[0][r1];
        const int k1 = p1 - row_pair_base(r1) - S.clip[0][r1];
        int pos = kImage;
        if (ok23 && n1 > 0 && k1 >= 0 && k1 < n1) {
          const int rank = (k3 * n2 + k2) * n1 + k1;
          const int kd = (S.dk[2][r3] * n2 + S.dk[1][r2]) * n1 + S.dk[0][r1];
          pos = S.rowoff[(r2 + 4 * r3) * 4 + r1] + (rank == kd ? 0 : (rank < kd ? rank + 1 : rank));
        }
        pk[p1 >> 1] |= (uint32_t)(pos * (int)sizeof(real)) << (16 * (p1 & 1));
      }
    }
  }
  uint32_t zA = 0, oA = 0, zC = 0;
  if (has_ess) {
    const int r2 = pair_row_of(xp2), r3 = pair_row_of(xp3);
    const int c2 = pair_c(xp2), c3 = pair_c(xp3);
    const bool diag23 = c2 == r2 + 2 && c3 == r3 + 2;
    uint32_t rb = 0, cb = 0;
#pragma unroll
    for (int r1 = 0; r1 < 4; ++r1) rb |= (uint32_t)(S.ess[r3 + 2][r2 + 2][r1 + 2] != 0) << r1;
#pragma unroll
    for (int c1 = 0; c1 < 7; ++c1) cb |= (uint32_t)(S.ess[c3][c2][c1] != 0) << c1;
#pragma unroll
    for (int p = 0; p < 16; ++p) {
      const bool re = (rb >> pair_row_of(p)) & 1u, ce = (cb >> pair_c(p)) & 1u;
      if (re || ce) zA |= 1u << p;
      if (re && diag23 && pair_c(p) == pair_s(p)) oA |= 1u << p;
      if (re) zC |= 1u << p;
    }
  }

  // ---- per-thread addresses of the z and y tasks
  const int zi = tid % 81;                     // (g1, g2) of the z task
  const int zg1 = zi % 9, zg2 = zi / 9;
  const int zbase = ((zg2 / 3) * 3 + zg1 / 3) * BI + zg1 % 3 + 3 * (zg2 % 3);
  const int zt1 = zg2 * 9 + zg1;

  unsigned char* const img = reinterpret_cast<unsigned char*>(&S.T1[0][0]);
  real* const U1 = &S.T2[0][0];               // vector scratch: [term][r3][g2][g1]
  real* const U2 = U1 + 4 * 324;              // [term][r3][r2][g1]
  const real ihx = (real)(1.0 / L.hx), ihy = (real)(1.0 / L.hy), ihz = (real)(1.0 / L.hz);

  int k = 0;
#pragma unroll 1
  for (int ph = 0; ph < 4; ++ph) {
    if (!((pm >> ph) & 1u)) continue;
    const int buf = k & 1;
    const bool ok = mbar_wait(&S.mbar[buf], (uint32_t)(k >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(&g_device_status, HM_STATUS_TIMEOUT);
        // the other buffer's copy, if one is in flight, before the CTA leaves
        const int nx = next_phase(ph);
        if (nx >= 0) (void)mbar_wait(&S.mbar[buf ^ 1], (uint32_t)((k + 1) >> 1) & 1u);
      }
      return;
    }
    const real* W = reinterpret_cast<const real*>(S.wbuf[buf]) + phase_off<real>(ph);
    double* const vals = ph == 0 ? o.vals[0] : ph == 1 ? o.vals[1] : ph == 2 ? o.vals[2] : o.vals[3];
    double* const vec = ph == 0 ? nullptr : ph == 1 ? o.vec_adj : ph == 2 ? o.vec_state : o.vec_param;
    const int after = next_phase(ph);
    const int after2 = after >= 0 ? next_phase(after) : -1;

    if (vals != nullptr) {
      // z: T1[0..2] from the phase's fields
      if (ph == PH_A) {
        if (tid < 81) z_task<TM, BI>(W + zbase, &S.T1[0][zt1]);
        else if (tid < 162) z_task<TK, BI>(W + zbase, &S.T1[1][zt1]);
      } else if (ph == PH_WMM) {
        if (tid < 81) z_task<TM, BI>(W + zbase, &S.T1[0][zt1]);
      } else {
        if (tid < 81) z_task<TM, BI>(W + zbase, &S.T1[0][zt1]);
        else if (tid < 162) z_task<TM, BI>(W + 27 + zbase, &S.T1[1][zt1]);
        else if (tid < 243) z_task<TR, BI>(W + 54 + zbase, &S.T1[2][zt1]);
      }
      __syncthreads();
      if (vec == nullptr && tid == 0 && after2 >= 0) {
        fence_proxy_async();
        issue_fields(&tmap, S, buf, after2, e1, e2, e3);
      }
      // y: T2[0] (the x-table-1 term), T2[1] (the two terms of x table 2)
      {
        const int i = tid < 144 ? tid : tid - 144;
        const int g1 = i % 9, p3 = i / 9;
        const int c1 = p3 * kT1P + g1, c2 = p3 * kT2P + g1;
        if (ph == PH_A) {
          if (tid < 144) y2_task<TK, TM>(&S.T1[0][c1], &S.T1[1][c1], &S.T2[1][c2], ihy * ihy, ihz * ihz);
          else y_task<TM>(&S.T1[0][c1], &S.T2[0][c2], ihx * ihx);
        } else if (ph == PH_WMM) {
          if (tid < 144) y_task<TM>(&S.T1[0][c1], &S.T2[0][c2], (real)1);
        } else {
          if (tid < 144) y2_task<TR, TM>(&S.T1[1][c1], &S.T1[2][c1], &S.T2[1][c2], ihy, ihz);
          else y_task<TM>(&S.T1[0][c1], &S.T2[0][c2], ihx);
        }
        if (ph != PH_WMM && tid >= 144 && tid < 176) {
          const int j = tid - 144 + 112;
          const int h1 = j % 9, q3 = j / 9;
          y_task<TM>(&S.T1[0][q3 * kT1P + h1], &S.T2[0][q3 * kT2P + h1], ph == PH_A ? ihx * ihx : ihx);
        }
      }
      __syncthreads();
      // x: the tile image
      {
        const int r = xp3 * kT2P + xp2 * 9;
        if (ph == PH_A) x_task<TK, TM, true>(&S.T2[0][r], &S.T2[1][r], img, pk, has_ess, zA, oA);
        else if (ph == PH_WMM) x_task<TM, TM, false>(&S.T2[0][r], (const real*)nullptr, img, pk, false, 0u, 0u);
        else x_task<TR, TM, true>(&S.T2[0][r], &S.T2[1][r], img, pk, has_ess, zC, 0u);
      }
      __syncthreads();
      // stream the image out: a warp per run of four consecutive rows
      const real* O = reinterpret_cast<const real*>(img);
#pragma unroll 1
      for (int run = warp; run < 16; run += 8) {
        const int a = clipped ? S.runoff[run] : (int)kTileTabs.runoff[run];
        const int b = clipped ? S.runoff[run + 1] : (int)kTileTabs.runoff[run + 1];
        double* dst = vals + (int64_t)S.rowptr[run];
        for (int j = lane; j < b - a; j += 32) dst[j] = (double)O[a + j];
      }
    }
    if (vec != nullptr) {
      // vector z stage (fields still resident)
      const int nt = phase_nterms(ph);
      for (int task = tid; task < nt * 81; task += 256) {
        const int j = task / 81, i = task % 81;
        const VTerm vt = phase_term(ph, j);
        const int g1 = i % 9, g2 = i / 9;
        real w[9];
        if (vt.f >= 0) {
          const real* col = W + 27 * vt.f + ((g2 / 3) * 3 + g1 / 3) * BI + g1 % 3 + 3 * (g2 % 3);
#pragma unroll
          for (int g = 0; g < 9; ++g) w[g] = col[(g / 3) * 9 * BI + (g % 3) * 9];
        } else {
          const bool in12 = ((vl[0] >> (g1 / 3)) & 1) && ((vl[1] >> (g2 / 3)) & 1);
#pragma unroll
          for (int g = 0; g < 9; ++g)
            w[g] = (in12 && ((vl[2] >> (g / 3)) & 1))
                       ? (real)(wq(g1 % 3) * wq(g2 % 3) * wq(g % 3) * L.hx * L.hy * L.hz)
                       : (real)0;
        }
        real* u1 = U1 + j * 324 + g2 * 9 + g1;
        if (vt.tz == VD) v1_task<VD>(w, u1);
        else v1_task<VB>(w, u1);
      }
      __syncthreads();
      if (tid == 0 && after2 >= 0) {
        fence_proxy_async();
        issue_fields(&tmap, S, buf, after2, e1, e2, e3);
      }
      for (int task = tid; task < nt * 36; task += 256) {
        const int j = task / 36, i = task % 36;
        const int g1 = i % 9, r3 = i / 9;
        const VTerm vt = phase_term(ph, j);
        const real* u1 = U1 + j * 324 + r3 * 81 + g1;
        real* u2 = U2 + j * 144 + r3 * 36 + g1;
        if (vt.ty == VD) v2_task<VD>(u1, u2);
        else v2_task<VB>(u1, u2);
      }
      __syncthreads();
      if (tid < 16) {
        const int r2 = tid & 3, r3 = tid >> 2;
        real y[4] = {0, 0, 0, 0};
        for (int j = 0; j < nt; ++j) {
          const VTerm vt = phase_term(ph, j);
          const real scale = vt.f < 0 ? (real)(-o.f)
                           : ph == PH_WMM ? (real)1 : (j == 0 ? ihx : j == 1 ? ihy : ihz);
          const real* u2 = U2 + j * 144 + r3 * 36 + r2 * 9;
          if (vt.tx == VD) v3_task<VD>(u2, y, scale);
          else v3_task<VB>(u2, y, scale);
        }
        const int gy = 4 * t2 + r2, gz = 4 * t3 + r3;
        if (gy < L.Ny && gz < L.Nz) {
#pragma unroll
          for (int r1 = 0; r1 < 4; ++r1) {
            const int gx = 4 * t1 + r1;
            if (gx >= L.Nx) continue;
            double v = (double)y[r1];
            if (o.zero_ess && ph != PH_WMM && S.ess[r3 + 2][r2 + 2][r1 + 2]) v = 0.0;
            vec[gx + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)] = v;
          }
        }
      }
    }
    // the image (T1) and the y buffers are rewritten by the next phase
    __syncthreads();
    ++k;
  }
}

// ------------------------------------------------------------ host side
namespace {
inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// the quadrature array as a 4D tensor (216 reals per element, ex, ey, ez)
template <typename real>
int make_quad_map(const Lattice& L, const void* quad, CUtensorMap* m) {
  auto fn = encode_fn();
  if (fn == nullptr) return HM_ERR_CUDA;
  if ((reinterpret_cast<uintptr_t>(quad) & 15u) != 0) return HM_ERR_ARG;
  const cuuint64_t es = sizeof(real);
  cuuint64_t dims[4] = {216, (cuuint64_t)L.nx, (cuuint64_t)L.ny, (cuuint64_t)L.nz};
  cuuint64_t strides[3] = {216 * es, 216 * es * (cuuint64_t)L.nx,
                           216 * es * (cuuint64_t)L.nx * (cuuint64_t)L.ny};
  cuuint32_t box[4] = {(cuuint32_t)TileCfg<real>::BI, 3, 3, 3};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                        4, const_cast<void*>(quad), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HM_OK : HM_ERR_CUDA;
}

template <typename real>
int launch_assemble_t(const Lattice& L, const void* quad, const int32_t* indptr,
                      const uint8_t* ess, const AssembleOut& o, void* stream) {
  const size_t smem = sizeof(TileSmem<real>);
  static std::mutex mu;
  static bool configured[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return HM_ERR_CUDA;
  {
    std::lock_guard<std::mutex> g(mu);
    if (dev < 64 && !configured[dev]) {
      if (cudaFuncSetAttribute(k_tile_assemble<real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem) != cudaSuccess)
        return HM_ERR_CUDA;
      configured[dev] = true;
    }
  }
  CUtensorMap m;
  const int rc = make_quad_map<real>(L, quad, &m);
  if (rc) return rc;
  dim3 grid(L.tx, L.ty, L.tz);
  k_tile_assemble<real><<<grid, 256, smem, S_(stream)>>>(m, L, ess, indptr, o);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
}  // namespace

}  // namespace hm

using namespace hm;

int hm_launch_assemble(const Lattice& L, const void* quad, int precision, const int32_t* indptr,
                       const uint8_t* ess, double f, double* vA, double* vC, double* vWum,
                       double* vWmm, double* vs, double* vp, double* va, int zero_ess, void* stream) {
  AssembleOut o;
  o.vals[0] = vA; o.vals[1] = vC; o.vals[2] = vWum; o.vals[3] = vWmm;
  o.vec_state = vs; o.vec_param = vp; o.vec_adj = va; o.f = f; o.zero_ess = zero_ess;
  if ((vA || vC || vWum || vWmm) && indptr == nullptr) return HM_ERR_ARG;
  if (precision == HM_FP32) return launch_assemble_t<float>(L, quad, indptr, ess, o, stream);
  return launch_assemble_t<double>(L, quad, indptr, ess, o, stream);
}

extern "C" int hm_device_status(uint32_t* out, int clear) {
  if (!out) return HM_ERR_ARG;
  unsigned int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_device_status, sizeof(v)) != cudaSuccess) return HM_ERR_CUDA;
  *out = v;
  if (clear) {
    const unsigned int z = 0;
    if (cudaMemcpyToSymbol(g_device_status, &z, sizeof(z)) != cudaSuccess) return HM_ERR_CUDA;
  }
  return HM_OK;
}
