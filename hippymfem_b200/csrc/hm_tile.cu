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
// diagonal first and then its columns ascending (z, then y, then x rank).  Runs start
// after an even pad (chosen to spread the image stores over the shared-memory banks;
// at least 2 after the first run), and a tile may shift a run by one more slot so that
// it has the parity of its CSR offset (the bulk copy-out wants 16-byte alignment on
// both sides) without reaching the next run.
constexpr int kRunPad[16] = {10, 10, 14, 10, 10, 2, 8, 2, 2, 10, 14, 10, 4, 6, 2, 12};
struct alignas(16) TileTabs {
  uint16_t inv[16][16][16];  // [p3][p2][p1] -> position in the tile image
  uint16_t runoff[16];       // start of run r2 + 4 r3 (before the tile's parity shift)
  uint16_t runlen[16];       // its length
};
HM_HD constexpr TileTabs make_tile_tabs() {
  TileTabs t{};
  int off = 0;
  for (int run = 0; run < 16; ++run) {
    const int r2 = run & 3, r3 = run >> 2;
    off += kRunPad[run];
    t.runoff[run] = (uint16_t)off;
    const int start = off;
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
    t.runlen[run] = (uint16_t)(off - start);
  }
  return t;
}
__device__ const TileTabs kTileTabs = make_tile_tabs();
// the run starts and lengths (as kTileTabs.runoff / runlen) folded into immediates, so
// that the tile set-up reads them without a load
struct RunTabs { int off[16]; int len[16]; };
HM_HD constexpr RunTabs make_run_tabs() {
  RunTabs t{};
  int off = 0;
  for (int run = 0; run < 16; ++run) {
    const int n2 = row_stencil(run & 3), n3 = row_stencil(run >> 2);
    off += kRunPad[run];
    t.off[run] = off;
    int len = 0;
    for (int r1 = 0; r1 < 4; ++r1) len += row_stencil(r1) * n2 * n3;
    t.len[run] = len;
    off += len;
  }
  return t;
}
HM_HD constexpr bool run_tabs_agree() {
  for (int i = 0; i < 16; ++i)
    if (make_run_tabs().off[i] != make_tile_tabs().runoff[i] ||
        make_run_tabs().len[i] != make_tile_tabs().runlen[i])
      return false;
  return true;
}
static_assert(run_tabs_agree(), "run tables");
template <int Q = 0>
__device__ __forceinline__ int run_sel(int run, bool len) {
  if constexpr (Q < 16) {
    constexpr int o = make_run_tabs().off[Q], n = make_run_tabs().len[Q];
    return run == Q ? (len ? n : o) : run_sel<Q + 1>(run, len);
  } else {
    return 0;
  }
}
HM_HD constexpr int run_pad_total() {
  int s = 0;
  for (int i = 0; i < 16; ++i) s += kRunPad[i];
  return s;
}
HM_HD constexpr bool run_pads_ok() {
  for (int i = 1; i < 16; ++i)
    if (kRunPad[i] < 2 || (kRunPad[i] & 1)) return false;
  return (kRunPad[0] & 1) == 0;
}
static_assert(run_pads_ok(), "even pads, at least 2 between runs");

// Geometry of the field buffers.  A phase's TMA box is [ez 3][ey 3][ex 3][BI] reals:
// BI consecutive reals of each element's 216 (8 fields x 27 points) from x0 on, which
// covers the phase's (up to) three fields; x0 keeps the copy 16-byte aligned and the
// fields start `off` reals into each element's row.
template <typename real> struct TileCfg;
template <> struct TileCfg<double> { static constexpr int BI = 86, AL = 2; };
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
constexpr int kSink = 16 * kT1P * 3 - 1;   // the image's sink slot (outputs outside the mesh)
static_assert(4096 + run_pad_total() + 16 <= kSink, "the padded image fits in T1");

template <typename real>
struct TileSmem {
  static constexpr int kBuf = ((27 * TileCfg<real>::BI * (int)sizeof(real) + 127) / 128) * 128;
  unsigned char wbuf[2][kBuf];   // the two field buffers (TMA destinations)
  real T1[3][16 * kT1P];         // z-contracted; the tile image (to kSink) aliases it
  real T2[2][16 * kT2P];         // y-contracted; the vector scratch aliases it
  unsigned long long mbar[2];    // completion of the two buffers' copies
  int32_t rowptr[16];            // CSR offset of row (0, r2, r3), [r2 + 4 r3]
  int32_t runstart[16];          // image offset of each run
  int32_t runlen[16];            // and its length
  int32_t rowoff[64];            // image offsets of the rows (clipped tiles)
  uint8_t ess[7][7][7];          // Dirichlet markers of the halo'd nodes [s3][s2][s1]
  int8_t nst[3][4];              // stencil size of each owned row, per axis (0: no row)
  int8_t clip[3][4];             // columns clipped at the low end of that stencil
  int8_t dk[3][4];               // the row's own place in its (clipped) stencil
};
static_assert(sizeof(TileSmem<double>) <= 113 * 1024, "two CTAs per SM");

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

// bulk copy of a stretch of the image to global memory (both ends 16-byte aligned,
// size a multiple of 16), and the waits on this thread's copies
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
               "r"(smem_u32(ssrc)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

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
// offsets pk (two 16-bit offsets per word); with ESS the elimination masks apply.  With
// ROWS the values before elimination are also summed per row r1 into rs (the block's
// row sums: its assembled vector, by the partition of unity of the parameter basis).
template <int TX1, int TX2, bool TWO, bool ESS, bool ROWS, typename real, int P = 0>
__device__ __forceinline__ void x_outputs(const real (&w1)[9], const real (&w2)[9],
                                          unsigned char* __restrict__ img, const uint32_t (&pk)[8],
                                          uint32_t zmask, uint32_t omask, real (&rs)[4]) {
  if constexpr (P < 16) {
    real v = pchain<TX1, P>(w1);
    if constexpr (TWO) v = pchain_acc<TX2, P>(w2, v);
    if constexpr (ROWS) {
      if constexpr (P == row_pair_base(pair_row_of(P))) rs[pair_row_of(P)] = v;
      else rs[pair_row_of(P)] += v;
    }
    if constexpr (ESS) {
      if ((zmask >> P) & 1u) v = ((omask >> P) & 1u) ? (real)1 : (real)0;
    }
    const uint32_t off = (P & 1) ? (pk[P >> 1] >> 16) : (pk[P >> 1] & 0xffffu);
    *reinterpret_cast<real*>(img + off) = v;
    x_outputs<TX1, TX2, TWO, ESS, ROWS, real, P + 1>(w1, w2, img, pk, zmask, omask, rs);
  }
}
template <int TX1, int TX2, bool TWO, bool ROWS, typename real>
__device__ __forceinline__ void x_task(const real* __restrict__ row1, const real* __restrict__ row2,
                                       unsigned char* __restrict__ img, const uint32_t (&pk)[8],
                                       bool ess, uint32_t zmask, uint32_t omask, real (&rs)[4]) {
  real w1[9], w2[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) {
    w1[l] = row1[l];
    w2[l] = TWO ? row2[l] : (real)0;
  }
  if (ess) x_outputs<TX1, TX2, TWO, true, ROWS>(w1, w2, img, pk, zmask, omask, rs);
  else x_outputs<TX1, TX2, TWO, false, ROWS>(w1, w2, img, pk, zmask, omask, rs);
}

// ------------------------------------------------------------ vector stages
// dR/dp = sum_g E.grad phi - f w|J| phi,  dR/du = sum_g F.grad phi,  dR/dm = sum_g W psi,
// by the same sum factorisation with single-index tables of the owned rows.  The terms
// of a phase: field j with table VD on axis j (the gradient terms of C and Wum phases),
// or VB everywhere (Wmm).  The source term -f w|J| phi separates into three 1D sums.
template <int PH> HM_HD constexpr int vec_nterms() { return PH == PH_WMM ? 1 : 3; }
template <int PH, int J, int AXIS> HM_HD constexpr int vec_tab() {
  return PH == PH_WMM ? VB : (J == AXIS ? VD : VB);
}

// z: the (g1, g2) column of field J -> U1[J][r3][g2][g1]
template <int PH, int J, int BI, typename real>
__device__ __forceinline__ void vz_task(const real* __restrict__ col, real* __restrict__ u1) {
  real w[9];
#pragma unroll
  for (int g = 0; g < 9; ++g) w[g] = col[(g / 3) * 9 * BI + (g % 3) * 9];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(vec_tab<PH, J, 2>(), r, t), w[vrow_g0(r) + t], acc);
    u1[r * 81] = acc;
  }
}
template <int PH, int BI, typename real>
__device__ __forceinline__ void vec_z(const real* __restrict__ W, real* __restrict__ U1, int tid) {
  if (tid >= 81 * vec_nterms<PH>()) return;
  const int j = tid / 81, i = tid % 81;
  const int g1 = i % 9, g2 = i / 9;
  const real* col = W + 27 * j + ((g2 / 3) * 3 + g1 / 3) * BI + g1 % 3 + 3 * (g2 % 3);
  real* u1 = U1 + j * 324 + g2 * 9 + g1;
  if (j == 0) vz_task<PH, 0, BI>(col, u1);
  else if (j == 1) vz_task<PH, 1, BI>(col, u1);
  else vz_task<PH, 2, BI>(col, u1);
}
// y: (g1, r3) of term J -> U2[J][r3][r2][g1]
template <int PH, int J, typename real>
__device__ __forceinline__ void vy_task(const real* __restrict__ u1, real* __restrict__ u2) {
  real w[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) w[l] = u1[l * 9];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    real acc = 0;
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t < vrow_cnt(r)) acc = fma((real)vrow_coef(vec_tab<PH, J, 1>(), r, t), w[vrow_g0(r) + t], acc);
    u2[r * 9] = acc;
  }
}
template <int PH, typename real>
__device__ __forceinline__ void vec_y(const real* __restrict__ U1, real* __restrict__ U2, int tid) {
  if (tid >= 36 * vec_nterms<PH>()) return;
  const int j = tid / 36, i = tid % 36;
  const int g1 = i % 9, r3 = i / 9;
  const real* u1 = U1 + j * 324 + r3 * 81 + g1;
  real* u2 = U2 + j * 144 + r3 * 36 + g1;
  if (j == 0) vy_task<PH, 0>(u1, u2);
  else if (j == 1) vy_task<PH, 1>(u1, u2);
  else vy_task<PH, 2>(u1, u2);
}
// x: output row r1 of (r2, r3): sum of the terms, scaled, plus the source
template <int PH, int J, int R1, typename real>
__device__ __forceinline__ real vx_term(const real* __restrict__ u2) {
  real acc = 0;
#pragma unroll
  for (int t = 0; t < 6; ++t)
    if (t < vrow_cnt(R1)) acc = fma((real)vrow_coef(vec_tab<PH, J, 0>(), R1, t), u2[vrow_g0(R1) + t], acc);
  return acc;
}
// sum_t B(r, g0 + t) w(g0 + t) over the points of elements inside the mesh (bits vl)
template <int R, typename real>
__device__ __forceinline__ real src_1d(int vl) {
  real acc = 0;
#pragma unroll
  for (int t = 0; t < 6; ++t)
    if (t < vrow_cnt(R) && ((vl >> ((vrow_g0(R) + t) / 3)) & 1))
      acc = fma((real)vrow_coef(VB, R, t), (real)wq((vrow_g0(R) + t) % 3), acc);
  return acc;
}
template <typename real>
__device__ __forceinline__ real src_1d_rt(int r, int vl) {
  return r == 0 ? src_1d<0, real>(vl) : r == 1 ? src_1d<1, real>(vl) : r == 2 ? src_1d<2, real>(vl)
                                                                              : src_1d<3, real>(vl);
}
template <int PH, int R1, typename real>
__device__ __forceinline__ real vx_row(const real* __restrict__ U2, int r2, int r3, real ihx,
                                       real ihy, real ihz) {
  const int o = r3 * 36 + r2 * 9;
  if constexpr (PH == PH_WMM) {
    return vx_term<PH, 0, R1>(U2 + o);
  } else {
    real y = ihx * vx_term<PH, 0, R1>(U2 + o);
    y = fma(ihy, vx_term<PH, 1, R1>(U2 + 144 + o), y);
    return fma(ihz, vx_term<PH, 2, R1>(U2 + 288 + o), y);
  }
}
template <int PH, typename real>
__device__ __forceinline__ real vec_x(const real* __restrict__ U2, int r1, int r2, int r3, real ihx,
                                      real ihy, real ihz) {
  return r1 == 0 ? vx_row<PH, 0>(U2, r2, r3, ihx, ihy, ihz)
       : r1 == 1 ? vx_row<PH, 1>(U2, r2, r3, ihx, ihy, ihz)
       : r1 == 2 ? vx_row<PH, 2>(U2, r2, r3, ihx, ihy, ihz)
                 : vx_row<PH, 3>(U2, r2, r3, ihx, ihy, ihz);
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
  const int xp2 = tid & 15, xp3 = tid >> 4;    // this thread's x task (p2, p3)
  // the copy-out of run xp3 is issued by lane 0 or 16 of a warp (two runs per warp)
  const bool issuer = xp2 == 0;
  // its image offsets in an interior tile, loaded before the set-up's other global reads
  // are waited for (one round trip to memory instead of two)
  const uint4* const tab = reinterpret_cast<const uint4*>(&kTileTabs.inv[xp3][xp2][0]);
  const uint4 tab_a = __ldg(tab), tab_b = __ldg(tab + 1);

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
  // the Dirichlet markers of the halo'd nodes [s3][s2][s1] (343, two per thread at most):
  // loaded now, stored to shared memory at the end of the first phase's y stage (of its
  // z stage for a vector alone), so that their latency hides behind the first field
  // copy and those stages
  uint8_t em[2] = {0, 0};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int i = tid + 256 * h;
    const int s1 = i % 7, s2 = (i / 7) % 7, s3 = i / 49;
    const int gx = 4 * t1 - 2 + s1, gy = 4 * t2 - 2 + s2, gz = 4 * t3 - 2 + s3;
    if (i < 343 && ess != nullptr && gx >= 0 && gx < L.Nx && gy >= 0 && gy < L.Ny && gz >= 0 &&
        gz < L.Nz)
      em[h] = ess[gx + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)];
  }
  // CSR offsets of the rows (0, r2, r3): the lattice pattern's, computed rather than
  // loaded.  The caller's indptr is loaded at the same rows and compared at the last
  // barrier before this tile's first global write (the end of the first phase's x stage,
  // or of its y stage for a vector alone), the load's latency hidden behind the first
  // field copy and the stages: a pattern other than the lattice's is rejected
  // (HM_STATUS_RANGE, nothing written by this tile).
  int32_t given = 0, expect = 0;
  if (tid < 16) {
    const int r2 = tid & 3, r3 = tid >> 2;
    const int gy = 4 * t2 + r2, gz = 4 * t3 + r3;
    const bool live = gy < L.Ny && gz < L.Nz;
    expect = live ? (int32_t)row_start(L, 4 * t1, gy, gz) : 0;
    S.rowptr[tid] = expect;
    given = (live && indptr != nullptr)
                ? __ldg(indptr + (4 * t1 + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)))
                : expect;
  } else if (tid == 16 && indptr != nullptr && t1 == L.tx - 1 && t2 == L.ty - 1 &&
             t3 == L.tz - 1) {
    // the last tile also checks the total
    expect = (int32_t)(stencil_prefix(L.Nx, L.Nx) * stencil_prefix(L.Ny, L.Ny) *
                       stencil_prefix(L.Nz, L.Nz));
    given = __ldg(indptr + L.ndof);
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
  __syncthreads();
  // image layout: run starts (with the parity of the run's CSR offset when the copy-out
  // is a bulk copy) and lengths; a clipped tile packs its clipped rows
  constexpr bool kBulk = sizeof(real) == 8;
  if (tid < 16) {
    const int run = tid;
    const int want = kBulk ? (S.rowptr[run] & 1) : 0;
    if (!clipped) {
      const int a0 = run_sel(run, false);
      S.runstart[run] = a0 + ((want - a0) & 1);
      S.runlen[run] = run_sel(run, true);
    } else {
      // this run's length and its rows' offsets in it; then the runs in order, each at
      // the first slot after the previous one with its parity: a scan over the 16
      // (length, parity) pairs, which every lane runs on shuffled copies
      const int n23 = S.nst[1][run & 3] * S.nst[2][run >> 2];
      int part[4], len = 0;
#pragma unroll
      for (int r1 = 0; r1 < 4; ++r1) {
        part[r1] = len;
        len += S.nst[0][r1] * n23;
      }
      int off = 0, mine = 0;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int lq = __shfl_sync(0xffffu, len, q);
        const int wq_ = __shfl_sync(0xffffu, want, q);
        off += (wq_ - off) & 1;
        if (q == run) mine = off;
        off += lq;
      }
      S.runstart[run] = mine;
      S.runlen[run] = len;
#pragma unroll
      for (int r1 = 0; r1 < 4; ++r1) S.rowoff[run * 4 + r1] = mine + part[r1];
    }
  }
  __syncthreads();

  // ---- this thread's x task (p2, p3): image byte offsets and elimination masks
  uint32_t pk[8];
  {
    if (!clipped) {
      const int run = pair_row_of(xp2) + 4 * pair_row_of(xp3);
      const uint32_t shift = (uint32_t)(S.runstart[run] - run_sel(run, false));   // 0 or 1
      const uint32_t v[8] = {tab_a.x, tab_a.y, tab_a.z, tab_a.w, tab_b.x, tab_b.y, tab_b.z, tab_b.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)   // both halves stay below 2^16
        pk[i] = (v[i] + shift * 0x10001u) * (uint32_t)sizeof(real);
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
        int pos = kSink;
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
  bool has_ess = false;
  // the elimination masks of this thread's x task, from the markers (at the first phase)
  auto ess_masks = [&]() {
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
  };

  // ---- per-thread addresses of the z tasks
  const int zi = tid % 81;                     // (g1, g2) of the z task
  const int zg1 = zi % 9, zg2 = zi / 9;
  const int zbase = ((zg2 / 3) * 3 + zg1 / 3) * BI + zg1 % 3 + 3 * (zg2 % 3);
  const int zt1 = zg2 * 9 + zg1;
  // the source term's 1D factors for this thread's vector output (r1, r2, r3)
  const int vr1 = tid >> 4, vr2 = tid & 3, vr3 = (tid >> 2) & 3;

  unsigned char* const img = reinterpret_cast<unsigned char*>(&S.T1[0][0]);
  real* const U1 = &S.T2[0][0];               // vector scratch: [term][r3][g2][g1]
  real* const U2 = U1 + 3 * 324;              // [term][r3][r2][g1]
  const real ihx = (real)(1.0 / L.hx), ihy = (real)(1.0 / L.hy), ihz = (real)(1.0 / L.hz);

  // a vector entry: the source term (dR/dp), elimination, the store
  auto write_vec = [&](int ph, real y) {
    double* const vec = ph == 1 ? o.vec_adj : ph == 2 ? o.vec_state : o.vec_param;
    if (ph == PH_C) {
      const real src = (real)(L.hx * L.hy * L.hz) * src_1d_rt<real>(vr1, vl[0]) *
                       src_1d_rt<real>(vr2, vl[1]) * src_1d_rt<real>(vr3, vl[2]);
      y = fma((real)(-o.f), src, y);
    }
    const int gx = 4 * t1 + vr1, gy = 4 * t2 + vr2, gz = 4 * t3 + vr3;
    if (gx < L.Nx && gy < L.Ny && gz < L.Nz) {
      double v = (double)y;
      if (o.zero_ess && ph != PH_WMM && S.ess[vr3 + 2][vr2 + 2][vr1 + 2]) v = 0.0;
      vec[gx + (int64_t)L.Nx * (gy + (int64_t)L.Ny * gz)] = v;
    }
  };

  int k = 0;
#pragma unroll 1
  for (int ph = 0; ph < 4; ++ph) {
    if (!((pm >> ph) & 1u)) continue;
    const int buf = k & 1;
    const bool ok = mbar_wait(&S.mbar[buf], (uint32_t)(k >> 1) & 1u);
    // the previous phase's image copies must have left the image before it is rewritten
    if (kBulk && issuer) bulk_wait_read();
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicOr(&g_device_status, HM_STATUS_TIMEOUT);
        // the other buffer's copy, if one is in flight, before the CTA leaves
        const int nx = next_phase(ph);
        if (nx >= 0) (void)mbar_wait(&S.mbar[buf ^ 1], (uint32_t)((k + 1) >> 1) & 1u);
      }
      if (kBulk && issuer) bulk_wait_all();
      return;
    }
    const real* W = reinterpret_cast<const real*>(S.wbuf[buf]) + phase_off<real>(ph);
    double* const vals = ph == 0 ? o.vals[0] : ph == 1 ? o.vals[1] : ph == 2 ? o.vals[2] : o.vals[3];
    double* const vec = ph == 0 ? nullptr : ph == 1 ? o.vec_adj : ph == 2 ? o.vec_state : o.vec_param;
    const int after = next_phase(ph);
    const int after2 = after >= 0 ? next_phase(after) : -1;
    // a barrier that, in the first phase, also takes the markers to shared memory and
    // then forms this thread's elimination masks (the last barrier before the x stage,
    // or before a vector's y stage)
    auto marker_barrier = [&]() {
      if (k != 0) {
        __syncthreads();
        return;
      }
      uint8_t* const es = &S.ess[0][0][0];
      es[tid] = em[0];
      if (tid + 256 < 343) es[tid + 256] = em[1];
      has_ess = __syncthreads_or(em[0] | em[1]) != 0;
      if (has_ess) ess_masks();
    };
    // a barrier that, in the first phase and with `check`, also compares the row
    // pointers (the last barrier before the tile's first global write): false (every
    // thread) when the tile must leave, its copies in flight (the next phase's, and the
    // one after it, issued into this buffer after the z stage) waited for
    auto checked_barrier = [&](bool check) -> bool {
      if (k != 0 || !check) {
        __syncthreads();
        return true;
      }
      if (!__syncthreads_or(given != expect)) return true;
      if (tid == 0) {
        atomicOr(&g_device_status, HM_STATUS_RANGE);
        if (after >= 0) (void)mbar_wait(&S.mbar[buf ^ 1], (uint32_t)((k + 1) >> 1) & 1u);
        if (after2 >= 0) (void)mbar_wait(&S.mbar[buf], (uint32_t)((k + 2) >> 1) & 1u);
      }
      if (kBulk && issuer) bulk_wait_all();
      return false;
    };
    // with its block, a phase's vector is the block's row sums (summed in the x stage)
    const bool rows = vals != nullptr && vec != nullptr;
    real rs[4] = {0, 0, 0, 0};

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
      if ((vec == nullptr || rows) && tid == 0 && after2 >= 0) {
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
      marker_barrier();
      // x: the tile image
      {
        const int r = xp3 * kT2P + xp2 * 9;
        if (ph == PH_A) {
          x_task<TK, TM, true, false>(&S.T2[0][r], &S.T2[1][r], img, pk, has_ess, zA, oA, rs);
        } else if (ph == PH_WMM) {
          if (rows) x_task<TM, TM, false, true>(&S.T2[0][r], (const real*)nullptr, img, pk, false, 0u, 0u, rs);
          else x_task<TM, TM, false, false>(&S.T2[0][r], (const real*)nullptr, img, pk, false, 0u, 0u, rs);
        } else {
          if (rows) x_task<TR, TM, true, true>(&S.T2[0][r], &S.T2[1][r], img, pk, has_ess, zC, 0u, rs);
          else x_task<TR, TM, true, false>(&S.T2[0][r], &S.T2[1][r], img, pk, has_ess, zC, 0u, rs);
        }
      }
      // row sums over the column pairs p2 of each row r2 (lanes b2 .. b2 + n2 - 1 of the
      // half-warp, summed in lane order into lane b2)
      if (rows) {
#pragma unroll
        for (int r1 = 0; r1 < 4; ++r1) {
          const real v = rs[r1];
          const real a1 = __shfl_down_sync(0xffffffffu, v, 1);
          const real a2 = __shfl_down_sync(0xffffffffu, v, 2);
          const real a3 = __shfl_down_sync(0xffffffffu, v, 3);
          const real a4 = __shfl_down_sync(0xffffffffu, v, 4);
          const real s3 = (v + a1) + a2;
          rs[r1] = (xp2 == 0 || xp2 == 8) ? (s3 + a3) + a4 : s3;
        }
      }
      if (kBulk) fence_proxy_async();   // the image stores, before the async copies read them
      if (!checked_barrier(true)) return;
      // the leaders' sums [r1][p3][r2] into the y buffer (free after the x stage); the sums
      // over p3 finish at the end of the phase
      if (rows && (xp2 == 0 || xp2 == 5 || xp2 == 8 || xp2 == 13)) {
        const int r2 = pair_row_of(xp2);
#pragma unroll
        for (int r1 = 0; r1 < 4; ++r1) S.T2[0][r1 * 64 + xp3 * 4 + r2] = rs[r1];
      }
      // stream the image out, run by run (four consecutive rows, one stretch of CSR)
      const real* O = reinterpret_cast<const real*>(img);
      if constexpr (kBulk) {
        if (issuer) {
          const int run = xp3, a0 = S.runstart[run], len = S.runlen[run];
          if (len > 0) {
            double* dst = vals + (int64_t)S.rowptr[run];
            const int h = S.rowptr[run] & 1;   // the values are 16-byte aligned
            if (h) dst[0] = (double)O[a0];
            const int body = (len - h) & ~1;
            if (body > 0) bulk_store(dst + h, O + a0 + h, (uint32_t)body * 8u);
            if ((len - h) & 1) dst[len - 1] = (double)O[a0 + len - 1];
          }
          bulk_commit();
        }
      } else {
#pragma unroll 1
        for (int run = warp; run < 16; run += 8) {
          const int a0 = S.runstart[run], len = S.runlen[run];
          double* dst = vals + (int64_t)S.rowptr[run];
          for (int j = lane; j < len; j += 32) dst[j] = (double)O[a0 + j];
        }
      }
    }
    if (vec != nullptr && !rows) {
      // the vector alone: z (fields still resident), y, x
      if (ph == PH_C) vec_z<PH_C, BI>(W, U1, tid);
      else if (ph == PH_WUM) vec_z<PH_WUM, BI>(W, U1, tid);
      else vec_z<PH_WMM, BI>(W, U1, tid);
      marker_barrier();
      if (tid == 0 && after2 >= 0) {
        fence_proxy_async();
        issue_fields(&tmap, S, buf, after2, e1, e2, e3);
      }
      if (ph == PH_C) vec_y<PH_C>(U1, U2, tid);
      else if (ph == PH_WUM) vec_y<PH_WUM>(U1, U2, tid);
      else vec_y<PH_WMM>(U1, U2, tid);
      if (!checked_barrier(true)) return;
      if (tid < 64) {
        real y = ph == PH_C ? vec_x<PH_C>(U2, vr1, vr2, vr3, ihx, ihy, ihz)
               : ph == PH_WUM ? vec_x<PH_WUM>(U2, vr1, vr2, vr3, ihx, ihy, ihz)
                              : vec_x<PH_WMM>(U2, vr1, vr2, vr3, ihx, ihy, ihz);
        write_vec(ph, y);
      }
    }
    // the y buffers are rewritten by the next phase
    __syncthreads();
    if (rows && tid < 64) {
      // row (vr1, vr2, vr3): its sums over the column pairs p3, in order
      const real* part = &S.T2[0][vr1 * 64 + row_pair_base(vr3) * 4 + vr2];
      real y = (part[0] + part[4]) + part[8];
      if (row_stencil(vr3) == 5) y = (y + part[12]) + part[16];
      write_vec(ph, y);
    }
    ++k;
  }
  if (kBulk && issuer) bulk_wait_all();
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
    if (dev < 0 || dev >= 64) return HM_ERR_UNSUPPORTED;
    if (!configured[dev]) {
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
  // the copy-out moves 16-byte aligned stretches of the value arrays
  for (double* v : {vA, vC, vWum, vWmm})
    if ((reinterpret_cast<uintptr_t>(v) & 15u) != 0) return HM_ERR_ARG;
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
