// Geometric multigrid preconditioner for the lattice Jacobian (sm_100a).
//
// The structured-lattice counterpart of the BoomerAMG preconditioner the reference puts
// in its Jacobian solves (algorithms/linSolvers.py:243-828): a symmetric V-cycle over
//   level 0   the Q2 lattice itself (the matrix-free operator and its Jacobi diagonal),
//   level 1   Q1 on the same elements (the Q2 lattice's vertices),
//   level l   Q1 on elements coarsened 2:1 while every axis stays even and >= 4,
// with Chebyshev-Jacobi smoothing (degree s before and after, the same polynomial, so the
// cycle is symmetric and positive: a fixed linear preconditioner for CG) and a
// Chebyshev solve of higher degree on the coarsest level.  Between any two levels the
// node lattices are 2:1 (F = 2C - 1 nodes per axis: the Q1 space is nested in Q2 and in
// the next finer Q1), so one trilinear prolongation P and its transpose R = P^T (full
// weighting) serve every pair.  Coarse operators are rediscretised: Q1 stiffness with
// one coefficient per element, the Gauss-weighted mean of e^m over the Q2 element
// (level 1), the mean of the 8 children above.  The Dirichlet nodes must be the whole
// boundary: eliminated rows are the identity on every level and restricted residuals
// are zero there.  The set-up is FP64; the cycle runs in FP64 or, on request, in FP32
// on single-precision copies of the level data (the caller's residual read and the result
// written in FP64, the CG around it unchanged).  Deterministic, and free of host
// synchronisation after set-up, so a CG iteration with its V-cycle can be captured as a
// CUDA graph.
#include <cmath>
#include <new>
#include <type_traits>
#include <vector>

#include "hm_common.cuh"
#include "hm_internal.h"

namespace hm {

// a level in the cycle's precision T (the set-up keeps an FP64 copy of every level)
template <typename T>
struct MGLevelT {
  int nx, ny, nz;        // elements
  int Nx, Ny, Nz;        // nodes per axis
  double hx, hy, hz;     // element sizes
  int64_t nodes, elems;
  T* coef;               // per element (levels >= 1)
  T* diag;               // Jacobi diagonal (level 0: the caller's; FP64 levels only)
  T* idiag;              // its reciprocal, by which the smoothers multiply
  T *x, *b, *r, *d, *t;
  double* cheb;          // Chebyshev on the device: [0] theta (d0 = r / (theta diag)),
                         // [1 + k] c1_k, [1 + kChebMax + k] c2_k (d = c1 d + c2 r / diag)
  int degree;
  T* cinv;               // coarsest level with few interior nodes: the inverse of its
                         // interior block (row-major), solved exactly; else nullptr
};
using MGLevel = MGLevelT<double>;
constexpr int kChebMax = 40;

}  // namespace hm

struct hm_mg {
  hm::Lattice L;
  int nlev;
  hm::MGLevel lv[16];
  void* jac;             // level-0 operator data (FP64, from hm_lattice_jacobian_prepare)
  const uint8_t* ess;
  int degree, coarse_degree;
  double* scratch;       // partial sums of the set-up's inner products, eigenvalue state
  const uint8_t* checked_ess;   // the markers last found to be the whole boundary
  int tail_first;        // first level of the one-CTA tail (nlev: none)
  int fused;             // degree-1 smoothing steps fused with their operator pass
  // the FP32 cycle (single != 0): every level's vectors, coefficients, reciprocal
  // diagonal and coarse inverse in single precision, refreshed from the FP64 set-up; the
  // level-0 operator data (the points' D, then the element results) in jac32
  int single;
  hm::MGLevelT<float> lv32[16];
  float* jac32;
};

namespace hm {

constexpr int kMGBlocks = 296;

__device__ __forceinline__ bool on_boundary(int i, int j, int k, int Nx, int Ny, int Nz) {
  return i == 0 || j == 0 || k == 0 || i == Nx - 1 || j == Ny - 1 || k == Nz - 1;
}

// a product rounded on its own (no contraction into a neighbouring add)
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// (A_l x)[n] for a Q1 level: node-centric, identity on the boundary, boundary values of
// x taken as zero in the interior rows; x given by xv(node)
template <typename T, typename XV>
__device__ __forceinline__ T q1_apply_with(const MGLevelT<T>& lv, int64_t n, XV xv) {
  const int i = (int)(n % lv.Nx);
  const int64_t t = n / lv.Nx;
  const int j = (int)(t % lv.Ny), k = (int)(t / lv.Ny);
  if (on_boundary(i, j, k, lv.Nx, lv.Ny, lv.Nz)) return xv(n);
  // 1D element matrices: k = [1 -1; -1 1] / h, m = [2 1; 1 2] h / 6
  const T kx[2] = {T(1.0 / lv.hx), T(-1.0 / lv.hx)}, ky[2] = {T(1.0 / lv.hy), T(-1.0 / lv.hy)},
          kz[2] = {T(1.0 / lv.hz), T(-1.0 / lv.hz)};
  const T mx[2] = {T(lv.hx / 3.0), T(lv.hx / 6.0)}, my[2] = {T(lv.hy / 3.0), T(lv.hy / 6.0)},
          mz[2] = {T(lv.hz / 3.0), T(lv.hz / 6.0)};
  T xs[3][3][3];
#pragma unroll
  for (int dk = 0; dk < 3; ++dk)
#pragma unroll
    for (int dj = 0; dj < 3; ++dj)
#pragma unroll
      for (int di = 0; di < 3; ++di) {
        const int ii = i + di - 1, jj = j + dj - 1, kk = k + dk - 1;
        xs[dk][dj][di] = on_boundary(ii, jj, kk, lv.Nx, lv.Ny, lv.Nz)
                             ? T(0) : xv(ii + (int64_t)lv.Nx * (jj + (int64_t)lv.Ny * kk));
      }
  T acc = T(0);
#pragma unroll
  for (int e3 = 0; e3 < 2; ++e3)
#pragma unroll
    for (int e2 = 0; e2 < 2; ++e2)
#pragma unroll
      for (int e1 = 0; e1 < 2; ++e1) {
        // element (i-1+e1, j-1+e2, k-1+e3); the node's local index is 1 - e
        const T c = lv.coef[(i - 1 + e1) + (int64_t)lv.nx * ((j - 1 + e2) + (int64_t)lv.ny * (k - 1 + e3))];
        T s = T(0);
#pragma unroll
        for (int b3 = 0; b3 < 2; ++b3)
#pragma unroll
          for (int b2 = 0; b2 < 2; ++b2)
#pragma unroll
            for (int b1 = 0; b1 < 2; ++b1) {
              // K[a][b] with a = 1 - e, so |a - b| = |1 - e - b|: entry 0 on the diagonal
              const int o1 = (1 - e1) != b1, o2 = (1 - e2) != b2, o3 = (1 - e3) != b3;
              const T kab = kx[o1] * my[o2] * mz[o3] + mx[o1] * ky[o2] * mz[o3] +
                            mx[o1] * my[o2] * kz[o3];
              s = fma(kab, xs[e3 + b3][e2 + b2][e1 + b1], s);
            }
        acc = fma(c, s, acc);
      }
  return acc;
}
template <typename T>
__device__ __forceinline__ T q1_apply_at(const MGLevelT<T>& lv, const T* __restrict__ x, int64_t n) {
  return q1_apply_with(lv, n, [&](int64_t m) { return x[m]; });
}
// A Chebyshev-Jacobi step of degree 1 of a Q1 level with its operator pass (the same
// arithmetic as k_cheb_start / k_cheb_step / k_cheb_finish around k_q1_apply):
//   from zero (pre-smoothing):  x = d = b idiag / theta,  r = b - A d
//   from xin (post-smoothing):  xout = xin + (b - A xin) idiag / theta   (xout != xin)
template <typename T>
__global__ void __launch_bounds__(256) k_q1_cheb1_from_zero(MGLevelT<T> lv, const T* __restrict__ b) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= lv.nodes) return;
  const T inv_theta = T(1.0 / lv.cheb[0]);
  const T* __restrict__ idiag = lv.idiag;
  // the products rounded on their own (mul_rn), as the step-by-step kernels store them,
  // so that no multiply-add contraction changes a bit
  const T t = q1_apply_with(lv, n, [&](int64_t m) { return mul_rn(inv_theta * b[m], idiag[m]); });
  lv.x[n] = mul_rn(inv_theta * b[n], idiag[n]);
  lv.r[n] = b[n] - t;
}
template <typename T>
__global__ void __launch_bounds__(256) k_q1_cheb1_from_x(MGLevelT<T> lv, const T* __restrict__ b,
                                                         const T* __restrict__ xin,
                                                         T* __restrict__ xout) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= lv.nodes) return;
  const T inv_theta = T(1.0 / lv.cheb[0]);
  const T t = q1_apply_at(lv, xin, n);
  xout[n] = xin[n] + mul_rn(inv_theta * (b[n] - t), lv.idiag[n]);
}
template <typename T>
__global__ void __launch_bounds__(256) k_q1_apply(MGLevelT<T> lv, const T* __restrict__ x,
                                                  T* __restrict__ y) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n < lv.nodes) y[n] = q1_apply_at(lv, x, n);
}

__global__ void k_q1_diag(MGLevel lv, double* __restrict__ diag) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= lv.nodes) return;
  const int i = (int)(n % lv.Nx);
  const int64_t t = n / lv.Nx;
  const int j = (int)(t % lv.Ny), k = (int)(t / lv.Ny);
  if (on_boundary(i, j, k, lv.Nx, lv.Ny, lv.Nz)) { diag[n] = 1.0; return; }
  const double kaa = (1.0 / lv.hx) * (lv.hy / 3.0) * (lv.hz / 3.0) +
                     (lv.hx / 3.0) * (1.0 / lv.hy) * (lv.hz / 3.0) +
                     (lv.hx / 3.0) * (lv.hy / 3.0) * (1.0 / lv.hz);
  double c = 0.0;
  for (int e3 = 0; e3 < 2; ++e3)
    for (int e2 = 0; e2 < 2; ++e2)
      for (int e1 = 0; e1 < 2; ++e1)
        c += lv.coef[(i - 1 + e1) + (int64_t)lv.nx * ((j - 1 + e2) + (int64_t)lv.ny * (k - 1 + e3))];
  diag[n] = c * kaa;
}

// level-1 coefficients: sum_q D(q) / |e| (D = w|J| e^m in the operator's SoA layout)
__global__ void k_coef_from_q2(int64_t ne, const double* __restrict__ Dq, double inv_vol,
                               double* __restrict__ coef) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 27; ++q) s += Dq[(int64_t)q * ne + e];
  coef[e] = s * inv_vol;
}

__global__ void k_recip(int64_t n, const double* __restrict__ a, double* __restrict__ ia) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) ia[i] = 1.0 / a[i];
}

// a coarse element's coefficient: the mean of its 8 children
__global__ void k_coef_coarsen(MGLevel f, MGLevel c, const double* __restrict__ cf,
                               double* __restrict__ cc) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= c.elems) return;
  const int ex = (int)(e % c.nx);
  const int64_t t = e / c.nx;
  const int ey = (int)(t % c.ny), ez = (int)(t / c.ny);
  double s = 0.0;
  for (int z = 0; z < 2; ++z)
    for (int y = 0; y < 2; ++y)
      for (int x = 0; x < 2; ++x)
        s += cf[(2 * ex + x) + (int64_t)f.nx * ((2 * ey + y) + (int64_t)f.ny * (2 * ez + z))];
  cc[e] = 0.125 * s;
}

// b_c = R r_f (full weighting, the transpose of trilinear interpolation); 0 on the
// coarse boundary
template <typename T>
__device__ __forceinline__ T restrict_at(const MGLevelT<T>& f, const MGLevelT<T>& c,
                                         const T* __restrict__ rf, int64_t n) {
  const int i = (int)(n % c.Nx);
  const int64_t t = n / c.Nx;
  const int j = (int)(t % c.Ny), k = (int)(t / c.Ny);
  if (on_boundary(i, j, k, c.Nx, c.Ny, c.Nz)) return T(0);
  const T w[3] = {T(0.5), T(1.0), T(0.5)};
  T s = T(0);
#pragma unroll
  for (int dk = 0; dk < 3; ++dk)
#pragma unroll
    for (int dj = 0; dj < 3; ++dj) {
      const T wjk = w[dj] * w[dk];
      const int64_t row = (int64_t)f.Nx * ((2 * j + dj - 1) + (int64_t)f.Ny * (2 * k + dk - 1));
#pragma unroll
      for (int di = 0; di < 3; ++di) s = fma(wjk * w[di], rf[row + 2 * i + di - 1], s);
    }
  return s;
}
template <typename T>
__global__ void k_restrict(MGLevelT<T> f, MGLevelT<T> c, const T* __restrict__ rf,
                           T* __restrict__ bc) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n < c.nodes) bc[n] = restrict_at(f, c, rf, n);
}

// x_f += P x_c (trilinear); fine boundary nodes untouched
template <typename T>
__device__ __forceinline__ void prolong_add_at(const MGLevelT<T>& f, const MGLevelT<T>& c,
                                               const T* __restrict__ xc,
                                               T* __restrict__ xf, int64_t n) {
  const int i = (int)(n % f.Nx);
  const int64_t t = n / f.Nx;
  const int j = (int)(t % f.Ny), k = (int)(t / f.Ny);
  if (on_boundary(i, j, k, f.Nx, f.Ny, f.Nz)) return;
  const int ci0 = i >> 1, cj0 = j >> 1, ck0 = k >> 1;
  const int ni = (i & 1) + 1, nj = (j & 1) + 1, nk = (k & 1) + 1;
  const T wi = (i & 1) ? T(0.5) : T(1.0), wj = (j & 1) ? T(0.5) : T(1.0), wk = (k & 1) ? T(0.5) : T(1.0);
  T s = T(0);
  for (int dk = 0; dk < nk; ++dk)
    for (int dj = 0; dj < nj; ++dj)
      for (int di = 0; di < ni; ++di)
        s += xc[(ci0 + di) + (int64_t)c.Nx * ((cj0 + dj) + (int64_t)c.Ny * (ck0 + dk))];
  xf[n] += wi * wj * wk * s;
}
template <typename T>
__global__ void k_prolong_add(MGLevelT<T> f, MGLevelT<T> c, const T* __restrict__ xc,
                              T* __restrict__ xf) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n < f.nodes) prolong_add_at(f, c, xc, xf, n);
}

// Chebyshev-Jacobi (idiag: the reciprocal of the Jacobi diagonal): start (r = b - t, or
// r = b with t == nullptr; d = r idiag / theta; x = 0 when zero_x), step (x += d; r -= t;
// d = c1 d + c2 r idiag unless last), finish (x += d)
template <typename T>
__global__ void k_cheb_start(int64_t n, const T* __restrict__ b, const T* __restrict__ t,
                             const T* __restrict__ idiag, const double* __restrict__ cheb,
                             int zero_x, T* __restrict__ x, T* __restrict__ r,
                             T* __restrict__ d) {
  const T inv_theta = T(1.0 / cheb[0]);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T ri = t ? b[i] - t[i] : b[i];
    r[i] = ri;
    d[i] = inv_theta * ri * idiag[i];
    if (zero_x) x[i] = T(0);
  }
}
template <typename T>
__global__ void k_cheb_step(int64_t n, T* __restrict__ x, T* __restrict__ d,
                            T* __restrict__ r, const T* __restrict__ t,
                            const T* __restrict__ idiag, const double* __restrict__ cheb,
                            int k, int last) {
  const T c1 = T(cheb[1 + k]), c2 = T(cheb[1 + kChebMax + k]);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T di = d[i];
    x[i] += di;
    const T ri = r[i] - t[i];
    r[i] = ri;
    if (!last) d[i] = fma(c1, di, c2 * ri * idiag[i]);
  }
}
template <typename T>
__global__ void k_cheb_finish(int64_t n, T* __restrict__ x, const T* __restrict__ d) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += d[i];
}

// ---- exact solve of a small coarsest level
// Interior node q of a level <-> (1 + q % (Nx-2), 1 + (q / (Nx-2)) % (Ny-2), ...).
constexpr int kCoarseDirectMax = 64;
template <typename T>
__device__ __forceinline__ int64_t interior_node(const MGLevelT<T>& lv, int q) {
  const int ax = lv.Nx - 2, ay = lv.Ny - 2;
  return (1 + q % ax) + (int64_t)lv.Nx * ((1 + (q / ax) % ay) + (int64_t)lv.Ny * (1 + q / (ax * ay)));
}
template <typename T>
__host__ __device__ inline int interior_count(const MGLevelT<T>& lv) {
  return (lv.Nx - 2) * (lv.Ny - 2) * (lv.Nz - 2);
}
// set-up (one CTA): the interior block column by column (the operator on unit vectors in
// lv.t), then its inverse by Gauss-Jordan elimination (SPD: no pivoting), into lv.cinv
__global__ void __launch_bounds__(256) k_coarse_factor(MGLevel lv) {
  __shared__ double A[kCoarseDirectMax][kCoarseDirectMax + 1];
  const int n = interior_count(lv);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int64_t i = tid; i < lv.nodes; i += nt) lv.t[i] = 0.0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    if (tid == 0) lv.t[interior_node(lv, j)] = 1.0;
    __syncthreads();
    for (int i = tid; i < n; i += nt) A[i][j] = q1_apply_at(lv, lv.t, interior_node(lv, i));
    __syncthreads();
    if (tid == 0) lv.t[interior_node(lv, j)] = 0.0;
    __syncthreads();
  }
  for (int k = 0; k < n; ++k) {
    const double p = A[k][k];
    __syncthreads();
    if (tid == 0) A[k][k] = 1.0;
    __syncthreads();
    for (int j = tid; j < n; j += nt) A[k][j] = A[k][j] / p;
    __syncthreads();
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e % n;
      if (i != k && j != k) A[i][j] = fma(-A[i][k], A[k][j], A[i][j]);
    }
    __syncthreads();
    for (int i = tid; i < n; i += nt)
      if (i != k) A[i][k] = -A[i][k] * A[k][k];
    __syncthreads();
  }
  for (int e = tid; e < n * n; e += nt) lv.cinv[e] = A[e / n][e % n];
}
// x = A_l^{-1} b for the small coarsest level, inside one CTA (x zero on the boundary)
template <typename T>
__device__ void coarse_direct(const MGLevelT<T>& lv, const T* __restrict__ b, T* __restrict__ x) {
  const int n = interior_count(lv);
  for (int64_t i = threadIdx.x; i < lv.nodes; i += blockDim.x) x[i] = T(0);
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    T acc = T(0);
    for (int j = 0; j < n; ++j) acc = fma(lv.cinv[i * n + j], b[interior_node(lv, j)], acc);
    x[interior_node(lv, i)] = acc;
  }
  __syncthreads();
}
template <typename T>
__global__ void __launch_bounds__(256) k_coarse_solve(MGLevelT<T> lv, const T* __restrict__ b,
                                                      T* __restrict__ x) {
  coarse_direct(lv, b, x);
}

// ---- the small levels of a cycle in one CTA
// The Q1 levels from the first with at most kTailNodes nodes down to the coarsest hold a
// few thousand nodes together; launched level by level they cost ~14 launches per level
// and 2 per step of the coarse solve, each mostly launch latency.  One CTA runs that
// whole part of the V-cycle (the same smoothing, restriction and prolongation, node for
// node, with block barriers where the launches were).
constexpr int kTailMax = 8;
constexpr int64_t kTailNodes = 1000;
constexpr int kTailThreads = 512;
template <typename T>
struct MGTail {
  MGLevelT<T> lv[kTailMax];
  int count;
};
// Chebyshev smoothing of level lv inside the CTA (as smooth() launches it)
template <typename T>
__device__ void tail_smooth(const MGLevelT<T>& lv, bool zero_x, bool want_r, int degree) {
  const int64_t n = lv.nodes;
  const int tid = threadIdx.x, nt = blockDim.x;
  const T* __restrict__ b = lv.b;
  T* __restrict__ x = lv.x;
  T* __restrict__ r = lv.r;
  T* __restrict__ d = lv.d;
  T* __restrict__ t = lv.t;
  const T* __restrict__ idiag = lv.idiag;
  const T inv_theta = T(1.0 / lv.cheb[0]);
  if (!zero_x) {
    for (int64_t i = tid; i < n; i += nt) t[i] = q1_apply_at(lv, x, i);
    __syncthreads();
  }
  for (int64_t i = tid; i < n; i += nt) {
    const T ri = zero_x ? b[i] : b[i] - t[i];
    r[i] = ri;
    d[i] = inv_theta * ri * idiag[i];
    if (zero_x) x[i] = T(0);
  }
  __syncthreads();
  for (int k = 1; k <= degree; ++k) {
    const bool last = k == degree;
    if (last && !want_r) {
      for (int64_t i = tid; i < n; i += nt) x[i] += d[i];
      __syncthreads();
      break;
    }
    for (int64_t i = tid; i < n; i += nt) t[i] = q1_apply_at(lv, d, i);
    __syncthreads();
    const T c1 = T(lv.cheb[1 + k]), c2 = T(lv.cheb[1 + kChebMax + k]);
    for (int64_t i = tid; i < n; i += nt) {
      const T di = d[i];
      x[i] += di;
      const T ri = r[i] - t[i];
      r[i] = ri;
      if (!last) d[i] = fma(c1, di, c2 * ri * idiag[i]);
    }
    __syncthreads();
  }
}
// the V-cycle from T.lv[0] (right-hand side in its b, result in its x) to the coarsest
template <typename R>
__global__ void __launch_bounds__(kTailThreads) k_mg_tail(const __grid_constant__ MGTail<R> T) {
  __shared__ MGLevelT<R> L[kTailMax];
  if (threadIdx.x < (unsigned)T.count) L[threadIdx.x] = T.lv[threadIdx.x];
  __syncthreads();
  const int nl = T.count;
  for (int l = 0; l + 1 < nl; ++l) {
    tail_smooth(L[l], true, true, L[l].degree);
    for (int64_t i = threadIdx.x; i < L[l + 1].nodes; i += blockDim.x)
      L[l + 1].b[i] = restrict_at(L[l], L[l + 1], L[l].r, i);
    __syncthreads();
  }
  if (L[nl - 1].cinv) coarse_direct(L[nl - 1], L[nl - 1].b, L[nl - 1].x);
  else tail_smooth(L[nl - 1], true, false, L[nl - 1].degree);
  for (int l = nl - 2; l >= 0; --l) {
    for (int64_t i = threadIdx.x; i < L[l].nodes; i += blockDim.x)
      prolong_add_at(L[l], L[l + 1], L[l + 1].x, L[l].x, i);
    __syncthreads();
    tail_smooth(L[l], false, false, L[l].degree);
  }
}

// set-up: a deterministic pseudo-random start vector (0 on the boundary), partial sums of
// a.b, and v = w / (s * diag)
__global__ void k_mg_seed(MGLevel lv, double* __restrict__ v) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= lv.nodes) return;
  const int i = (int)(n % lv.Nx);
  const int64_t t = n / lv.Nx;
  const int j = (int)(t % lv.Ny), k = (int)(t / lv.Ny);
  uint64_t h = (uint64_t)n * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  h ^= h >> 31; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 29;
  v[n] = on_boundary(i, j, k, lv.Nx, lv.Ny, lv.Nz) ? 0.0 : (double)(h >> 11) * 0x1.0p-53 - 0.5;
}
__global__ void __launch_bounds__(256) k_mg_dot(int64_t n, const double* __restrict__ a,
                                                const double* __restrict__ b,
                                                const double* __restrict__ w,
                                                double* __restrict__ part) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s = fma(a[i] * (w ? w[i] : 1.0), b[i], s);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}
// partials of v.w, v.diag.v and w.w (slots 0, 1, 2)
__global__ void __launch_bounds__(256) k_mg_dot3(int64_t n, const double* __restrict__ v,
                                                 const double* __restrict__ w,
                                                 const double* __restrict__ diag,
                                                 double* __restrict__ part) {
  __shared__ double sh[32];
  double a = 0.0, b = 0.0, c = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double vi = v[i], wi = w[i];
    a = fma(vi, wi, a);
    b = fma(vi * diag[i], vi, b);
    c = fma(wi, wi, c);
  }
  a = block_sum(a, sh);
  b = block_sum(b, sh);
  c = block_sum(c, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = a;
    part[kMGBlocks + blockIdx.x] = b;
    part[2 * kMGBlocks + blockIdx.x] = c;
  }
}
// eig[0] = v.Av / v.Dv (kept while the iteration is defined), eig[1] = 1 / |w|
__global__ void k_mg_eig_step(const double* __restrict__ part, double* __restrict__ eig) {
  __shared__ double sh[32];
  double v[3];
  for (int q = 0; q < 3; ++q) {
    double t = 0.0;
    for (int b = threadIdx.x; b < kMGBlocks; b += blockDim.x) t += part[q * kMGBlocks + b];
    v[q] = block_sum(t, sh);
  }
  if (threadIdx.x == 0) {
    if (v[1] > 0.0 && v[2] > 0.0 && isfinite(v[0] / v[1])) {
      eig[0] = v[0] / v[1];
      eig[1] = 1.0 / sqrt(v[2]);
    } else {
      eig[1] = 0.0;
    }
  }
}
__global__ void k_mg_scale_div(int64_t n, const double* __restrict__ w, const double* __restrict__ diag,
                               const double* __restrict__ eig, double* __restrict__ v) {
  const double s = eig[1];
  if (s == 0.0) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = s * w[i] / diag[i];
}
// the Chebyshev coefficients of the interval [hi / lo_div, hi], hi = 1.1 lambda
__global__ void k_mg_cheb_coeffs(const double* __restrict__ eig, double lo_div, int degree,
                                 double* __restrict__ cheb) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double hi = 1.1 * eig[0], lo = hi / lo_div;
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
  double rho_old = 1.0 / sigma;
  cheb[0] = theta;
  for (int k = 1; k <= degree && k < kChebMax; ++k) {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    cheb[1 + k] = rho * rho_old;
    cheb[1 + kChebMax + k] = 2.0 * rho / delta;
    rho_old = rho;
  }
}

}  // namespace hm

using namespace hm;

namespace {
inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }
inline int blocks_for(int64_t n) { return (int)((n + 255) / 256); }

// the levels of the cycle in precision T
template <typename T> MGLevelT<T>* levels_of(hm_mg* mg);
template <> MGLevelT<double>* levels_of<double>(hm_mg* mg) { return mg->lv; }
template <> MGLevelT<float>* levels_of<float>(hm_mg* mg) { return mg->lv32; }

// clean: x is zero on the Dirichlet nodes (the level-0 element pass then skips the
// markers); every vector of a cycle is when its right-hand side is
template <typename T>
int apply_level(hm_mg* mg, int l, const T* x, T* y, bool clean, cudaStream_t s) {
  if (l == 0) {
    if constexpr (std::is_same<T, double>::value) {
      if (clean) return hm_launch_apply_A_clean(mg->L, mg->jac, mg->ess, x, y, (void*)s);
      return hm_launch_apply_A(mg->L, mg->jac, HM_FP64, mg->ess, x, y, (void*)s);
    } else {
      return hm_launch_apply_A32(mg->L, mg->jac32, mg->ess, x, y, clean, (void*)s);
    }
  }
  const MGLevelT<T>& lv = levels_of<T>(mg)[l];
  k_q1_apply<T><<<blocks_for(lv.nodes), 256, 0, s>>>(lv, x, y);
  return HM_OK;
}

// Chebyshev smoothing of A_l x = b: from x = 0 (zero_x) or from the given x; with
// want_r the residual b - A x of the result is left in lv.r
template <typename T>
int smooth(hm_mg* mg, int l, const T* b, T* x, bool zero_x, bool want_r, int degree,
           bool clean, cudaStream_t s) {
  MGLevelT<T>& lv = levels_of<T>(mg)[l];
  int rc;
  const int g = kMGBlocks;
  if (zero_x) {
    k_cheb_start<T><<<g, 256, 0, s>>>(lv.nodes, b, nullptr, lv.idiag, lv.cheb, 1, x, lv.r, lv.d);
  } else {
    if ((rc = apply_level<T>(mg, l, x, lv.t, clean, s))) return rc;
    k_cheb_start<T><<<g, 256, 0, s>>>(lv.nodes, b, lv.t, lv.idiag, lv.cheb, 0, x, lv.r, lv.d);
  }
  for (int k = 1; k <= degree; ++k) {
    const bool last = k == degree;
    if (last && !want_r) {
      k_cheb_finish<T><<<g, 256, 0, s>>>(lv.nodes, x, lv.d);
      break;
    }
    if ((rc = apply_level<T>(mg, l, lv.d, lv.t, clean, s))) return rc;
    k_cheb_step<T><<<g, 256, 0, s>>>(lv.nodes, x, lv.d, lv.r, lv.t, lv.idiag, lv.cheb, k, last ? 1 : 0);
  }
  return HM_OK;
}

// The V-cycle from level l for A_l x = b.  *out: where the result lies -- x, except
// for a Q1 level whose fused post-smoothing writes it to the level's lv.t.  In FP32 the
// fused level-0 steps are taken by vcycle_single (they read and write FP64 vectors).
template <typename T>
int vcycle(hm_mg* mg, int l, const T* b, T* x, bool clean, cudaStream_t s, T** out) {
  int rc;
  *out = x;
  MGLevelT<T>* lvs = levels_of<T>(mg);
  if (l == mg->tail_first && b == lvs[l].b && x == lvs[l].x) {
    MGTail<T> TL{};
    TL.count = mg->nlev - l;
    for (int q = 0; q < TL.count; ++q) TL.lv[q] = lvs[l + q];
    k_mg_tail<T><<<1, kTailThreads, 0, s>>>(TL);
    return HM_OK;
  }
  if (l == mg->nlev - 1) {
    if (lvs[l].cinv) {
      k_coarse_solve<T><<<1, 256, 0, s>>>(lvs[l], b, x);
      return HM_OK;
    }
    return smooth<T>(mg, l, b, x, true, false, mg->coarse_degree, clean, s);
  }
  MGLevelT<T>& lv = lvs[l];
  MGLevelT<T>& cv = lvs[l + 1];
  // degree 1 fused with the operator: on level 0 when every vector is zero on the
  // Dirichlet nodes (inside the solves), on a Q1 level when its own buffers carry it
  constexpr bool kFP64 = std::is_same<T, double>::value;
  const bool fuse = mg->fused && mg->degree == 1 &&
                    (l == 0 ? kFP64 && clean : (b == lv.b && x == lv.x));
  if (fuse && l == 0) {
    if constexpr (kFP64) {
      if ((rc = hm_launch_cheb1_from_zero(mg->L, mg->jac, mg->ess, b, lv.idiag, lv.cheb, x, lv.r,
                                          (void*)s)))
        return rc;
    }
  } else if (fuse) {
    k_q1_cheb1_from_zero<T><<<blocks_for(lv.nodes), 256, 0, s>>>(lv, b);
  } else if ((rc = smooth<T>(mg, l, b, x, true, true, mg->degree, clean, s))) {
    return rc;
  }
  k_restrict<T><<<blocks_for(cv.nodes), 256, 0, s>>>(lv, cv, lv.r, cv.b);
  T* xc = nullptr;
  if ((rc = vcycle<T>(mg, l + 1, cv.b, cv.x, clean, s, &xc))) return rc;
  k_prolong_add<T><<<blocks_for(lv.nodes), 256, 0, s>>>(lv, cv, xc, x);
  if (fuse && l == 0) {
    if constexpr (kFP64)
      return hm_launch_cheb1_from_x(mg->L, mg->jac, mg->ess, b, lv.idiag, lv.cheb, x, (void*)s);
  }
  if (fuse) {
    k_q1_cheb1_from_x<T><<<blocks_for(lv.nodes), 256, 0, s>>>(lv, b, x, lv.t);
    *out = lv.t;
    return HM_OK;
  }
  return smooth<T>(mg, l, b, x, false, false, mg->degree, clean, s);
}

__global__ void k_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_to_double(int64_t n, const float* __restrict__ a, double* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

// z = V(r) with the cycle in FP32: r and z FP64.  With degree-1 fused smoothing inside
// the solves (clean) the level-0 passes read r and write z themselves; otherwise r is
// rounded to FP32 first and the result widened at the end.
int vcycle_single(hm_mg* mg, const double* r, double* z, bool clean, cudaStream_t s) {
  MGLevelT<float>* lv = mg->lv32;
  int rc;
  if (mg->fused && mg->degree == 1 && clean && mg->nlev > 1) {
    const MGLevel& l0 = mg->lv[0];
    if ((rc = hm_launch_cheb1_from_zero32(mg->L, mg->jac32, mg->ess, r, l0.idiag, l0.cheb,
                                          lv[0].x, lv[0].r, (void*)s)))
      return rc;
    k_restrict<float><<<blocks_for(lv[1].nodes), 256, 0, s>>>(lv[0], lv[1], lv[0].r, lv[1].b);
    float* xc = nullptr;
    if ((rc = vcycle<float>(mg, 1, lv[1].b, lv[1].x, clean, s, &xc))) return rc;
    k_prolong_add<float><<<blocks_for(lv[0].nodes), 256, 0, s>>>(lv[0], lv[1], xc, lv[0].x);
    return hm_launch_cheb1_from_x32(mg->L, mg->jac32, mg->ess, r, l0.idiag, l0.cheb, lv[0].x, z,
                                    (void*)s);
  }
  k_to_float<<<kMGBlocks, 256, 0, s>>>(lv[0].nodes, r, lv[0].b);
  float* out = nullptr;
  if ((rc = vcycle<float>(mg, 0, lv[0].b, lv[0].x, clean, s, &out))) return rc;
  k_to_double<<<kMGBlocks, 256, 0, s>>>(lv[0].nodes, out, z);
  return HM_OK;
}

// the one-CTA tail: the Q1 levels (l >= 1) of at most max_nodes nodes, at most kTailMax
// of them (max_nodes = 0: none)
void set_tail(hm_mg* mg, int64_t max_nodes) {
  mg->tail_first = mg->nlev;
  for (int l = mg->nlev - 1; l >= 1 && mg->lv[l].nodes <= max_nodes && mg->nlev - l <= kTailMax; --l)
    mg->tail_first = l;
}

// the level hierarchy of a lattice (no memory touched)
int plan_levels(const Lattice& L, MGLevel* lv, int max_levels) {
  int nl = 0;
  MGLevel z{};
  z.nx = L.nx; z.ny = L.ny; z.nz = L.nz;
  z.Nx = L.Nx; z.Ny = L.Ny; z.Nz = L.Nz;
  z.hx = L.hx; z.hy = L.hy; z.hz = L.hz;
  z.nodes = L.ndof; z.elems = L.ne;
  lv[nl++] = z;
  MGLevel q = z;                       // Q1 on the same elements
  q.Nx = L.nx + 1; q.Ny = L.ny + 1; q.Nz = L.nz + 1;
  q.nodes = (int64_t)q.Nx * q.Ny * q.Nz;
  if (L.nx < 2 || L.ny < 2 || L.nz < 2) return nl;
  lv[nl++] = q;
  while (nl < max_levels) {
    const MGLevel& f = lv[nl - 1];
    if ((f.nx & 1) || (f.ny & 1) || (f.nz & 1) || f.nx < 4 || f.ny < 4 || f.nz < 4) break;
    MGLevel c{};
    c.nx = f.nx / 2; c.ny = f.ny / 2; c.nz = f.nz / 2;
    c.Nx = c.nx + 1; c.Ny = c.ny + 1; c.Nz = c.nz + 1;
    c.hx = 2 * f.hx; c.hy = 2 * f.hy; c.hz = 2 * f.hz;
    c.nodes = (int64_t)c.Nx * c.Ny * c.Nz;
    c.elems = (int64_t)c.nx * c.ny * c.nz;
    lv[nl++] = c;
  }
  return nl;
}

// the coarsest level is solved exactly (through its inverse) when it is a Q1 level with
// few interior nodes
bool exact_coarsest(const hm_mg* mg, int l) {
  if (mg->nlev < 2 || l != mg->nlev - 1) return false;
  const int ni = interior_count(mg->lv[l]);
  return ni >= 1 && ni <= kCoarseDirectMax;
}

// the FP32 copies of the level data on work32 (in floats; each piece starts on 128 bytes)
int64_t layout_single(hm_mg* mg, float* work32) {
  float* w = work32;
  int64_t used = 0;
  auto take = [&](int64_t n) {
    const int64_t m = (n + 31) / 32 * 32;
    float* p = w ? w + used : nullptr;
    used += m;
    return p;
  };
  const Lattice& L = mg->L;
  float* jac = take(54 * L.ne);
  if (work32) mg->jac32 = jac;
  for (int l = 0; l < mg->nlev; ++l) {
    const MGLevel& d = mg->lv[l];
    MGLevelT<float> f{};
    f.nx = d.nx; f.ny = d.ny; f.nz = d.nz;
    f.Nx = d.Nx; f.Ny = d.Ny; f.Nz = d.Nz;
    f.hx = d.hx; f.hy = d.hy; f.hz = d.hz;
    f.nodes = d.nodes; f.elems = d.elems;
    f.coef = l >= 1 ? take(d.elems) : nullptr;
    f.diag = nullptr;
    f.idiag = take(d.nodes);
    f.x = take(d.nodes); f.b = take(d.nodes); f.r = take(d.nodes);
    f.d = take(d.nodes); f.t = take(d.nodes);
    f.cinv = exact_coarsest(mg, l) ? take(kCoarseDirectMax * kCoarseDirectMax) : nullptr;
    f.cheb = d.cheb;
    f.degree = d.degree;
    if (work32) mg->lv32[l] = f;
  }
  return used;
}

// the FP32 level data from the FP64 set-up (the point's D, coefficients, reciprocal
// diagonals, the coarse inverse; the Chebyshev coefficients are shared)
void refresh_single(hm_mg* mg, cudaStream_t s) {
  const Lattice& L = mg->L;
  k_to_float<<<4 * kMGBlocks, 256, 0, s>>>(27 * L.ne, static_cast<const double*>(mg->jac), mg->jac32);
  for (int l = 0; l < mg->nlev; ++l) {
    const MGLevel& d = mg->lv[l];
    MGLevelT<float>& f = mg->lv32[l];
    f.degree = d.degree;
    k_to_float<<<kMGBlocks, 256, 0, s>>>(d.nodes, d.idiag, f.idiag);
    if (l >= 1) k_to_float<<<kMGBlocks, 256, 0, s>>>(d.elems, d.coef, f.coef);
    if (d.cinv) {
      const int ni = interior_count(d);
      k_to_float<<<1, 256, 0, s>>>((int64_t)ni * ni, d.cinv, f.cinv);
    }
  }
}

__global__ void k_count_mismatch(Lattice L, const uint8_t* __restrict__ ess, unsigned* __restrict__ bad) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= L.ndof) return;
  const int i = (int)(n % L.Nx);
  const int64_t t = n / L.Nx;
  const int j = (int)(t % L.Ny), k = (int)(t / L.Ny);
  const bool b = on_boundary(i, j, k, L.Nx, L.Ny, L.Nz);
  if ((ess != nullptr && ess[n] != 0) != b) atomicAdd(bad, 1u);
}
}  // namespace

// inside the MG-PCG, whose residuals are zero on the Dirichlet nodes
int hm_mg_vcycle(hm_mg* mg, const double* r, double* z, void* stream) {
  if (mg->single) return vcycle_single(mg, r, z, true, S_(stream));
  double* out = nullptr;
  return vcycle<double>(mg, 0, r, z, true, S_(stream), &out);
}
bool hm_mg_flexible(const hm_mg* mg) { return mg->single != 0; }
const double* hm_mg_level0_diag(const hm_mg* mg) { return mg->lv[0].diag; }
void* hm_mg_jac(const hm_mg* mg) { return mg->jac; }
const uint8_t* hm_mg_ess(const hm_mg* mg) { return mg->ess; }
const hm::Lattice* hm_mg_lattice(const hm_mg* mg) { return &mg->L; }

extern "C" int64_t hm_mg_workspace_bytes(const hm_lattice* h) {
  const Lattice* L = hm_lattice_geometry(h);
  if (!L) return 0;
  MGLevel lv[16];
  const int nl = plan_levels(*L, lv, 16);
  int64_t doubles = 4 * L->ndof + 3 * kMGBlocks + 64 + nl * (2 * kChebMax + 8) +
                    kCoarseDirectMax * kCoarseDirectMax + 8;
  for (int l = 1; l < nl; ++l) doubles += lv[l].elems + 7 * lv[l].nodes + 8;
  return doubles * (int64_t)sizeof(double);
}

extern "C" int hm_mg_create(const hm_lattice* h, void* work, int degree, int coarse_degree,
                            hm_mg** out) {
  const Lattice* L = hm_lattice_geometry(h);
  if (!L || !work || !out || degree < 1 || degree >= kChebMax || coarse_degree < 1 ||
      coarse_degree >= kChebMax)
    return HM_ERR_ARG;
  hm_mg* mg = new (std::nothrow) hm_mg();
  if (!mg) return HM_ERR_NOMEM;
  mg->L = *L;
  mg->degree = degree;
  mg->coarse_degree = coarse_degree;
  mg->nlev = plan_levels(*L, mg->lv, 16);
  set_tail(mg, kTailNodes);
  mg->fused = 1;
  mg->single = 0;
  mg->jac32 = nullptr;
  double* w = static_cast<double*>(work);
  auto take = [&](int64_t n) { double* p = w; w += n; return p; };
  mg->scratch = take(3 * kMGBlocks + 64);
  mg->checked_ess = nullptr;
  for (int l = 0; l < mg->nlev; ++l) mg->lv[l].cheb = take(2 * kChebMax + 8);
  MGLevel& z = mg->lv[0];
  z.r = take(L->ndof); z.d = take(L->ndof); z.t = take(L->ndof); z.idiag = take(L->ndof);
  z.x = z.b = nullptr; z.coef = nullptr; z.diag = nullptr;
  for (int l = 1; l < mg->nlev; ++l) {
    MGLevel& lv = mg->lv[l];
    lv.coef = take(lv.elems);
    lv.diag = take(lv.nodes);
    lv.idiag = take(lv.nodes);
    lv.x = take(lv.nodes); lv.b = take(lv.nodes); lv.r = take(lv.nodes);
    lv.d = take(lv.nodes); lv.t = take(lv.nodes);
    lv.cinv = nullptr;
    w += 8;
  }
  z.cinv = nullptr;
  // an exact coarse solve when the coarsest Q1 level has few interior nodes
  if (exact_coarsest(mg, mg->nlev - 1))
    mg->lv[mg->nlev - 1].cinv = take(kCoarseDirectMax * kCoarseDirectMax);
  *out = mg;
  return HM_OK;
}

// the point's operator: coefficients, diagonals and eigenvalue bounds, all on the device
// (the first set-up with a marker array checks it: one synchronisation)
extern "C" int hm_mg_setup(hm_mg* mg, void* jac, const uint8_t* ess, const double* diag,
                           void* stream) {
  if (!mg || !jac || !ess || !diag) return HM_ERR_ARG;
  cudaStream_t s = S_(stream);
  const Lattice& L = mg->L;
  // the Dirichlet nodes must be exactly the boundary (checked once per marker array)
  if (ess != mg->checked_ess) {
    unsigned* bad = reinterpret_cast<unsigned*>(mg->scratch + 3 * kMGBlocks + 8);
    if (cudaMemsetAsync(bad, 0, sizeof(unsigned), s) != cudaSuccess) return HM_ERR_CUDA;
    k_count_mismatch<<<blocks_for(L.ndof), 256, 0, s>>>(L, ess, bad);
    unsigned hbad = 0;
    if (cudaMemcpyAsync(&hbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return HM_ERR_CUDA;
    if (hbad != 0) return HM_ERR_UNSUPPORTED;
    mg->checked_ess = ess;
  }
  mg->jac = jac;
  mg->ess = ess;
  mg->lv[0].diag = const_cast<double*>(diag);
  // coefficients and diagonals of the Q1 levels
  if (mg->nlev > 1) {
    MGLevel& q = mg->lv[1];
    k_coef_from_q2<<<blocks_for(L.ne), 256, 0, s>>>(L.ne, static_cast<const double*>(jac),
                                                    1.0 / (L.hx * L.hy * L.hz), q.coef);
    for (int l = 2; l < mg->nlev; ++l)
      k_coef_coarsen<<<blocks_for(mg->lv[l].elems), 256, 0, s>>>(mg->lv[l - 1], mg->lv[l],
                                                                  mg->lv[l - 1].coef, mg->lv[l].coef);
    for (int l = 1; l < mg->nlev; ++l)
      k_q1_diag<<<blocks_for(mg->lv[l].nodes), 256, 0, s>>>(mg->lv[l], mg->lv[l].diag);
  }
  for (int l = 0; l < mg->nlev; ++l)
    k_recip<<<blocks_for(mg->lv[l].nodes), 256, 0, s>>>(mg->lv[l].nodes, mg->lv[l].diag,
                                                        mg->lv[l].idiag);
  // largest eigenvalue of D^{-1} A per level, on the device: power iteration with the
  // Rayleigh quotient v.Av / v.Dv (10 steps from a fixed start); smoothing interval
  // [hi/4, hi], the coarsest level's solve on [hi/64, hi]
  double* part = mg->scratch;
  double* eig = mg->scratch + 3 * kMGBlocks;
  for (int l = 0; l < mg->nlev; ++l) {
    MGLevel& lv = mg->lv[l];
    double* v = lv.d;
    double* w = lv.t;
    k_mg_seed<<<blocks_for(lv.nodes), 256, 0, s>>>(lv, v);
    if (cudaMemsetAsync(eig, 0, 2 * sizeof(double), s) != cudaSuccess) return HM_ERR_CUDA;
    for (int it = 0; it < 10; ++it) {
      const int rc = apply_level(mg, l, v, w, true, s);   // v is zero on the boundary
      if (rc) return rc;
      k_mg_dot3<<<kMGBlocks, 256, 0, s>>>(lv.nodes, v, w, lv.diag, part);
      k_mg_eig_step<<<1, 256, 0, s>>>(part, eig);
      k_mg_scale_div<<<kMGBlocks, 256, 0, s>>>(lv.nodes, w, lv.diag, eig, v);
    }
    const bool coarsest = l == mg->nlev - 1;
    lv.degree = coarsest ? mg->coarse_degree : mg->degree;
    k_mg_cheb_coeffs<<<1, 32, 0, s>>>(eig, coarsest ? 64.0 : 4.0, lv.degree, lv.cheb);
    if (coarsest && lv.cinv) k_coarse_factor<<<1, 256, 0, s>>>(lv);
  }
  if (mg->single) refresh_single(mg, s);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

extern "C" int hm_mg_set_tail_nodes(hm_mg* mg, int64_t max_nodes) {
  if (!mg || max_nodes < 0) return HM_ERR_ARG;
  set_tail(mg, max_nodes);
  return HM_OK;
}

extern "C" int64_t hm_mg_single_workspace_bytes(const hm_lattice* h) {
  const Lattice* L = hm_lattice_geometry(h);
  if (!L) return 0;
  hm_mg probe{};
  probe.L = *L;
  probe.nlev = plan_levels(*L, probe.lv, 16);
  return layout_single(&probe, nullptr) * (int64_t)sizeof(float);
}

// the cycle in FP32 on work32 (hm_mg_single_workspace_bytes), or back in FP64 (null);
// after a set-up the FP32 data are formed at once, on stream
extern "C" int hm_mg_set_single(hm_mg* mg, void* work32, void* stream) {
  if (!mg) return HM_ERR_ARG;
  if (work32 == nullptr) {
    mg->single = 0;
    return HM_OK;
  }
  layout_single(mg, static_cast<float*>(work32));
  mg->single = 1;
  if (mg->jac) {
    refresh_single(mg, S_(stream));
    if (cudaGetLastError() != cudaSuccess) return HM_ERR_CUDA;
  }
  return HM_OK;
}

extern "C" int hm_mg_set_fused(hm_mg* mg, int fused) {
  if (!mg) return HM_ERR_ARG;
  mg->fused = fused != 0;
  return HM_OK;
}

extern "C" int hm_mg_apply(hm_mg* mg, const double* r, double* z, void* stream) {
  if (!mg || !r || !z || !mg->jac) return HM_ERR_ARG;
  double* out = nullptr;
  const int rc = mg->single ? vcycle_single(mg, r, z, false, S_(stream))
                            : vcycle<double>(mg, 0, r, z, false, S_(stream), &out);
  if (rc) return rc;
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}

extern "C" int hm_mg_levels(const hm_mg* mg) { return mg ? mg->nlev : 0; }

extern "C" int hm_mg_destroy(hm_mg* mg) {
  delete mg;
  return HM_OK;
}
