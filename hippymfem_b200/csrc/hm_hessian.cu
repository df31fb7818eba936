// The reduced-Hessian action behind the C ABI: ReducedHessian.mult
// (hippymfem/modeling/reducedHessian.py:87-131) for the Q2 log-conductivity problem at
// an assembled linearization point,
//   uhat = A^{-1} (C x)                         (incremental forward solve)
//   phat = A^{-T} (W_uu uhat - W_um x)          (incremental adjoint solve; A^T = A)
//   y    = W_mm x + C^T phat - W_mu uhat        (TrueHessian; GNHessian: y = C^T phat)
// with both right-hand sides zeroed on the Dirichlet dofs (solveIncremental,
// modeling/PDEVariationalProblem.py:1583-1609) and W_uu = B^T B / noise_variance of the
// pointwise misfit (modeling/misfit.py:102-110).  The blocks are CSR on the lattice
// pattern (transposed products through its transpose map); the solves run on the
// caller's solve plan (FP64 Jacobi-, multigrid- or mixed-precision PCG).  Every step is
// one of the library's own launches on the caller's stream; the plan's convergence
// checks are its only host synchronisations.
#include <new>

#include "hm_common.cuh"
#include "hm_internal.h"

struct hm_hessian {
  int64_t n;
  const int32_t* indptr;
  const int32_t* indices;
  const int32_t* tpos;
  const double* C;
  const double* Wum;        // NULL with Wmm: Gauss-Newton
  const double* Wmm;
  int64_t nobs;
  const int32_t* B_indptr;  // observation operator (nobs x n) and its transpose (n x nobs)
  const int32_t* B_indices;
  const double* B_vals;
  const int32_t* Bt_indptr;
  const int32_t* Bt_indices;
  const double* Bt_vals;
  double inv_noise;
  const uint8_t* ess;
  hm_pcg_plan* plan;
  double* plan_b;
  double* plan_x;
  double* t;                // work: n
  double* uhat;             // work: n
  double* bu;               // work: nobs
};

namespace {
inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// dst = src with the Dirichlet entries zeroed
__global__ void k_masked_copy(int64_t n, const uint8_t* __restrict__ ess, const double* __restrict__ src,
                              double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (ess != nullptr && ess[i]) ? 0.0 : src[i];
}

int masked_copy(int64_t n, const uint8_t* ess, const double* src, double* dst, void* stream) {
  const int64_t want = (n + 255) / 256;
  k_masked_copy<<<(int)(want < 2368 ? want : 2368), 256, 0, S_(stream)>>>(n, ess, src, dst);
  return cudaGetLastError() == cudaSuccess ? HM_OK : HM_ERR_CUDA;
}
}  // namespace

extern "C" int64_t hm_hessian_workspace_bytes(int64_t n, int64_t nobs) {
  if (n < 0 || nobs < 0) return 0;
  return 8 * (2 * n + (nobs > 0 ? nobs : 1)) + 256;
}

extern "C" int hm_hessian_create(const hm_lattice* h, const int32_t* d_indptr,
                                 const int32_t* d_indices, const int32_t* d_tpos,
                                 const double* d_vals_C, const double* d_vals_Wum,
                                 const double* d_vals_Wmm, int64_t nobs,
                                 const int32_t* d_B_indptr, const int32_t* d_B_indices,
                                 const double* d_B_vals, const int32_t* d_Bt_indptr,
                                 const int32_t* d_Bt_indices, const double* d_Bt_vals,
                                 double noise_variance, const uint8_t* d_ess, hm_pcg_plan* plan,
                                 void* d_work, hm_hessian** out) {
  const hm::Lattice* L = h ? hm_lattice_geometry(h) : nullptr;
  if (!L || !d_indptr || !d_indices || !d_tpos || !d_vals_C || !plan || !d_work || !out)
    return HM_ERR_ARG;
  if ((d_vals_Wum == nullptr) != (d_vals_Wmm == nullptr)) return HM_ERR_ARG;
  if (nobs < 0) return HM_ERR_ARG;
  if (nobs > 0 && (!d_B_indptr || !d_B_indices || !d_B_vals || !d_Bt_indptr || !d_Bt_indices ||
                   !d_Bt_vals || !(noise_variance > 0)))
    return HM_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(d_work) & 7u) != 0) return HM_ERR_ARG;
  hm_hessian* H = new (std::nothrow) hm_hessian();
  if (!H) return HM_ERR_NOMEM;
  H->n = L->ndof;
  H->indptr = d_indptr; H->indices = d_indices; H->tpos = d_tpos;
  H->C = d_vals_C; H->Wum = d_vals_Wum; H->Wmm = d_vals_Wmm;
  H->nobs = nobs;
  H->B_indptr = d_B_indptr; H->B_indices = d_B_indices; H->B_vals = d_B_vals;
  H->Bt_indptr = d_Bt_indptr; H->Bt_indices = d_Bt_indices; H->Bt_vals = d_Bt_vals;
  H->inv_noise = nobs > 0 ? 1.0 / noise_variance : 0.0;
  H->ess = d_ess;
  H->plan = plan;
  if (hm_plan_buffers(plan, &H->plan_b, &H->plan_x) != HM_OK) {
    delete H;
    return HM_ERR_ARG;
  }
  double* w = static_cast<double*>(d_work);
  H->t = w;
  H->uhat = w + H->n;
  H->bu = w + 2 * H->n;
  *out = H;
  return HM_OK;
}

extern "C" int hm_hessian_destroy(hm_hessian* H) {
  delete H;
  return HM_OK;
}

#define HM_TRY(call)          \
  do {                        \
    const int rc_ = (call);   \
    if (rc_ != HM_OK) return rc_; \
  } while (0)

extern "C" int hm_hessian_apply(hm_hessian* H, const double* d_x, double* d_y, double rtol,
                                int maxiter, int* iterations, void* stream) {
  if (!H || !d_x || !d_y || d_x == d_y || !(rtol > 0) || maxiter <= 0) return HM_ERR_ARG;
  const int64_t n = H->n;
  int it[2] = {0, 0}, upd = 0;
  double rel = 0.0;
  // uhat = A^{-1} (C x), right-hand side zeroed on the Dirichlet dofs
  HM_TRY(hm_csr_spmv(n, H->indptr, H->indices, H->C, d_x, H->t, 1.0, 0.0, stream));
  HM_TRY(masked_copy(n, H->ess, H->t, H->plan_b, stream));
  HM_TRY(hm_pcg_plan_solve(H->plan, rtol, 0.1, 64, maxiter, &it[0], &upd, &rel, stream));
  if (cudaMemcpyAsync(H->uhat, H->plan_x, 8 * n, cudaMemcpyDeviceToDevice, S_(stream)) != cudaSuccess)
    return HM_ERR_CUDA;
  // phat = A^{-T} (W_uu uhat - W_um x)
  if (H->nobs > 0) {
    HM_TRY(hm_csr_spmv(H->nobs, H->B_indptr, H->B_indices, H->B_vals, H->uhat, H->bu, 1.0, 0.0,
                       stream));
    HM_TRY(hm_csr_spmv(n, H->Bt_indptr, H->Bt_indices, H->Bt_vals, H->bu, H->t, H->inv_noise, 0.0,
                       stream));
  } else if (cudaMemsetAsync(H->t, 0, 8 * n, S_(stream)) != cudaSuccess) {
    return HM_ERR_CUDA;
  }
  if (H->Wum)
    HM_TRY(hm_csr_spmv(n, H->indptr, H->indices, H->Wum, d_x, H->t, -1.0, 1.0, stream));
  HM_TRY(masked_copy(n, H->ess, H->t, H->plan_b, stream));
  HM_TRY(hm_pcg_plan_solve(H->plan, rtol, 0.1, 64, maxiter, &it[1], &upd, &rel, stream));
  // y = W_mm x + C^T phat - W_mu uhat
  if (H->Wmm) {
    HM_TRY(hm_csr_spmv(n, H->indptr, H->indices, H->Wmm, d_x, d_y, 1.0, 0.0, stream));
    HM_TRY(hm_csr_spmv_t(n, H->indptr, H->indices, H->tpos, H->C, H->plan_x, d_y, 1.0, 1.0, stream));
    HM_TRY(hm_csr_spmv_t(n, H->indptr, H->indices, H->tpos, H->Wum, H->uhat, d_y, -1.0, 1.0,
                         stream));
  } else {
    HM_TRY(hm_csr_spmv_t(n, H->indptr, H->indices, H->tpos, H->C, H->plan_x, d_y, 1.0, 0.0, stream));
  }
  if (iterations) {
    iterations[0] = it[0];
    iterations[1] = it[1];
  }
  return HM_OK;
}
