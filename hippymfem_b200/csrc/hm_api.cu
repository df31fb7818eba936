// C ABI of libhippymfem_b200: argument checks, the lattice handle and dispatch.
#include <cstdlib>
#include <new>

#include "hm_common.cuh"
#include "hm_internal.h"

struct hm_lattice {
  hm::Lattice L;
};

namespace {
inline bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }
}  // namespace

const hm::Lattice* hm_lattice_geometry(const hm_lattice* h) { return &h->L; }

extern "C" const char* hm_error_string(int code) {
  switch (code) {
    case HM_OK: return "ok";
    case HM_ERR_ARG: return "invalid argument or size mismatch";
    case HM_ERR_CUDA: return "CUDA runtime error";
    case HM_ERR_NONFINITE: return "non-finite values";
    case HM_ERR_NOMEM: return "workspace too small";
    case HM_ERR_NOCONV: return "iterative solve did not converge";
    case HM_ERR_RANGE: return "index out of range";
    case HM_ERR_UNSUPPORTED: return "unsupported case";
    default: return "unknown error";
  }
}

extern "C" int hm_version(void) { return 100; }

extern "C" int hm_lattice_create(int nx, int ny, int nz, double Lx, double Ly, double Lz,
                                 hm_lattice** out) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || !(Lx > 0) || !(Ly > 0) || !(Lz > 0)) return HM_ERR_ARG;
  hm::Lattice L;
  L.nx = nx; L.ny = ny; L.nz = nz;
  L.Nx = 2 * nx + 1; L.Ny = 2 * ny + 1; L.Nz = 2 * nz + 1;
  L.tx = (L.Nx + 3) / 4; L.ty = (L.Ny + 3) / 4; L.tz = (L.Nz + 3) / 4;
  L.hx = Lx / nx; L.hy = Ly / ny; L.hz = Lz / nz;
  L.ne = (int64_t)nx * ny * nz;
  L.ndof = (int64_t)L.Nx * L.Ny * L.Nz;
  // int32 CSR (hypre's HYPRE_Int): nnz and the entry count must fit
  const int64_t nnz = (8LL * nx + 1) * (8LL * ny + 1) * (8LL * nz + 1);
  if (nnz > INT32_MAX || L.ne * 729 > INT32_MAX || L.tz > 65535 || L.ty > 65535) return HM_ERR_UNSUPPORTED;
  hm_lattice* h = new (std::nothrow) hm_lattice;
  if (!h) return HM_ERR_NOMEM;
  h->L = L;
  *out = h;
  return HM_OK;
}

extern "C" int hm_lattice_destroy(hm_lattice* h) {
  delete h;
  return HM_OK;
}

extern "C" int hm_lattice_sizes(const hm_lattice* h, int precision, int64_t* ne, int64_t* ndof,
                                int64_t* nnz, int64_t* quad_bytes) {
  if (!h) return HM_ERR_ARG;
  const hm::Lattice& L = h->L;
  if (ne) *ne = L.ne;
  if (ndof) *ndof = L.ndof;
  if (nnz) *nnz = (8LL * L.nx + 1) * (8LL * L.ny + 1) * (8LL * L.nz + 1);
  if (quad_bytes) *quad_bytes = L.ne * 216 * (precision == HM_FP32 ? 4 : 8);
  return HM_OK;
}

extern "C" int hm_lattice_pattern(const hm_lattice* h, int32_t* indptr, int32_t* indices,
                                  int32_t* slot, void* stream) {
  if (!h || !indptr) return HM_ERR_ARG;
  return hm_launch_pattern(h->L, indptr, indices, slot, stream);
}

extern "C" int hm_lattice_transpose_map(const hm_lattice* h, const int32_t* indptr, int32_t* tpos,
                                        void* stream) {
  if (!h || !indptr || !tpos) return HM_ERR_ARG;
  return hm_launch_tpos(h->L, indptr, tpos, stream);
}

extern "C" int hm_lattice_quadrature(const hm_lattice* h, const double* u, const double* m,
                                     const double* p, int precision, void* quad, uint32_t* status,
                                     void* stream) {
  if (!h || !u || !m || !p || !quad || !status) return HM_ERR_ARG;
  if (precision != HM_FP64 && precision != HM_FP32) return HM_ERR_ARG;
  if (!aligned8(u) || !aligned8(m) || !aligned8(p) || !aligned8(quad)) return HM_ERR_ARG;
  return hm_launch_quad(h->L, u, m, p, precision, quad, status, stream);
}

extern "C" int hm_lattice_quadrature_dir(const hm_lattice* h, const double* u, const double* m,
                                         const double* p, const double* mhat, int precision,
                                         void* quad, uint32_t* status, void* stream) {
  if (!h || !u || !m || !p || !mhat || !quad || !status) return HM_ERR_ARG;
  if (precision != HM_FP64 && precision != HM_FP32) return HM_ERR_ARG;
  if (!aligned8(u) || !aligned8(m) || !aligned8(p) || !aligned8(mhat) || !aligned8(quad))
    return HM_ERR_ARG;
  return hm_launch_quad(h->L, u, m, p, precision, quad, status, stream, mhat);
}

extern "C" int hm_lattice_assemble(const hm_lattice* h, const void* quad, int precision,
                                   const int32_t* indptr, const uint8_t* ess, double f,
                                   double* vA, double* vC, double* vWum, double* vWmm,
                                   double* vs, double* vp, double* va, int zero_ess, void* stream) {
  if (!h || !quad) return HM_ERR_ARG;
  if (precision != HM_FP64 && precision != HM_FP32) return HM_ERR_ARG;
  if ((vA || vC || vWum || vWmm) && !indptr) return HM_ERR_ARG;
  if (!(vA || vC || vWum || vWmm || vs || vp || va)) return HM_OK;
  return hm_launch_assemble(h->L, quad, precision, indptr, ess, f, vA, vC, vWum, vWmm, vs, vp, va,
                            zero_ess, stream);
}

extern "C" int64_t hm_lattice_jacobian_bytes(const hm_lattice* h, int precision) {
  if (!h) return 0;
  return 2 * 27 * h->L.ne * (precision == HM_FP32 ? 4 : 8);
}

extern "C" int hm_lattice_jacobian_prepare(const hm_lattice* h, const void* quad,
                                           int quad_precision, void* jac, int precision,
                                           void* stream) {
  if (!h || !quad || !jac) return HM_ERR_ARG;
  if (precision != HM_FP64 && precision != HM_FP32) return HM_ERR_ARG;
  if (quad_precision != HM_FP64 && quad_precision != HM_FP32) return HM_ERR_ARG;
  return hm_launch_jacobian_prepare(h->L, quad, quad_precision, jac, precision, stream);
}

extern "C" int hm_lattice_apply_A(const hm_lattice* h, void* jac, int precision,
                                  const uint8_t* ess, const double* x, double* y, void* stream) {
  if (!h || !jac || !x || !y || x == y) return HM_ERR_ARG;
  if (precision != HM_FP64 && precision != HM_FP32) return HM_ERR_ARG;
  return hm_launch_apply_A(h->L, jac, precision, ess, x, y, stream);
}

extern "C" int hm_lattice_diag_A(const hm_lattice* h, const void* quad, int precision,
                                 const uint8_t* ess, double* diag, void* stream) {
  if (!h || !quad || !diag) return HM_ERR_ARG;
  if (precision != HM_FP64 && precision != HM_FP32) return HM_ERR_ARG;
  return hm_launch_diag_A(h->L, quad, precision, ess, diag, stream);
}

// the operator of a PCG: a CSR block or the lattice's matrix-free Jacobian
int hm_pcg_operator(int64_t n, const int32_t* indptr, const int32_t* indices, const double* vals,
                    const hm::Lattice* L, const void* quad, int precision, const uint8_t* ess,
                    const double* x, double* y, void* stream) {
  if (L) return hm_launch_apply_A(*L, const_cast<void*>(quad), precision, ess, x, y, stream);
  return hm_csr_spmv(n, indptr, indices, vals, x, y, 1.0, 0.0, stream);
}

extern "C" int hm_pcg_impl(int64_t n, const int32_t* indptr, const int32_t* indices,
                           const double* vals, const hm::Lattice* L, const void* quad,
                           int precision, const uint8_t* ess, const double* diag, const double* b,
                           double* x, double rtol, int maxiter, int check_every, void* work,
                           int* iterations, double* relres, void* stream);

extern "C" int hm_pcg(int64_t n, const int32_t* indptr, const int32_t* indices, const double* vals,
                      const hm_lattice* lattice, const void* quad, int precision,
                      const uint8_t* ess, const double* diag, const double* b, double* x,
                      double rtol, int maxiter, int check_every, void* work, int* iterations,
                      double* relres, void* stream) {
  const hm::Lattice* L = lattice ? &lattice->L : nullptr;
  if (L) {
    if (!quad || n != L->ndof) return HM_ERR_ARG;
  } else if (!indptr || !indices || !vals) {
    return HM_ERR_ARG;
  }
  return hm_pcg_impl(n, indptr, indices, vals, L, quad, precision, ess, diag, b, x, rtol, maxiter,
                     check_every, work, iterations, relres, stream);
}

extern "C" int64_t hm_pcg_mixed_workspace_bytes(int64_t n);
extern "C" int hm_pcg_mixed_impl(const hm::Lattice* L, void* jac64, void* jac32, const uint8_t* ess,
                                 const double* diag, const double* b, double* x, double rtol,
                                 double delta, int max_updates, int maxiter, int check_every,
                                 void* work, int* iterations, int* updates, double* relres,
                                 void* stream);

extern "C" int hm_pcg_mixed(const hm_lattice* lattice, void* jac64, void* jac32, const uint8_t* ess,
                            const double* diag, const double* b, double* x, double rtol,
                            double delta, int max_updates, int maxiter, int check_every,
                            void* work, int* iterations, int* updates, double* relres, void* stream) {
  if (!lattice) return HM_ERR_ARG;
  return hm_pcg_mixed_impl(&lattice->L, jac64, jac32, ess, diag, b, x, rtol, delta, max_updates,
                           maxiter, check_every, work, iterations, updates, relres, stream);
}
