// Launchers shared between the translation units of libhippymfem_b200.
#pragma once

#include <cstdint>

#include "../../include/hippymfem_b200.h"

namespace hm {
struct Lattice;
}

// the geometry behind a lattice handle
const hm::Lattice* hm_lattice_geometry(const hm_lattice* h);

int hm_launch_pattern(const hm::Lattice& L, int32_t* indptr, int32_t* indices, int32_t* slot,
                      void* stream);
int hm_launch_tpos(const hm::Lattice& L, const int32_t* indptr, int32_t* tpos, void* stream);
int hm_launch_quad(const hm::Lattice& L, const double* u, const double* m, const double* p,
                   int precision, void* quad, uint32_t* status, void* stream,
                   const double* mhat = nullptr);
int hm_launch_assemble(const hm::Lattice& L, const void* quad, int precision,
                       const int32_t* indptr, const uint8_t* ess, double f, double* vA,
                       double* vC, double* vWum, double* vWmm, double* vs, double* vp,
                       double* va, int zero_ess, void* stream);
int hm_launch_jacobian_prepare(const hm::Lattice& L, const void* quad, int quad_precision,
                               void* jac, int precision, void* stream);
int hm_launch_apply_A(const hm::Lattice& L, void* jac, int precision, const uint8_t* ess,
                      const double* x, double* y, void* stream);
int hm_launch_diag_A(const hm::Lattice& L, const void* quad, int precision,
                     const uint8_t* ess, double* diag, void* stream);
int hm_launch_apply_A_dot(const hm::Lattice& L, void* jac, int precision, const uint8_t* ess,
                          const double* x, double* y, double* part, void* stream,
                          double* sc = nullptr, unsigned* counter = nullptr);
int64_t hm_apply_dot_parts(const hm::Lattice& L);
int hm_launch_apply_A32_dot(const hm::Lattice& L, void* jac32, const uint8_t* ess, const float* x,
                            float* y, double* part, void* stream, double* sc = nullptr,
                            unsigned* counter = nullptr);
// y = A x for an x that is zero on the Dirichlet nodes (FP64 operator)
int hm_launch_apply_A_clean(const hm::Lattice& L, void* jac, const uint8_t* ess, const double* x,
                            double* y, void* stream);
// x = b on the Dirichlet nodes
int hm_launch_ess_take_b(const hm::Lattice& L, const uint8_t* ess, const double* b, double* x,
                         void* stream);
// the right-hand side and solution buffers a solve plan was created with
int hm_plan_buffers(const hm_pcg_plan* plan, double** b, double** x);
// one Chebyshev-Jacobi step of degree 1 of the multigrid smoother on the lattice
// operator, fused with the operator pass: from zero (x = b idiag / theta, r = b - A x)
// or from x (x += (b - A x) idiag / theta); theta = cheb[0], idiag the reciprocal of the
// Jacobi diagonal
int hm_launch_cheb1_from_zero(const hm::Lattice& L, void* jac, const uint8_t* ess, const double* b,
                              const double* idiag, const double* cheb, double* x, double* r,
                              void* stream);
int hm_launch_cheb1_from_x(const hm::Lattice& L, void* jac, const uint8_t* ess, const double* b,
                           const double* idiag, const double* cheb, double* x, void* stream);
// the FP32 operator (jac32: the points' D in FP32, then the FP32 element results) on
// FP32 vectors; clean: x zero on the Dirichlet nodes
int hm_launch_apply_A32(const hm::Lattice& L, void* jac32, const uint8_t* ess, const float* x,
                        float* y, bool clean, void* stream);
// the two fused smoothing steps above with the FP32 operator: from zero, b FP64 in, x and
// r FP32 out; from x (FP32), the result z = x + (b - A x) idiag / theta written in FP64
int hm_launch_cheb1_from_zero32(const hm::Lattice& L, void* jac32, const uint8_t* ess,
                                const double* b, const double* idiag, const double* cheb,
                                float* x, float* r, void* stream);
int hm_launch_cheb1_from_x32(const hm::Lattice& L, void* jac32, const uint8_t* ess, const double* b,
                             const double* idiag, const double* cheb, const float* x, double* z,
                             void* stream);
