/*
 * hippymfem_b200 -- C ABI of the B200 kernels for the Q2 log-conductivity diffusion
 * path:  -div(e^m grad u) = f  on hexahedra, density  e^m grad u . grad p - f p.
 *
 * Conventions
 *   - every function returns an int status: HM_OK (0) or one of HM_ERR_*;
 *   - pointers named d_* are device pointers (any allocator: torch, cudaMalloc, ...);
 *     the library allocates no device memory in any of these calls: scratch is passed
 *     in as a workspace whose size the *_workspace_bytes functions report;
 *   - `stream` is a cudaStream_t passed as void* (NULL: the legacy default stream);
 *     every launch goes to that stream and nothing synchronises unless stated;
 *   - d_status, where taken, is one device uint32 that kernels OR bits into
 *     (HM_STATUS_*); the caller zeroes it and reads it when it wants to;
 *   - slots follow the reference: STATE = 0, PARAMETER = 1, ADJOINT = 2
 *     (hippymfem/modeling/variables.py); a block (i, j) has test slot i as rows.
 *
 * The interfaces each call replaces are named as file:line in the hIPPyMFEM tree.
 */
#ifndef HIPPYMFEM_B200_H
#define HIPPYMFEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; the Python layer maps them onto the reference's exceptions */
#define HM_OK 0
#define HM_ERR_ARG 1         /* ValueError: sizes or arguments do not match        */
#define HM_ERR_CUDA 2        /* a CUDA runtime call failed                          */
#define HM_ERR_NONFINITE 3   /* RuntimeError: non-finite element values            */
#define HM_ERR_NOMEM 4       /* MemoryError: a workspace is too small              */
#define HM_ERR_NOCONV 5      /* an iterative solve did not reach its tolerance     */
#define HM_ERR_RANGE 6       /* an index was out of range                          */
#define HM_ERR_UNSUPPORTED 7 /* a case this build does not cover                   */

/* bits of the device status word */
#define HM_STATUS_NONFINITE 1u
#define HM_STATUS_RANGE 2u
#define HM_STATUS_TIMEOUT 4u  /* a bounded wait in a kernel gave up: its outputs are invalid */

/* arithmetic of the element contractions; CSR values are always FP64 */
#define HM_FP64 0
#define HM_FP32 1

const char* hm_error_string(int code);
int hm_version(void);

/* The library's own device status word on the current device: bits (HM_STATUS_*) that
 * kernels without a d_status argument set -- HM_STATUS_TIMEOUT when the assembly's
 * wait for its staged data gave up.  Synchronises the device; with clear != 0 the word
 * is reset.  No counterpart in the reference (its host kernels cannot time out). */
int hm_device_status(uint32_t* out, int clear);

/* ------------------------------------------------------------------ sparsity pattern
 * hm_pattern_build: CSR graph and entry->slot map of the element-assembly map of one
 * element group, from its two dof tables.  Replaces patternbuild.build_tables
 * (hippymfem/fem/patternbuild.py:209-253) and the sort route of
 * ScatterPattern._build (hippymfem/fem/pattern.py:548-663); identical arrays.
 *   tdofs (ne, ndt), cdofs (ne, ndr): host int64 dof tables, row-major;
 *   entry k = (e*ndt + a)*ndr + b is row tdofs[e,a], column cdofs[e,b];
 *   diag_first: rows lead with their diagonal (a square pattern, as hypre keeps it).
 * Two calls: with indices == NULL and slot == NULL it fills indptr (nrow+1) and *nnz;
 * with both given (indices of capacity >= *nnz, slot of ne*ndt*ndr) it fills all.
 * Host memory, nthreads host threads (0: all). */
int hm_pattern_build(const int64_t* tdofs, const int64_t* cdofs, int64_t ne, int ndt,
                     int ndr, int64_t nrow, int64_t ncol, int diag_first, int nthreads,
                     int32_t* indptr, int32_t* indices, int64_t indices_capacity,
                     int32_t* slot, int64_t* nnz);

/* --------------------------------------------------------------- structured lattice
 * A uniform nx x ny x nz hexahedral mesh of [0,Lx]x[0,Ly]x[0,Lz] with the Q2 dofs
 * numbered lexicographically on the (2nx+1)(2ny+1)(2nz+1) node lattice and elements
 * e = ex + nx (ey + ny ez); element-local dof a = a1 + 3 a2 + 9 a3.  Plays the role of
 * MeshBatches / ElementGroup / SpaceTables (hippymfem/fem/elementbatch.py:159-294,
 * 413-565) for this mesh: geometry and dof tables are arithmetic, nothing is stored.
 * The handle is host memory only; it may be shared by any number of streams. */
typedef struct hm_lattice hm_lattice;

int hm_lattice_create(int nx, int ny, int nz, double Lx, double Ly, double Lz,
                      hm_lattice** out);
int hm_lattice_destroy(hm_lattice* h);
/* ne, ndof, nnz of a Q2 x Q2 block, and the bytes of the quadrature workspace of
 * hm_lattice_quadrature at the given precision */
int hm_lattice_sizes(const hm_lattice* h, int precision, int64_t* ne, int64_t* ndof,
                     int64_t* nnz, int64_t* quad_bytes);

/* The pattern of a Q2 x Q2 block on the lattice, on the device, arithmetically:
 * d_indptr (ndof+1), d_indices (nnz) and, if d_slot is not NULL, the entry->slot map
 * (ne*729) -- the arrays hm_pattern_build / patternbuild.build_tables give for the
 * lattice's dof table.  Replaces get_pattern (hippymfem/fem/pattern.py:1094). */
int hm_lattice_pattern(const hm_lattice* h, int32_t* d_indptr, int32_t* d_indices,
                       int32_t* d_slot, void* stream);

/* Position of the transposed entry: d_tpos[s] = slot of (col, row) for the entry s =
 * (row, col) of the lattice pattern (structurally symmetric).  Lets a block be applied
 * transposed as a gather (hm_csr_spmv_t), the B200 replacement of
 * HypreParMatrix::MultTranspose in apply_ij (modeling/PDEVariationalProblem.py:1629). */
int hm_lattice_transpose_map(const hm_lattice* h, const int32_t* d_indptr,
                             int32_t* d_tpos, void* stream);

/* Quadrature data of the point (u, m, p): per element and Gauss point
 * D = w|J| e^m, E = D grad u, F = D grad p, W = D grad u . grad p, the pointwise
 * second derivatives of the density that the quadrature route of the reference's
 * element kernel forms (hippymfem/fem/kernel.py:1431-1485) after the field
 * evaluation of _eval_field (kernel.py:378-394).  d_quad: quad_bytes of workspace.
 * Non-finite values set HM_STATUS_NONFINITE in *d_status (require_finite_arrays,
 * modeling/PDEVariationalProblem.py:1844-1892). */
int hm_lattice_quadrature(const hm_lattice* h, const double* d_u, const double* d_m,
                          const double* d_p, int precision, void* d_quad,
                          uint32_t* d_status, void* stream);

/* The same quadrature data with D = w|J| e^m mhat: the derivative of the pointwise
 * data along a parameter direction mhat.  Assembled by hm_lattice_assemble with f = 0,
 * its vectors are the second-order products of the point (u, m, p) applied to mhat --
 * ADJOINT: C mhat, STATE: W_um mhat, PARAMETER: W_mm mhat -- without any block formed:
 * the matrix-free element HVP of the reference (hvp_block, hippymfem/fem/kernel.py:
 * 1756-1782, behind apply_ij_at, modeling/PDEVariationalProblem.py:1672). */
int hm_lattice_quadrature_dir(const hm_lattice* h, const double* d_u, const double* d_m,
                              const double* d_p, const double* d_mhat, int precision,
                              void* d_quad, uint32_t* d_status, void* stream);

/* Fused assembly from quadrature data: the CSR values of the blocks whose pointer is
 * not NULL -- A = d2R/dp du (ADJOINT, STATE), C = d2R/dp dm (ADJOINT, PARAMETER),
 * Wum = d2R/du dm (STATE, PARAMETER), Wmm = d2R/dm dm -- in the lattice pattern
 * (d_indptr of hm_lattice_pattern), each value written once, with the folded
 * Dirichlet elimination of hippymfem/fem/bcs.py:13-30 on the nodes d_ess marks
 * (uint8 per dof, NULL: none): A rows and columns zeroed with a unit diagonal, C and
 * Wum rows zeroed, Wmm untouched.  And the assembled vectors whose pointer is not
 * NULL: dR/du (STATE), dR/dm (PARAMETER), dR/dp (ADJOINT, the residual with source f);
 * with zero_ess_vectors the STATE and ADJOINT ones are zeroed on d_ess.  The value
 * arrays and d_quad must be 16-byte aligned (HM_ERR_ARG otherwise; cudaMalloc and
 * torch allocations are).  d_indptr must be the lattice pattern's (required when a
 * block is asked for, else it may be NULL); the kernel compares it with the lattice's
 * row offsets, and a tile that finds another pattern writes nothing and sets
 * HM_STATUS_RANGE in the library's status word (hm_device_status).  For a caller's own
 * dof numbering, assemble in the lattice pattern and map the values with
 * hm_lattice_caller_map + hm_gather_f64.  Replaces setLinearizationPoint's shared pass (modeling/PDEVariationalProblem.py:
 * 1372-1482), _jacobian (:542), _residual (:423), element_matrices_many /
 * element_vectors (hippymfem/fem/kernel.py:2048,2070) and the scatter
 * ScatterPattern.data (hippymfem/fem/pattern.py:749-791). */
int hm_lattice_assemble(const hm_lattice* h, const void* d_quad, int precision,
                        const int32_t* d_indptr, const uint8_t* d_ess, double f,
                        double* d_vals_A, double* d_vals_C, double* d_vals_Wum,
                        double* d_vals_Wmm, double* d_vec_state, double* d_vec_param,
                        double* d_vec_adjoint, int zero_ess_vectors, void* stream);

/* beta * (boundary mass) added in place to a block's values in the lattice pattern
 * (d_vals, nnz of hm_lattice_sizes): beta int_{boundary} phi_n phi_c ds over the whole
 * box boundary, the Robin term the reference's BiLaplacianPrior adds with robin_bc=True
 * (beta = sqrt(gamma delta) / 1.42, modeling/prior.py:941-944). */
int hm_lattice_add_boundary_mass(const hm_lattice* h, double beta, double* d_vals, void* stream);

/* The assembled vectors straight from the fields, without the pointwise-data
 * workspace: dR/du (STATE), dR/dm (PARAMETER), dR/dp (ADJOINT, with the source f) at
 * (u, m, p), or with d_mhat != NULL the second-order products along mhat (D = w|J| e^m
 * mhat, no source: ADJOINT C mhat, STATE W_um mhat, PARAMETER W_mm mhat, rows not
 * eliminated) -- the vectors hm_lattice_quadrature(_dir) + hm_lattice_assemble give,
 * summed in another fixed order (equal to rounding; deterministic).  One pass evaluates
 * the fields at each element's 27 points and contracts its element vectors, a node
 * gather sums them; the replacement of element_vectors + assemble_vector
 * (hippymfem/fem/kernel.py:2070-2078, fem/pattern.py:1186-1233) and of the directional
 * products of apply_ij_at (modeling/PDEVariationalProblem.py:1672).  With
 * zero_ess_vectors the STATE and ADJOINT vectors are zeroed on d_ess.  d_work:
 * hm_lattice_vectors_workspace_bytes(h, number of vectors asked for).  Non-finite
 * pointwise values set HM_STATUS_NONFINITE in *d_status. */
int64_t hm_lattice_vectors_workspace_bytes(const hm_lattice* h, int nvectors);
int hm_lattice_vectors(const hm_lattice* h, const double* d_u, const double* d_m,
                       const double* d_p, const double* d_mhat, double f, const uint8_t* d_ess,
                       double* d_vec_state, double* d_vec_param, double* d_vec_adjoint,
                       int zero_ess_vectors, void* d_work, uint32_t* d_status, void* stream);

/* The vectors of hm_lattice_vectors at (u, m, p) (no mhat, no elimination) for a caller
 * that holds them already at a point (u0, m0, p0): the kept vectors d_kept_* (one for
 * every vector asked for) where (u, m, p) equals (u0, m0, p0) entry for entry, else the
 * vectors computed from the fields -- decided on the device (d_same: one uint32 of
 * scratch, nonzero when the points were equal), so the call never waits for the GPU.
 * The reference's residual and gradient at the linearization point
 * (modeling/PDEVariationalProblem.py:423, :1365) with its shared pass. */
int hm_lattice_vectors_at(const hm_lattice* h, const double* d_u, const double* d_m,
                          const double* d_p, const double* d_u0, const double* d_m0,
                          const double* d_p0, const double* d_kept_state,
                          const double* d_kept_param, const double* d_kept_adjoint, double f,
                          double* d_vec_state, double* d_vec_param, double* d_vec_adjoint,
                          void* d_work, uint32_t* d_same, uint32_t* d_status, void* stream);

/* Matrix-free Q2 operator y = A(D) x with the Jacobian's elimination (x zeroed on
 * d_ess, y = x there): the product apply_ij_at gives for (ADJOINT, STATE)
 * (modeling/PDEVariationalProblem.py:1672).  Its data d_jac (hm_lattice_jacobian_bytes)
 * holds D of the point in a layout the operator streams, filled once per point by
 * hm_lattice_jacobian_prepare from the quadrature data, and the operator's own scratch:
 * two applies with the same d_jac must not overlap on the GPU. */
int64_t hm_lattice_jacobian_bytes(const hm_lattice* h, int precision);
int hm_lattice_jacobian_prepare(const hm_lattice* h, const void* d_quad, int quad_precision,
                                void* d_jac, int precision, void* stream);
int hm_lattice_apply_A(const hm_lattice* h, void* d_jac, int precision, const uint8_t* d_ess,
                       const double* d_x, double* d_y, void* stream);
/* diagonal of A(D) (eliminated rows: 1), for Jacobi preconditioning */
int hm_lattice_diag_A(const hm_lattice* h, const void* d_quad, int precision,
                      const uint8_t* d_ess, double* d_diag, void* stream);

/* The assembled vectors of hm_lattice_assemble (dR/du, dR/dm, dR/dp; any may be NULL,
 * not all) without any device allocation, for callers that cannot allocate when they
 * need them: a process whose GPU memory another runtime's pool already holds (JAX/XLA
 * preallocates most of the device by default; MFEM/hypre may run on an Umpire pool),
 * or a loop that must not pay for an allocation.  This entry point has no counterpart
 * in the reference.  Its scratch (the pointwise data of the elements) is a fixed
 * device array inside the library, so:
 *   - the lattice must have at most 8192 elements (e.g. 20^3); a larger one returns
 *     HM_ERR_NOMEM and launches nothing;
 *   - every GPU that loads the library holds those 14.2 MB until the process exits;
 *   - the first call on a device looks the array's address up for that device (with
 *     the device current): make that first call before any stream capture;
 *   - all calls share the array: calls that overlap on the GPU (other streams, other
 *     threads) race and give wrong results; calls in one stream are ordered and safe.
 *     Nothing has to be cleared between calls: each call overwrites the scratch it
 *     reads.  *d_status is OR-ed as by hm_lattice_quadrature. */
int hm_lattice_residual_noalloc(const hm_lattice* h, const double* d_u, const double* d_m,
                                const double* d_p, double f, const uint8_t* d_ess,
                                double* d_vec_state, double* d_vec_param,
                                double* d_vec_adjoint, int zero_ess_vectors,
                                uint32_t* d_status, void* stream);

/* Constant-exact single-precision blocks: the reference's mixed-precision element
 * matrices with consistent_block (hippymfem/fem/kernel.py:1503-1571).  Each element
 * matrix of the blocks whose pointer is not NULL is contracted in FP32 from the FP64
 * quadrature data d_quad (rounded to FP32) and corrected in FP64 by one rank-one term
 * per side so that its products with the element's constants are the FP64 ones (A and
 * Wmm symmetrized first and symmetric to the bit); the corrected matrices are summed
 * into the lattice pattern entry by entry in a fixed element order, with the folded
 * elimination of hm_lattice_assemble on d_ess.  The assembled blocks are then exact on
 * the constants (A 1 = 0 before elimination) to FP64 rounding.  d_work:
 * hm_lattice_consistent_workspace_bytes (one block's element matrices, FP64). */
int64_t hm_lattice_consistent_workspace_bytes(const hm_lattice* h);
int hm_lattice_assemble_consistent(const hm_lattice* h, const double* d_quad,
                                   const uint8_t* d_ess, double* d_vals_A, double* d_vals_C,
                                   double* d_vals_Wum, double* d_vals_Wmm, void* d_work,
                                   void* stream);

/* ------------------------------------------------------ the caller's dof numbering
 * The lattice numbers its Q2 dofs lexicographically; a caller whose space numbers them
 * otherwise (MFEM's element-to-dof table, hippymfem/fem/elementbatch.py:528-565, with
 * MFEM's element-local order) keeps its numbering:
 *
 * hm_lattice_dof_permutation (host memory): perm[n] = the caller's dof at lattice node
 *   n, from the caller's element dof table cdofs (ne x 27, its elements in the lattice's
 *   element order e = ex + nx (ey + ny ez)) and local[a] = the caller's element-local
 *   slot of lattice-local dof a = a1 + 3 a2 + 9 a3 (NULL: the same order).  HM_ERR_ARG
 *   when the table puts two dofs at one node or is not a bijection onto [0, ndof),
 *   HM_ERR_RANGE for a dof outside it.
 * hm_lattice_caller_map (device): d_src_pos[s] = the lattice-pattern position of entry s
 *   of the caller's pattern (d_cindptr / d_cindices: the arrays hm_pattern_build gives
 *   for the caller's table, the reference's ScatterPattern arrays, fem/pattern.py:
 *   548-663); the block values then reach the caller's CSR (the data array its
 *   HypreParMatrix aliases, fem/parmat.py:106-171) by hm_gather_f64(nnz, d_src_pos,
 *   lattice_vals, caller_vals).  A pattern that does not match sets HM_STATUS_RANGE in
 *   *d_status.
 * hm_gather_f64: d_dst[i] = d_src[d_idx[i]], i < n.  Vectors into the lattice:
 *   idx = perm; back to the caller: idx = perm's inverse. */
int hm_lattice_dof_permutation(const hm_lattice* h, const int64_t* cdofs, const int32_t* local,
                               int32_t* perm);
int hm_lattice_caller_map(const hm_lattice* h, const int32_t* d_perm, const int32_t* d_cindptr,
                          const int32_t* d_cindices, int32_t* d_src_pos, uint32_t* d_status,
                          void* stream);
int hm_gather_f64(int64_t n, const int32_t* d_idx, const double* d_src, double* d_dst,
                  void* stream);

/* The element matrices of a point: for elements e0 .. e0 + count - 1, the (27 x 27)
 * matrices of A, C, Wum and Wmm (each output may be NULL) from the quadrature data of
 * hm_lattice_quadrature, FP64, at d_X[(e - e0) * 729 + local[a] * 27 + local[b]] (row:
 * test dof a, column: trial dof b; local: host array, NULL for the lattice order).
 * Not on the fused path (the assembly never forms them): the export of
 * QuadratureKernel.element_matrices / element_matrices_chunks
 * (hippymfem/fem/kernel.py:1964-2068) for inspection and parity checks. */
int hm_lattice_element_blocks(const hm_lattice* h, const void* d_quad, int precision, int64_t e0,
                              int64_t count, const int32_t* local, double* d_A, double* d_C,
                              double* d_Wum, double* d_Wmm, void* stream);

/* ----------------------------------------------------------------- sparse / solve
 * y = alpha * M x + beta * y for a CSR block (hypre's Mult, apply_ij). */
int hm_csr_spmv(int64_t nrow, const int32_t* d_indptr, const int32_t* d_indices,
                const double* d_vals, const double* d_x, double* d_y, double alpha,
                double beta, void* stream);
/* y = alpha * M^T x + beta * y for a square block with a structurally symmetric
 * pattern, through d_tpos of hm_lattice_transpose_map (MultTranspose, apply_ij). */
int hm_csr_spmv_t(int64_t nrow, const int32_t* d_indptr, const int32_t* d_indices,
                  const int32_t* d_tpos, const double* d_vals, const double* d_x,
                  double* d_y, double alpha, double beta, void* stream);
/* diagonal of a CSR block whose rows lead with their diagonal */
int hm_csr_diag(int64_t nrow, const int32_t* d_indptr, const double* d_vals,
                double* d_diag, void* stream);

/* Jacobi-preconditioned CG in FP64 for A x = b with A a CSR block (d_indptr != NULL)
 * or the lattice's matrix-free operator (lattice != NULL, d_quad its d_jac), stopped at
 * ||r||_2 <= rtol ||b||_2 or maxiter.  The B200 replacement of the incremental
 * solves' hypre PCG (modeling/PDEVariationalProblem.py:1583-1609,
 * algorithms/linSolvers.py:709).  x is the initial guess on entry.  The iteration
 * runs on the device; the host reads the residual norm every check_every
 * iterations (one synchronisation each).  d_work: hm_pcg_workspace_bytes(n). */
int64_t hm_pcg_workspace_bytes(int64_t n);
int hm_pcg(int64_t n, const int32_t* d_indptr, const int32_t* d_indices,
           const double* d_vals, const hm_lattice* lattice, const void* d_quad,
           int precision, const uint8_t* d_ess, const double* d_diag, const double* d_b,
           double* d_x, double rtol, int maxiter, int check_every, void* d_work,
           int* iterations, double* relres, void* stream);

/* Mixed-precision solve of A x = b on the lattice: conjugate gradients with reliable
 * updates.  The Jacobi-preconditioned recurrence runs in FP32 (FP32 operator d_jac32,
 * FP32 vectors, sums accumulated in FP64); whenever its residual has fallen by the
 * factor delta (0 < delta < 1, e.g. 0.1) since the last anchor, or it claims
 * convergence, the correction is added to the FP64 x and the true residual b - A x of
 * the FP64 operator d_jac64 replaces the recurrence's, the search direction kept.
 * Converged when ||b - A x||_2 <= rtol ||b||_2; a true residual that stops halving
 * between anchors (its rounding floor) ends the refinement, converged if within 10 rtol;
 * a refinement that ends short of that (or runs out of anchors) is finished by FP64
 * Jacobi-PCG from the current x, as the reference finishes its refined solves in
 * double (_solve_in_double).
 * x starts from zero.  The mixed-precision route of the reference's solves
 * (_refined_solve, modeling/PDEVariationalProblem.py:1220-1329, a single-precision
 * hypre inside FP64 refinement), here without restarting the Krylov space.
 * *iterations counts FP32 iterations, *updates the anchors.
 * d_work: hm_pcg_mixed_workspace_bytes(n).  HM_ERR_NOCONV after maxiter iterations or
 * max_updates anchors. */
int64_t hm_pcg_mixed_workspace_bytes(int64_t n);
int hm_pcg_mixed(const hm_lattice* lattice, void* d_jac64, void* d_jac32, const uint8_t* d_ess,
                 const double* d_diag, const double* d_b, double* d_x, double rtol,
                 double delta, int max_updates, int maxiter, int check_every, void* d_work,
                 int* iterations, int* updates, double* relres, void* stream);

/* A solve plan: one lattice Jacobian solve on fixed device buffers, for callers that
 * solve again and again with the same operator storage (a request loop keeping one
 * workspace per mesh size).  d_jac32 == NULL: FP64 Jacobi-PCG (d_work of
 * hm_pcg_workspace_bytes); otherwise the mixed-precision solve of hm_pcg_mixed (d_work
 * of hm_pcg_mixed_workspace_bytes).  The caller writes the right-hand side into d_b; a
 * solve starts from x = 0 and leaves the solution in d_x.  The operator data behind
 * d_jac64 / d_jac32 and d_diag may change between solves, the pointers may not.  A full
 * batch of check_every iterations is captured once as a CUDA graph (on the first solve
 * in a stream other than the legacy default stream) and replayed from then on.  A plan
 * is used by one host thread at a time.  The iterative solves of solveFwd/solveAdj/
 * solveIncremental (modeling/PDEVariationalProblem.py:1046-1609) on a resident workspace. */
typedef struct hm_pcg_plan hm_pcg_plan;
int hm_pcg_plan_create(const hm_lattice* lattice, void* d_jac64, void* d_jac32,
                       const uint8_t* d_ess, const double* d_diag, double* d_b, double* d_x,
                       void* d_work, int check_every, hm_pcg_plan** plan);
int hm_pcg_plan_solve(hm_pcg_plan* plan, double rtol, double delta, int max_updates,
                      int maxiter, int* iterations, int* updates, double* relres, void* stream);
int hm_pcg_plan_destroy(hm_pcg_plan* plan);

/* A solve group: FP64 solve plans (Jacobi or multigrid; the same check_every) solved
 * together, for a request loop that has several same-size solves ready at once -- the
 * batched counterpart of one plan's solve.  Each plan's right-hand side is its d_b, its
 * solution lands in its d_x (from zero, as hm_pcg_plan_solve).  Every full batch of
 * iterations of all plans is one CUDA graph (captured on the first group solve in a
 * stream other than the legacy default stream, each plan a branch of its own), and one
 * host synchronisation per batch reads all plans' convergence.  A plan that has
 * converged stops moving (its step lengths are zero), so each solution is bit for bit
 * the one its plan gives solved alone.  iterations / relres: one per plan.  The plans
 * may not be used elsewhere while the group solves; HM_ERR_NOCONV if any plan ends at
 * maxiter. */
typedef struct hm_pcg_group hm_pcg_group;
int hm_pcg_group_create(hm_pcg_plan** plans, int count, hm_pcg_group** group);
int hm_pcg_group_solve(hm_pcg_group* group, double rtol, int maxiter, int* iterations,
                       double* relres, void* stream);
int hm_pcg_group_destroy(hm_pcg_group* group);

/* Geometric multigrid preconditioner for the lattice Jacobian, the structured-lattice
 * counterpart of the BoomerAMG preconditioner of the reference's solves
 * (algorithms/linSolvers.py:243-828): a symmetric V-cycle Q2 -> Q1 on the same elements
 * -> Q1 coarsened 2:1 while every axis stays even and >= 4, Chebyshev-Jacobi smoothing
 * of `degree` before and after, a Chebyshev solve of `coarse_degree` on the coarsest
 * level, trilinear transfers, coarse operators rediscretised with element-mean
 * coefficients.  FP64.  The Dirichlet nodes must be the whole boundary
 * (HM_ERR_UNSUPPORTED otherwise).
 *   hm_mg_create: the hierarchy on d_work (hm_mg_workspace_bytes);
 *   hm_mg_setup: a point's operator -- d_jac64 of hm_lattice_jacobian_prepare (FP64),
 *     its markers and Jacobi diagonal (hm_lattice_diag_A); coarse coefficients,
 *     diagonals and the smoothers' eigenvalue bounds are computed on the device (the
 *     first set-up with a marker array checks it against the boundary: one
 *     synchronisation); again whenever the point changes;
 *   hm_mg_apply: z = V-cycle(r);
 *   hm_pcg_mg: PCG with the V-cycle (x: initial guess; d_work of hm_pcg_workspace_bytes);
 *   hm_pcg_plan_set_mg: a plan's FP64 solves use it (graph-captured with the V-cycle). */
typedef struct hm_mg hm_mg;
int64_t hm_mg_workspace_bytes(const hm_lattice* lattice);
int hm_mg_create(const hm_lattice* lattice, void* d_work, int degree, int coarse_degree,
                 hm_mg** mg);
int hm_mg_setup(hm_mg* mg, void* d_jac64, const uint8_t* d_ess, const double* d_diag,
                void* stream);
int hm_mg_apply(hm_mg* mg, const double* d_r, double* d_z, void* stream);
int hm_mg_levels(const hm_mg* mg);
/* The Q1 levels with at most max_nodes nodes (1000 by default; 0: none) run as one
 * CTA-wide kernel per cycle instead of level by level (the same arithmetic, node for
 * node; one launch instead of ~14 per level).  Set it before a plan's first solve: a
 * plan's captured iteration batches keep the launches they were captured with. */
int hm_mg_set_tail_nodes(hm_mg* mg, int64_t max_nodes);
/* With smoothing degree 1 (the default from a million dofs up) each smoothing step runs
 * as one pass with its level's operator: on level 0 inside the solves (every vector
 * zero on the Dirichlet nodes) the Q2 operator's two kernels carry the Chebyshev update,
 * on the Q1 levels one kernel does both; the arithmetic is the step-by-step one, bit for
 * bit (fused = 1, the default).  fused = 0 launches the steps one by one.  Set it before
 * a plan's first solve, as the tail. */
int hm_mg_set_fused(hm_mg* mg, int fused);
/* The cycle in FP32 (d_work32 of hm_mg_single_workspace_bytes), or in FP64 again
 * (d_work32 = NULL, the default).  The set-up stays FP64; each set-up (and this call,
 * after one, on `stream`) rounds the point's D, the coarse coefficients, the reciprocal
 * diagonals and the coarse inverse to FP32 copies.  r and z of hm_mg_apply stay FP64;
 * with fused degree-1 smoothing inside the solves the level-0 passes read the FP64
 * residual and write the FP64 result themselves.  A preconditioner of the FP64 CG
 * (hm_pcg_mg, plans): the recurrence, its inner products and the stopping test are
 * unchanged, so a solve meets the same tolerance.  With it the CG takes a
 * Polak-Ribiere-type step (beta = r+.(z+ - z) / r.z), the cycle being symmetric only to
 * FP32 rounding, and a solve
 * returns HM_ERR_NOCONV as soon as, past iteration 24, twelve iterations no longer halve
 * the residual: at high contrast (condition numbers near 1e7) FP32 rounding, relative to
 * the smooth part of the cycle's correction, swamps the rest; the caller then solves with
 * the FP64 cycle.  Set it before a plan's first solve, as the tail. */
int64_t hm_mg_single_workspace_bytes(const hm_lattice* lattice);
int hm_mg_set_single(hm_mg* mg, void* d_work32, void* stream);
int hm_mg_destroy(hm_mg* mg);
int hm_pcg_mg(hm_mg* mg, const double* d_b, double* d_x, double rtol, int maxiter,
              int check_every, void* d_work, int* iterations, double* relres, void* stream);
int hm_pcg_plan_set_mg(hm_pcg_plan* plan, hm_mg* mg);

/* The reduced-Hessian action ReducedHessian.mult (hippymfem/modeling/reducedHessian.py:
 * 87-131) at an assembled linearization point, misfit part (the caller adds R x of its
 * prior, as the reference's TrueHessian does unless misfit_only):
 *   uhat = A^{-1} C x,  phat = A^{-T} (W_uu uhat - W_um x),  y = W_mm x + C^T phat - W_mu uhat
 * (GNHessian, y = C^T phat, when d_vals_Wum and d_vals_Wmm are NULL); the right-hand
 * sides zeroed on d_ess as solveIncremental does (modeling/PDEVariationalProblem.py:
 * 1583-1609).  Blocks: CSR values on the lattice pattern (d_indptr, d_indices, d_tpos of
 * hm_lattice_transpose_map).  W_uu = B^T B / noise_variance (misfit.py:102-110) from the
 * observation operator B (nobs x ndof) and its transpose (hm_csr_transpose); nobs = 0:
 * no misfit term.  The two solves run on `plan` (its FP64, multigrid or mixed-precision
 * PCG, from zero, to rtol) through the plan's own right-hand side and solution buffers,
 * which the action overwrites.  d_work: hm_hessian_workspace_bytes(ndof, nobs).
 * iterations (may be NULL): the two solves' iteration counts.  One action at a time per
 * object (it shares the plan). */
typedef struct hm_hessian hm_hessian;
int64_t hm_hessian_workspace_bytes(int64_t ndof, int64_t nobs);
int hm_hessian_create(const hm_lattice* h, const int32_t* d_indptr, const int32_t* d_indices,
                      const int32_t* d_tpos, const double* d_vals_C, const double* d_vals_Wum,
                      const double* d_vals_Wmm, int64_t nobs, const int32_t* d_B_indptr,
                      const int32_t* d_B_indices, const double* d_B_vals,
                      const int32_t* d_Bt_indptr, const int32_t* d_Bt_indices,
                      const double* d_Bt_vals, double noise_variance, const uint8_t* d_ess,
                      hm_pcg_plan* plan, void* d_work, hm_hessian** out);
int hm_hessian_apply(hm_hessian* H, const double* d_x, double* d_y, double rtol, int maxiter,
                     int* iterations, void* stream);
int hm_hessian_destroy(hm_hessian* H);

/* ---------------------------------------------------------------- observations
 * The pointwise observation operator B (npts x ndof) of the lattice's Q2 space: row o
 * holds the 27 basis values at d_points[3 o .. 3 o + 2] in the element containing it,
 * columns ascending; d_indptr[o] = 27 o.  Replaces the reference's
 * PointwiseObservation._build (modeling/pointwiseObservation.py:94-170; MFEM FindPoints
 * and the element shape functions) for a uniform box.  Targets outside the box (beyond
 * 1e-12 of an element) or not finite return HM_ERR_RANGE, as the reference's
 * missing="raise" raises ValueError (:106-112); their rows are zeros.  d_work: at least
 * hm_lattice_observation_workspace_bytes(npts).  Synchronises with the stream to read
 * the range flag. */
int64_t hm_lattice_observation_workspace_bytes(int64_t npts);
int hm_lattice_observation(const hm_lattice* h, const double* d_points, int64_t npts,
                           int32_t* d_indptr, int32_t* d_indices, double* d_vals,
                           void* d_work, void* stream);
/* The transpose of an nrow x ncol CSR matrix with nnz entries, as CSR (ncol + 1 row
 * pointers, rows ordered by source row): B^T for the adjoint source and W_uu of the
 * pointwise misfit (modeling/misfit.py:65-110, PointwiseObservation.multTranspose
 * :210-224).  Deterministic whatever the order of its atomics.  Column indices outside
 * [0, ncol) or row pointers outside [0, nnz] return HM_ERR_RANGE.  d_work: at least
 * hm_csr_transpose_workspace_bytes(ncol).  Synchronises with the stream. */
int64_t hm_csr_transpose_workspace_bytes(int64_t ncol);
int hm_csr_transpose(int64_t nrow, int64_t ncol, int64_t nnz, const int32_t* d_indptr,
                     const int32_t* d_indices, const double* d_vals, int32_t* d_tindptr,
                     int32_t* d_tindices, double* d_tvals, void* d_work, void* stream);

/* deterministic FP64 dot product into *d_out (a fixed-order two-pass reduction) */
int64_t hm_dot_workspace_bytes(int64_t n);
int hm_dot(int64_t n, const double* d_x, const double* d_y, double* d_out, void* d_work,
           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HIPPYMFEM_B200_H */
