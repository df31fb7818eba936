"""The multigrid V-cycle run in FP32 (``Multigrid(precision="fp32")``,
``hm_mg_set_single``): the FP64 cycle to single-precision rounding, still symmetric and
positive to that rounding, refreshed at every set-up, and, as the preconditioner of the
FP64 CG, solves that meet the FP64 tolerance and agree with the FP64-cycle solves.
GPU."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL_CYCLE = 2e-5      # |V32 r - V64 r| / |V64 r|: FP32 rounding through one cycle
TOL_SYM32 = 2e-5      # (u, V32 v) vs (v, V32 u), relative to |u| |V32 v|
TOL_SOLVE = 1e-10     # solves to rtol 1e-12 with either cycle


def _jacobian(n, L=(1.0, 1.0, 1.0), seed=0, sigma=0.5):
    from hippymfem_b200 import BoxMesh, DirichletBC, PDEVariationalProblem, Q2Space
    from hippymfem_b200.synthetic import log_conductivity

    mesh = BoxMesh(n, L)
    V = Q2Space(mesh)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                 matrix_free_solves=True)
    m = V.project(lambda x: log_conductivity(x, seed=seed, sigma=sigma))
    A, _ = prob._jacobian([None, m, None])
    return mesh, V, prob, m, A


def _interior(mesh, bc_mask, seed):
    v = torch.as_tensor(np.random.default_rng(seed).standard_normal(mesh.ndof), device=mesh.device)
    return v.masked_fill_(bc_mask, 0.0)


def _rel(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("n,L,degree", [((16, 8, 12), (1.0, 0.6, 0.9), 2),
                                        ((32, 16, 24), (1.0, 0.5, 0.75), 1),
                                        ((24, 24, 24), (1.0, 1.0, 1.0), 1),
                                        ((8, 8, 8), (1.0, 1.0, 1.0), 3)])
def test_single_cycle_is_the_fp64_cycle_to_fp32_rounding(cuda, n, L, degree):
    """Every route through the FP32 cycle (generic level 0, fused level 0 inside a solve,
    the one-CTA tail or level by level) against the FP64 cycle of the same point."""
    import ctypes

    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.sparse import Multigrid

    mesh, V, prob, m, A = _jacobian(n, L, seed=1)
    r = _interior(mesh, prob.bc0.mask, 11)
    mg = Multigrid(mesh, degree=degree).setup(A.jac, A.ess, A._diag)
    ref = mg.apply(r, V.vector())
    mg.set_precision("fp32")
    for tail in (1000, 0):
        mg.set_tail_nodes(tail)
        for fused in (True, False):
            z = mg.set_fused(fused).apply(r, V.vector())
            assert z.dtype == torch.float64
            assert _rel(z, ref) <= TOL_CYCLE, (tail, fused, _rel(z, ref))
            assert float(z[prob.bc0.mask].abs().max()) == 0.0
    mg.set_tail_nodes(1000).set_fused(True)
    # back to FP64: the FP64 cycle, bit for bit
    assert torch.equal(mg.set_precision("fp64").apply(r, V.vector()), ref)
    # inside a solve (every vector zero on the Dirichlet nodes) the fused level-0 passes
    # read the FP64 residual and write the FP64 result: one iteration of hm_pcg_mg from
    # zero gives x = alpha V32(b)
    mg.set_precision("fp32")
    work = torch.empty(lib.hm_pcg_workspace_bytes(mesh.ndof) // 8 + 1, dtype=torch.float64,
                       device=cuda)
    x = V.vector()
    it, rr = ctypes.c_int(), ctypes.c_double()
    rc = lib.hm_pcg_mg(mg._mg, ptr(r), ptr(x), 1e-300, 1, 1, ptr(work), ctypes.byref(it),
                       ctypes.byref(rr), stream_ptr())
    assert rc in (0, 5), rc     # HM_OK or HM_ERR_NOCONV after the one iteration
    assert it.value == 1
    z32 = mg.apply(r, V.vector())
    alpha = float(torch.dot(x, z32) / torch.dot(z32, z32))
    assert _rel(x, alpha * z32) <= TOL_CYCLE


def test_single_cycle_is_symmetric_and_positive_to_fp32_rounding(cuda):
    from hippymfem_b200.sparse import Multigrid

    mesh, V, prob, m, A = _jacobian((16, 8, 12), (1.0, 0.6, 0.9))
    mg = Multigrid(mesh, precision="fp32").setup(A.jac, A.ess, A._diag)
    u = _interior(mesh, prob.bc0.mask, 1)
    v = _interior(mesh, prob.bc0.mask, 2)
    Vu, Vv = mg.apply(u, V.vector()), mg.apply(v, V.vector())
    a, b = float(torch.dot(u, Vv)), float(torch.dot(v, Vu))
    assert abs(a - b) <= TOL_SYM32 * float(u.norm() * Vv.norm())
    assert float(torch.dot(u, Vu)) > 0 and float(torch.dot(v, Vv)) > 0


def test_single_copies_follow_each_setup(cuda):
    """The FP32 level data are formed at every set-up: after moving to another point the
    FP32 cycle follows the new point's FP64 cycle."""
    from hippymfem_b200.sparse import Multigrid

    mesh, V, prob, m, A = _jacobian((16, 16, 16), seed=2)
    r = _interior(mesh, prob.bc0.mask, 5)
    mg = Multigrid(mesh, degree=1, precision="fp32").setup(A.jac, A.ess, A._diag)
    z_a = mg.apply(r, V.vector())
    m2 = V.project(lambda x: 0.8 * np.sin(3 * x[0]) * np.cos(2 * x[1]) + 0.3 * x[2])
    A2, _ = prob._jacobian([None, m2, None])
    mg.setup(A2.jac, A2.ess, A2._diag)
    z_b = mg.apply(r, V.vector())
    ref_b = Multigrid(mesh, degree=1).setup(A2.jac, A2.ess, A2._diag).apply(r, V.vector())
    assert _rel(z_b, ref_b) <= TOL_CYCLE
    assert _rel(z_a, ref_b) > 100 * TOL_CYCLE


@pytest.mark.parametrize("n,sigma", [((12, 12, 12), 0.5), ((32, 32, 32), 0.5),
                                     ((48, 24, 32), 0.5), ((32, 32, 32), 1.0),
                                     ((48, 48, 48), 1.0)])
def test_mg_pcg_with_the_single_cycle_meets_the_fp64_tolerance(cuda, n, sigma):
    """The FP64 CG with the FP32 cycle (a Polak-Ribiere-type step) meets the FP64
    tolerance: with the same iterations where the cycle is strong; where the contrast
    (sigma = 1: e^m over about e^-3..e^3) makes the FP32 cycle's rounding swamp its
    correction, the solve stalls or drifts, and the solver solves again with the FP64
    cycle -- then the FP64-cycle solve, bit for bit."""
    from hippymfem_b200.sparse import MGPCGSolver

    mesh, V, prob, m, A = _jacobian(n, seed=3, sigma=sigma)
    b = _interior(mesh, prob.bc0.mask, 3)
    x64, x32 = V.vector(), V.vector()
    s64 = MGPCGSolver(A, rel_tolerance=1e-12)
    s64.solve(x64, b)
    s32 = MGPCGSolver(A, rel_tolerance=1e-12, mg_precision="fp32")
    s32.solve(x32, b)
    assert s32.last.converged and s32.last.relres <= 1e-12
    assert _rel(x32, x64) <= TOL_SOLVE
    if sigma < 1.0:
        assert s32.fallbacks == 0
        assert s32.last.iterations <= s64.last.iterations + 2, (s64.last, s32.last)
    if s32.fallbacks:
        assert s32.mg.precision == "fp64"
        assert s32.last.iterations == s64.last.iterations and torch.equal(x32, x64)
    else:
        # the FP64 true residual of the FP32-cycle solve
        y = V.vector()
        A.mult(x32, y)
        assert float((b - y).norm()) <= 10e-12 * float(b.norm())
    if n == (48, 48, 48):
        assert s32.fallbacks == 1           # this contrast is beyond the FP32 cycle


def test_stalled_single_cycle_solve_stops_early(cuda):
    """The C ABI solve with the FP32 cycle stops with HM_ERR_NOCONV once twelve
    iterations no longer halve its residual, long before maxiter."""
    import ctypes

    from hippymfem_b200._lib import HM_ERR_NOCONV, HM_OK, lib, ptr, stream_ptr
    from hippymfem_b200.sparse import Multigrid

    mesh, V, prob, m, A = _jacobian((48, 48, 48), seed=3, sigma=1.0)
    b = _interior(mesh, prob.bc0.mask, 3)
    work = torch.empty(lib.hm_pcg_workspace_bytes(mesh.ndof) // 8 + 1, dtype=torch.float64,
                       device=cuda)
    mg = Multigrid(mesh, precision="fp32").setup(A.jac, A.ess, A._diag)
    x = V.vector()
    it, rr = ctypes.c_int(), ctypes.c_double()
    rc = lib.hm_pcg_mg(mg._mg, ptr(b), ptr(x), 1e-12, 2000, 4, ptr(work), ctypes.byref(it),
                       ctypes.byref(rr), stream_ptr())
    assert rc == HM_ERR_NOCONV and it.value < 1000, (rc, it.value, rr.value)
    # the FP64 cycle carries the same solve
    mg.set_precision("fp64")
    rc = lib.hm_pcg_mg(mg._mg, ptr(b), ptr(V.vector()), 1e-12, 2000, 4, ptr(work),
                       ctypes.byref(it), ctypes.byref(rr), stream_ptr())
    assert rc == HM_OK and rr.value <= 1e-12


def test_hessian_action_with_the_single_cycle(cuda):
    """``solver_precision="mixed"`` with ``preconditioner="mg"``: the FP64 CG with the FP32
    cycle, the same Hessian action as the FP64 cycle's."""
    from hippymfem_b200 import (DirichletBC, Model, PDEVariationalProblem,
                                PointwiseStateObservation, ReducedHessian)
    from hippymfem_b200.synthetic import interior_points

    out = []
    for precision in ("fp64", "mixed"):
        mesh, V, prob0, m, A = _jacobian((16, 16, 16), seed=2)
        prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                     preconditioner="mg", solver_precision=precision)
        pts = interior_points(128, seed=4)
        misfit = PointwiseStateObservation(V, pts, data=np.zeros(128), noise_variance=1e-4)
        model = Model(prob, None, misfit)
        u, p = V.vector(), V.vector()
        x = [u, m, p]
        model.solveFwd(u, x)
        model.solveAdj(p, x)
        model.setPointForHessianEvaluations(x)
        H = ReducedHessian(model)
        v = torch.as_tensor(np.random.default_rng(5).standard_normal(mesh.ndof), device=cuda)
        y = V.vector()
        H.mult(v, y)
        out.append(y)
        assert prob.solver.mg.precision == ("fp32" if precision == "mixed" else "fp64")
    assert _rel(out[1], out[0]) <= 1e-9
