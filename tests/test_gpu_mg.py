"""The lattice multigrid preconditioner: a symmetric positive V-cycle, MG-PCG solves that
agree with Jacobi-PCG, few iterations, the Hessian action with either, and the
graph-replayed plan.  GPU."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL_SOLVE = 1e-10     # MG-PCG vs Jacobi-PCG, both at rtol 1e-12
TOL_SYM = 1e-12       # (u, V v) vs (v, V u), relative to |u| |V v|


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


def _interior(mesh, V, bc_mask, seed):
    v = torch.as_tensor(np.random.default_rng(seed).standard_normal(mesh.ndof), device=mesh.device)
    return v.masked_fill_(bc_mask, 0.0)


def test_vcycle_is_symmetric_and_positive(cuda):
    from hippymfem_b200.sparse import Multigrid

    mesh, V, prob, m, A = _jacobian((16, 8, 12), (1.0, 0.6, 0.9))
    mg = Multigrid(mesh).setup(A.jac, A.ess, A._diag)
    assert mg.levels >= 3
    u = _interior(mesh, V, prob.bc0.mask, 1)
    v = _interior(mesh, V, prob.bc0.mask, 2)
    Vu, Vv = V.vector(), V.vector()
    mg.apply(u, Vu)
    mg.apply(v, Vv)
    a, b = float(torch.dot(u, Vv)), float(torch.dot(v, Vu))
    assert abs(a - b) <= TOL_SYM * float(u.norm() * Vv.norm())
    assert float(torch.dot(u, Vu)) > 0 and float(torch.dot(v, Vv)) > 0


@pytest.mark.parametrize("n,L", [((64, 32, 32), (1.0, 0.5, 0.5)), ((16, 8, 12), (1.0, 0.6, 0.9))])
def test_one_cta_tail_matches_the_level_by_level_cycle(cuda, n, L):
    """The small levels run as one CTA-wide kernel: the same cycle as their level-by-level
    launches (the same arithmetic node for node), at every tail size."""
    from hippymfem_b200.sparse import Multigrid

    mesh, V, prob, m, A = _jacobian(n, L)
    r = _interior(mesh, V, prob.bc0.mask, 7)
    mg = Multigrid(mesh).setup(A.jac, A.ess, A._diag)
    ref = mg.set_tail_nodes(0).apply(r, V.vector())
    for nodes in (5000, 40000, 10 ** 9):
        z = mg.set_tail_nodes(nodes).apply(r, V.vector())
        err = float((z - ref).abs().max() / ref.abs().max())
        assert err <= 1e-14, (nodes, err)


@pytest.mark.parametrize("n", [(12, 12, 12), (32, 32, 32)])
def test_mg_pcg_matches_jacobi_pcg_in_few_iterations(cuda, n):
    from hippymfem_b200.sparse import MGPCGSolver, PCGSolver

    mesh, V, prob, m, A = _jacobian(n)
    b = _interior(mesh, V, prob.bc0.mask, 3)
    x1, x2 = V.vector(), V.vector()
    s1 = PCGSolver(A, rel_tolerance=1e-12)
    s1.solve(x1, b)
    s2 = MGPCGSolver(A, rel_tolerance=1e-12)
    s2.solve(x2, b)
    assert s2.last.converged
    assert float((x1 - x2).norm()) <= TOL_SOLVE * float(x1.norm())
    assert s2.last.iterations <= max(40, s1.last.iterations // 5), (s1.last, s2.last)


def test_hessian_action_with_multigrid(cuda):
    from hippymfem_b200 import (DirichletBC, Model, PDEVariationalProblem,
                                PointwiseStateObservation, ReducedHessian)
    from hippymfem_b200.synthetic import interior_points

    out = []
    for pre in ("jacobi", "mg"):
        mesh, V, prob0, m, A = _jacobian((16, 16, 16), seed=2)
        prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                     matrix_free_solves=True, preconditioner=pre)
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
    assert float((out[0] - out[1]).norm()) <= 1e-9 * float(out[0].norm())


def test_plan_with_multigrid_replays_the_same_solve(cuda):
    from hippymfem_b200.sparse import MGPCGSolver, SolvePlan

    mesh, V, prob, m, A = _jacobian((12, 12, 8), seed=4)
    quad = prob._quadrature([None, m, None], "jacobian")
    plan = SolvePlan(mesh, prob.bc0.marker, "fp64", rel_tolerance=1e-10, check_every=4,
                     multigrid=True)
    s = torch.cuda.Stream()
    b = _interior(mesh, V, prob.bc0.mask, 6)
    outs = []
    with torch.cuda.stream(s):
        plan.set_point(quad)
        for _ in range(3):                       # capture, then replays
            x = V.vector()
            plan.solve(x, b)
            outs.append(x.clone())
    s.synchronize()
    ref = V.vector()
    solver = MGPCGSolver(A, rel_tolerance=1e-10, check_every=4)
    solver.solve(ref, b)
    for x in outs:
        assert torch.equal(x, outs[0])
    assert float((outs[0] - ref).norm()) <= 1e-12 * float(ref.norm())
    plan.close()


def test_c_abi_mg_pcg_matches_the_plan(cuda):
    """hm_pcg_mg (initial guess zero) against the plan-based solver."""
    import ctypes

    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.sparse import MGPCGSolver

    mesh, V, prob, m, A = _jacobian((8, 10, 12), seed=5)
    b = _interior(mesh, V, prob.bc0.mask, 7)
    s = MGPCGSolver(A, rel_tolerance=1e-12)
    ref = V.vector()
    s.solve(ref, b)
    work = torch.empty(lib.hm_pcg_workspace_bytes(mesh.ndof) // 8 + 1, dtype=torch.float64,
                       device=cuda)
    x = V.vector()
    it, rr = ctypes.c_int(), ctypes.c_double()
    check(lib.hm_pcg_mg(s.mg._mg, ptr(b), ptr(x), 1e-12, 200, 4, ptr(work), ctypes.byref(it),
                        ctypes.byref(rr), stream_ptr()))
    assert it.value == s.last.iterations
    assert torch.equal(x, ref)


@pytest.mark.parametrize("n,L", [((32, 16, 24), (1.0, 0.5, 0.75)), ((16, 16, 16), (1.0, 1.0, 1.0))])
def test_fused_degree_one_smoothing_is_the_step_by_step_cycle(cuda, n, L):
    """With smoothing degree 1 each step runs fused with its level's operator pass (on
    level 0 inside the solves, where every vector is zero on the Dirichlet nodes): the
    V-cycle and a whole MG-PCG solve are bit for bit those of the step-by-step launches."""
    import ctypes

    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.sparse import Multigrid

    mesh, V, prob, m, A = _jacobian(n, L, seed=3)
    r = _interior(mesh, V, prob.bc0.mask, 8)
    mg = Multigrid(mesh, degree=1).setup(A.jac, A.ess, A._diag)
    zf = mg.set_fused(True).apply(r, V.vector())
    zs = mg.set_fused(False).apply(r, V.vector())
    assert torch.equal(zf, zs)
    work = torch.empty(lib.hm_pcg_workspace_bytes(mesh.ndof) // 8 + 1, dtype=torch.float64,
                       device=cuda)
    out = []
    for fused in (True, False):
        mg.set_fused(fused)
        x = V.vector()
        it, rr = ctypes.c_int(), ctypes.c_double()
        check(lib.hm_pcg_mg(mg._mg, ptr(r), ptr(x), 1e-12, 200, 4, ptr(work), ctypes.byref(it),
                            ctypes.byref(rr), stream_ptr()))
        out.append((x, it.value, rr.value))
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]
    assert torch.equal(out[0][0], out[1][0])
    assert out[0][2] <= 1e-12
