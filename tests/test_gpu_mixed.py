"""Mixed precision: conjugate gradients in FP32 with reliable updates to the FP64 true
residual give the FP64 answers to the stated tolerance.  GPU."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL_SOLVE = 1e-10     # relative difference of the two solves' results (both at rtol 1e-12)
TOL_HESS = 1e-10      # relative difference of the Hessian actions


def _model(n, precision, seed=0):
    from hippymfem_b200 import (BoxMesh, DirichletBC, Model, PDEVariationalProblem,
                                PointwiseStateObservation, Q2Space)
    from hippymfem_b200.synthetic import interior_points, log_conductivity

    mesh = BoxMesh(n)
    V = Q2Space(mesh)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                 matrix_free_solves=True, solver_precision=precision)
    pts = interior_points(64, seed=seed + 10)
    data = np.random.default_rng(seed).standard_normal(64) * 1e-3
    misfit = PointwiseStateObservation(V, pts, data=data, noise_variance=1e-4)
    m = V.project(lambda x: log_conductivity(x, seed=seed, sigma=0.5))
    return mesh, V, prob, Model(prob, None, misfit), m


def test_mixed_forward_solve_matches_fp64(cuda):
    res = {}
    for prec in ("fp64", "mixed"):
        mesh, V, prob, model, m = _model((10, 9, 8), prec)
        u = V.vector()
        prob.solveFwd(u, [u, m, None])
        assert prob.last_solve.converged
        res[prec] = u.cpu().numpy()
    a, b = res["fp64"], res["mixed"]
    assert np.abs(a - b).max() <= TOL_SOLVE * np.abs(a).max()


def test_mixed_hessian_action_matches_fp64(cuda):
    from hippymfem_b200 import ReducedHessian

    out = {}
    for prec in ("fp64", "mixed"):
        mesh, V, prob, model, m = _model((9, 8, 10), prec, seed=1)
        u, p = V.vector(), V.vector()
        x = [u, m, p]
        model.solveFwd(u, x)
        model.solveAdj(p, x)
        model.setPointForHessianEvaluations(x)
        H = ReducedHessian(model)
        v = torch.as_tensor(np.random.default_rng(3).standard_normal(mesh.ndof), device=cuda)
        y = V.vector()
        H.mult(v, y)
        out[prec] = y.cpu().numpy()
    a, b = out["fp64"], out["mixed"]
    assert np.linalg.norm(a - b) <= TOL_HESS * np.linalg.norm(a)


def test_mixed_solver_reports_refinements(cuda):
    from hippymfem_b200 import MatrixFreeJacobian
    from hippymfem_b200.sparse import MixedPCGSolver

    mesh, V, prob, model, m = _model((8, 8, 8), "fp64")
    quad = prob._quadrature([None, m, None], "t")
    A = MatrixFreeJacobian(mesh, quad, prob.bc0.marker)
    s = MixedPCGSolver(A, quad, rel_tolerance=1e-12, reliable_delta=0.1)
    b = torch.as_tensor(np.random.default_rng(5).standard_normal(mesh.ndof), device=cuda)
    prob.bc0.zero(b)
    x = V.vector()
    s.solve(x, b)
    assert s.last.converged and s.last_updates >= 2 and s.last.relres <= 1e-12
    r = V.vector()
    A.mult(x, r)
    assert (r - b).norm().item() <= 1e-11 * b.norm().item()
