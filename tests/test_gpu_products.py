"""Matrix-free second-order products (directional quadrature data + vector kernels)
against the assembled blocks, and the Hessian action either way.  GPU."""

import numpy as np
import pytest
import torch

from hippymfem_b200.problem import ADJOINT, PARAMETER, STATE

pytestmark = pytest.mark.gpu

TOL = 1e-12          # a product, relative to the assembled block's product (max norm)
TOL_HESS = 1e-10     # Hessian actions, both with solves at rtol 1e-12


def _point(n, seed=0):
    from hippymfem_b200 import BoxMesh, DirichletBC, PDEVariationalProblem, Q2Space

    mesh = BoxMesh(n, (1.0, 0.8, 1.2))
    V = Q2Space(mesh)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                 matrix_free_solves=True)
    rng = np.random.default_rng(seed)
    x = [torch.as_tensor(s * rng.standard_normal(mesh.ndof), device=mesh.device)
         for s in (1.0, 0.3, 1.0)]
    return mesh, V, prob, x, rng


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


def test_directional_products_match_assembled_blocks(cuda):
    mesh, V, prob, x, rng = _point((6, 5, 7))
    prob.setLinearizationPoint(x)                  # assembled C, W_um, W_mm
    for (i, j) in [(ADJOINT, PARAMETER), (PARAMETER, ADJOINT), (STATE, PARAMETER),
                   (PARAMETER, STATE), (PARAMETER, PARAMETER)]:
        d = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
        ref, got = V.vector(), V.vector()
        prob.apply_ij(i, j, d, ref)
        prob.apply_ij_at(i, j, prob._lin_point, d, got)
        assert _rel(got, ref) <= TOL, ((i, j), _rel(got, ref))


def test_matrix_free_hessian_matches_assembled(cuda):
    from hippymfem_b200 import Model, PointwiseStateObservation, ReducedHessian
    from hippymfem_b200.synthetic import interior_points

    out = []
    for mf in (False, True):
        mesh, V, prob, x, rng = _point((8, 7, 6), seed=3)
        pts = interior_points(128, seed=5) * np.array([1.0, 0.8, 1.2])   # inside the box
        misfit = PointwiseStateObservation(V, pts, data=np.zeros(128), noise_variance=1e-4)
        model = Model(prob, None, misfit)
        u, p = V.vector(), V.vector()
        xx = [u, x[PARAMETER], p]
        model.solveFwd(u, xx)
        model.solveAdj(p, xx)
        prob.setLinearizationPoint(xx, matrix_free=mf)
        model.misfit.setLinearizationPoint(xx)
        H = ReducedHessian(model)
        v = torch.as_tensor(np.random.default_rng(9).standard_normal(mesh.ndof), device=cuda)
        y = V.vector()
        H.mult(v, y)
        out.append(y)
    assert float((out[0] - out[1]).norm() / out[0].norm()) <= TOL_HESS
