"""The autograd wrappers of the derivative kernels against central finite differences
(h = 1e-6, 16 seeded random directions, as the reference's test_kernels.py:377-451 and
modelVerify.py:34-131 check theirs).  GPU."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

H = 1e-6
NDIR = 16
TOL_RESIDUAL = 1e-6   # directional derivative of <w, r(u, m)>, relative
TOL_REDUCED = 1e-5    # through two solves at rtol 1e-12: FD error ~ 1e-12 / h
TOL_HESSIAN = 1e-4    # H v against the central difference of the gradient, relative norm


def _setup(n, lines=False, seed=0):
    from hippymfem_b200 import (BoxMesh, DirichletBC, Model, PDEVariationalProblem,
                                PointwiseStateObservation, Q2Space)
    from hippymfem_b200.synthetic import interior_points, log_conductivity, vertical_lines

    mesh = BoxMesh(n)
    V = Q2Space(mesh)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                 matrix_free_solves=True)
    pts = vertical_lines(60, 64, seed=3) if lines else interior_points(256, seed=seed + 10)
    m = V.project(lambda x: log_conductivity(x, seed=seed, sigma=0.3))
    # data from a second field, with 1% noise
    u_true = V.vector()
    mt = V.project(lambda x: log_conductivity(x, seed=seed + 1, sigma=0.3))
    prob.solveFwd(u_true, [u_true, mt, None])
    from hippymfem_b200.modeling import observation_operator
    d = observation_operator(mesh, pts) @ u_true.cpu().numpy()
    sigma = 0.01 * float(np.abs(d).max())
    d = d + np.random.default_rng(seed + 20).normal(0.0, sigma, d.shape)
    misfit = PointwiseStateObservation(V, pts, data=d, noise_variance=sigma ** 2)
    prob._jac_cache = None
    return mesh, V, prob, misfit, Model(prob, None, misfit), m


def _directions(nd, k, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(nd) for _ in range(k)]


def test_residual_vjp_matches_central_differences(cuda):
    from hippymfem_b200.autograd import Residual

    mesh, V, prob, misfit, model, m = _setup((6, 5, 7))
    rng = np.random.default_rng(1)
    u = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda).requires_grad_(True)
    m = m.clone().requires_grad_(True)
    w = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
    L = torch.dot(w, Residual.apply(u, m, prob))
    gu, gm = torch.autograd.grad(L, (u, m))
    for du, dm in zip(_directions(mesh.ndof, NDIR, 2), _directions(mesh.ndof, NDIR, 3)):
        du = torch.as_tensor(du, device=cuda)
        dm = torch.as_tensor(dm, device=cuda)
        with torch.no_grad():
            lp = torch.dot(w, Residual.apply(u + H * du, m + H * dm, prob))
            lm = torch.dot(w, Residual.apply(u - H * du, m - H * dm, prob))
        fd = float((lp - lm) / (2 * H))
        an = float(torch.dot(gu, du) + torch.dot(gm, dm))
        assert abs(fd - an) <= TOL_RESIDUAL * max(abs(an), 1e-30), (fd, an)


@pytest.mark.parametrize("n,lines", [((12, 12, 12), False), ((32, 32, 32), True)])
def test_reduced_gradient_matches_central_differences(cuda, n, lines):
    """The misfit gradient through ForwardSolve + Observe (the 32^3 case: 60 vertical
    lines x 64 depths, 1% noise)."""
    from hippymfem_b200.autograd import reduced_misfit

    mesh, V, prob, misfit, model, m = _setup(n, lines)
    m = m.clone().requires_grad_(True)
    J = reduced_misfit(m, prob, misfit)
    (g,) = torch.autograd.grad(J, m)
    for d in _directions(mesh.ndof, NDIR, 5):
        d = torch.as_tensor(d, device=cuda)
        with torch.no_grad():
            jp = reduced_misfit(m + H * d, prob, misfit)
            jm = reduced_misfit(m - H * d, prob, misfit)
        fd = float((jp - jm) / (2 * H))
        an = float(torch.dot(g, d))
        assert abs(fd - an) <= TOL_REDUCED * max(abs(an), 1e-30), (fd, an)


def test_recompute_gives_the_stored_gradient(cuda):
    from hippymfem_b200.autograd import reduced_misfit

    mesh, V, prob, misfit, model, m = _setup((10, 9, 8))
    m1 = m.clone().requires_grad_(True)
    (g1,) = torch.autograd.grad(reduced_misfit(m1, prob, misfit), m1)
    m2 = m.clone().requires_grad_(True)
    (g2,) = torch.autograd.grad(reduced_misfit(m2, prob, misfit, recompute=True), m2)
    assert torch.equal(g1, g2)


def test_gradient_vjp_is_the_hessian_action(cuda):
    """ReducedGradient's backward (the Hessian action) against the central difference of
    the gradient, and the gradient itself against the reduced-misfit route."""
    from hippymfem_b200.autograd import ReducedGradient, reduced_misfit

    mesh, V, prob, misfit, model, m = _setup((10, 10, 10))
    mm = m.clone().requires_grad_(True)
    g = ReducedGradient.apply(mm, model)
    m2 = m.clone().requires_grad_(True)
    (g2,) = torch.autograd.grad(reduced_misfit(m2, prob, misfit), m2)
    assert float((g - g2).detach().norm()) <= 1e-9 * float(g2.norm())
    for d in _directions(mesh.ndof, 4, 7):
        v = torch.as_tensor(d, device=cuda)
        (hv,) = torch.autograd.grad(g, mm, v, retain_graph=True)
        with torch.no_grad():
            gp = ReducedGradient.apply(m + H * v, model)
            gm = ReducedGradient.apply(m - H * v, model)
        fd = (gp - gm) / (2 * H)
        assert float((fd - hv).norm()) <= TOL_HESSIAN * float(hv.norm())
