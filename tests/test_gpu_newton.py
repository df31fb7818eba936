"""The BiLaplacian prior's operators against the oracle and known answers, the full
cost's gradient against central differences, and Newton-CG to convergence.  GPU."""

import math

import numpy as np
import pytest
import torch

from oracle import q2

pytestmark = pytest.mark.gpu

TOL = 1e-12        # assembled operators vs the oracle, relative to the largest entry
TOL_SOLVE = 1e-8   # R^{-1} R v = v through two solves at rtol 1e-12 each
TOL_FD = 1e-5      # full-cost gradient vs central differences (h = 1e-6)


def _prior(n, L=(1.0, 1.0, 1.0), gamma=0.1, delta=2.0):
    from hippymfem_b200 import BiLaplacianPrior, BoxMesh, Q2Space

    mesh = BoxMesh(n, L)
    V = Q2Space(mesh)
    return mesh, V, BiLaplacianPrior(V, gamma, delta)


def test_prior_operators_match_the_oracle_and_known_answers(cuda):
    n, L, gamma, delta = (5, 4, 3), (1.0, 0.7, 1.3), 0.1, 2.0
    mesh, V, prior = _prior(n, L, gamma, delta)
    mo = q2.Lattice(n, L)
    E = mo.edofs()
    pat = q2.build_tables(E, E, mo.ndof, mo.ndof, True)
    x = mesh.node_coords()[:, 0]
    zero = np.zeros(mo.ndof)
    K = q2.scatter(pat[2], q2.element_blocks(mo, E, zero, np.full(mo.ndof, math.log(gamma)),
                                              zero)["A"], pat[3])
    Md = q2.scatter(pat[2], q2.element_blocks(mo, E, x, np.full(mo.ndof, math.log(delta)),
                                               x)["Wmm"], pat[3])
    M1 = q2.scatter(pat[2], q2.element_blocks(mo, E, x, zero, x)["Wmm"], pat[3])
    ap, m = prior.A.values.cpu().numpy(), prior.M.values.cpu().numpy()
    ref = K + Md
    assert np.abs(ap - ref).max() <= TOL * np.abs(ref).max()
    assert np.abs(m - M1).max() <= TOL * np.abs(M1).max()
    vol = L[0] * L[1] * L[2]
    one = torch.ones(mesh.ndof, dtype=torch.float64, device=cuda)
    y = V.vector()
    prior.M.mult(one, y)
    assert abs(float(y.sum()) - vol) <= 1e-12 * vol                     # int 1 = |Omega|
    xt = torch.as_tensor(x, device=cuda)
    prior.A.mult(xt, y)
    want = gamma * vol + delta * vol * L[0] ** 2 / 3.0                  # int gamma|grad x|^2 + delta x^2
    assert abs(float(torch.dot(y, xt)) - want) <= 1e-12 * want
    v = torch.as_tensor(np.random.default_rng(0).standard_normal(mesh.ndof), device=cuda)
    Rv, back = V.vector(), V.vector()
    prior.R.mult(v, Rv)
    prior.Rsolver.solve(back, Rv)
    assert float((back - v).norm()) <= TOL_SOLVE * float(v.norm())


def _inverse_problem(n=10, nobs=64, seed=0):
    from hippymfem_b200 import (DirichletBC, Model, PDEVariationalProblem,
                                PointwiseStateObservation)
    from hippymfem_b200.synthetic import interior_points, log_conductivity

    mesh, V, prior = _prior((n, n, n), gamma=0.05, delta=0.5)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                 matrix_free_solves=True)
    mt = V.project(lambda x: log_conductivity(x, seed=seed + 1, sigma=0.5))
    ut = V.vector()
    prob.solveFwd(ut, [ut, mt, None])
    pts = interior_points(nobs, seed=seed + 2)
    from hippymfem_b200.modeling import observation_operator
    d = observation_operator(mesh, pts) @ ut.cpu().numpy()
    sigma = 0.01 * float(np.abs(d).max())
    d = d + np.random.default_rng(seed + 3).normal(0.0, sigma, d.shape)
    misfit = PointwiseStateObservation(V, pts, data=d, noise_variance=sigma ** 2)
    return mesh, V, prob, Model(prob, prior, misfit)


def test_full_cost_gradient_matches_central_differences(cuda):
    mesh, V, prob, model = _inverse_problem(8)
    rng = np.random.default_rng(4)
    m = torch.as_tensor(0.1 * rng.standard_normal(mesh.ndof), device=cuda)

    def cost(mm):
        u = V.vector()
        x = [u, mm, None]
        model.solveFwd(u, x)
        return model.cost(x)[0]

    u, p = V.vector(), V.vector()
    x = [u, m, p]
    model.solveFwd(u, x)
    model.solveAdj(p, x)
    g = V.vector()
    model.evalGradientParameter(x, g)
    H = 1e-6
    for _ in range(4):
        d = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
        fd = (cost(m + H * d) - cost(m - H * d)) / (2 * H)
        an = float(torch.dot(g, d))
        assert abs(fd - an) <= TOL_FD * abs(an), (fd, an)


def test_newton_cg_converges(cuda):
    from hippymfem_b200.newton import ReducedSpaceNewtonCG, ReducedSpaceNewtonCG_ParameterList

    mesh, V, prob, model = _inverse_problem(10)
    prm = ReducedSpaceNewtonCG_ParameterList()
    prm["print_level"] = -1
    prm["rel_tolerance"] = 1e-6
    prm["max_iter"] = 25
    solver = ReducedSpaceNewtonCG(model, prm)
    x = [V.vector(), V.vector(), V.vector()]
    solver.solve(x)
    assert solver.converged and solver.reason in (1, 3), (solver.reason, solver.history[-1:])
    costs = [h["cost"] for h in solver.history]
    assert all(b <= a * (1 + 1e-12) for a, b in zip(costs, costs[1:]))
    # the gradient at the result (fresh adjoint) is small against the initial one
    g = V.vector()
    model.solveAdj(x[2], x)
    gn = model.evalGradientParameter(x, g)
    assert gn <= 1e-5 * solver.history[0]["gradnorm"]


def test_newton_cg_iterates_match_the_oracle_restatement(cuda):
    """The device Newton-CG against the oracle's restatement of ReducedSpaceNewtonCG._solve_ls
    (NewtonCG.py:262-375) with its Steihaug CG and Armijo step, on the same data, every
    solve direct in the oracle: step by step the same CG counts, step lengths and
    termination reason, and cost, |g| and (g, dm) to 1e-8."""
    from hippymfem_b200.newton import ReducedSpaceNewtonCG, ReducedSpaceNewtonCG_ParameterList
    from hippymfem_b200.synthetic import interior_points

    from oracle import newton as on

    n = 8
    mesh, V, prob, model = _inverse_problem(n)
    prm = ReducedSpaceNewtonCG_ParameterList()
    prm.update({"print_level": -1, "rel_tolerance": 1e-6, "max_iter": 25,
                "cg_incremental_tolerance": 0.0, "cg_preconditioner_tolerance": 0.0})
    solver = ReducedSpaceNewtonCG(model, prm)
    x = [V.vector(), V.vector(), V.vector()]
    solver.solve(x)
    ref = on.InverseProblem(n, interior_points(64, seed=2), model.misfit.d.cpu().numpy(),
                            model.misfit.noise_variance, gamma=0.05, delta=0.5)
    m, hist, reason, converged = on.newton_cg_ls(ref, np.zeros(ref.nd), rel_tolerance=1e-6,
                                                 max_iter=25)
    assert (solver.reason, solver.converged) == (reason, converged)
    assert len(solver.history) == len(hist) >= 3
    for a, b in zip(solver.history, hist):
        assert a["cg_it"] == b["cg_it"] and a["alpha"] == b["alpha"], (a, b)
        for k in ("cost", "misfit", "reg", "gradnorm"):
            assert abs(a[k] - b[k]) <= 1e-8 * abs(b[k]), (k, a, b)
        assert abs(a["gdm"] - b["gdm"]) <= 1e-8 * abs(b["gdm"]) + 1e-14, (a, b)
    assert np.linalg.norm(x[1].cpu().numpy() - m) <= 1e-7 * np.linalg.norm(m)


def test_trust_region_newton_cg_matches_the_oracle_restatement(cuda):
    """The trust-region globalization (NewtonCG.py:377-510, Steihaug CG inside the region
    of the prior's precision) against the oracle's restatement: the same CG counts,
    acceptances and termination; cost, |g| and radius to 1e-8, the reduction ratio to
    1e-5 (a difference of nearly equal costs)."""
    from hippymfem_b200.newton import ReducedSpaceNewtonCG, ReducedSpaceNewtonCG_ParameterList
    from hippymfem_b200.synthetic import interior_points

    from oracle import newton as on

    n = 8
    mesh, V, prob, model = _inverse_problem(n)
    prm = ReducedSpaceNewtonCG_ParameterList()
    prm.update({"print_level": -1, "rel_tolerance": 1e-6, "max_iter": 25, "globalization": "TR"})
    solver = ReducedSpaceNewtonCG(model, prm)
    x = [V.vector(), V.vector(), V.vector()]
    solver.solve(x)
    ref = on.InverseProblem(n, interior_points(64, seed=2), model.misfit.d.cpu().numpy(),
                            model.misfit.noise_variance, gamma=0.05, delta=0.5)
    m, hist, reason, converged = on.newton_cg_tr(ref, np.zeros(ref.nd), rel_tolerance=1e-6,
                                                 max_iter=25)
    assert (solver.reason, solver.converged) == (reason, converged)
    assert len(solver.history) == len(hist) >= 3
    for a, b in zip(solver.history, hist):
        assert a["cg_it"] == b["cg_it"] and a["accepted"] == b["accepted"], (a, b)
        for k in ("cost", "gradnorm", "radius"):
            assert abs(a[k] - b[k]) <= 1e-8 * abs(b[k]), (k, a, b)
        assert abs(a["rho"] - b["rho"]) <= 1e-5, (a, b)
    assert np.linalg.norm(x[1].cpu().numpy() - m) <= 1e-7 * np.linalg.norm(m)
