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


def _pattern_values(pat, mat):
    """The entries of a scipy matrix at the positions of a CSR pattern."""
    ip, ind = pat[0].astype(np.int64), pat[1].astype(np.int64)
    rows = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    return np.asarray(mat[rows, ind]).ravel()


def test_prior_robin_term_and_diagonal_theta(cuda):
    """robin_bc adds beta times the boundary mass (beta = sqrt(gamma delta) / 1.42; the
    oracle integrates it face element by face element); a diagonal Theta scales each
    direction's stiffness (against the oracle on the rescaled lattice and the known
    answers int gamma theta_d (d_d x_d)^2 = gamma theta_d |Omega|); a scalar Theta is
    gamma Theta; an off-diagonal Theta is refused."""
    from hippymfem_b200 import BiLaplacianPrior, BoxMesh, Q2Space

    n, L, gamma, delta = (4, 3, 5), (1.0, 0.7, 1.3), 0.1, 2.0
    mesh = BoxMesh(n, L)
    V = Q2Space(mesh)
    mo = q2.Lattice(n, L)
    E = mo.edofs()
    pat = q2.build_tables(E, E, mo.ndof, mo.ndof, True)
    zero = np.zeros(mo.ndof)
    x = mesh.node_coords()
    Md = q2.scatter(pat[2], q2.element_blocks(mo, E, x[:, 0], np.full(mo.ndof, math.log(delta)),
                                               x[:, 0])["Wmm"], pat[3])
    base = BiLaplacianPrior(V, gamma, delta).A.values.cpu().numpy()
    rob = BiLaplacianPrior(V, gamma, delta, robin_bc=True).A.values.cpu().numpy()
    beta = math.sqrt(gamma * delta) / 1.42
    want = base + beta * _pattern_values(pat, q2.boundary_mass(mo))
    assert np.abs(rob - want).max() <= TOL * np.abs(want).max()
    area = 2 * (L[0] * L[1] + L[1] * L[2] + L[0] * L[2])
    assert abs(np.sum(rob - base) - beta * area) <= 1e-12 * beta * area      # 1^T B 1 = |dOmega|

    theta = np.array([2.0, 0.5, 3.0])
    an = BiLaplacianPrior(V, gamma, delta, Theta=np.diag(theta)).A.values.cpu().numpy()
    K = an - Md
    ms = q2.Lattice(n, tuple(Ld / math.sqrt(t) for Ld, t in zip(L, theta)))
    Kref = q2.scatter(pat[2], q2.element_blocks(
        ms, E, zero, np.full(mo.ndof, math.log(gamma) + 0.5 * np.log(theta).sum()), zero)["A"],
        pat[3])
    assert np.abs(K - Kref).max() <= TOL * np.abs(Kref).max()
    Km = q2.csr(pat, K, (mo.ndof, mo.ndof))
    vol = L[0] * L[1] * L[2]
    for d in range(3):
        got = x[:, d] @ (Km @ x[:, d])
        assert abs(got - gamma * theta[d] * vol) <= 1e-12 * gamma * theta[d] * vol, d
    assert abs(x[:, 0] @ (Km @ x[:, 1])) <= 1e-12 * gamma * vol
    assert np.array_equal(an, BiLaplacianPrior(V, gamma, delta, Theta=theta).A.values.cpu().numpy())
    iso = BiLaplacianPrior(V, gamma, delta, Theta=2.0).A.values.cpu().numpy()
    g2 = BiLaplacianPrior(V, 2.0 * gamma, delta).A.values.cpu().numpy()
    assert np.abs(iso - g2).max() <= TOL * np.abs(g2).max()
    with pytest.raises(NotImplementedError):
        BiLaplacianPrior(V, gamma, delta, Theta=np.array([[1.0, 0.2, 0], [0.2, 1, 0], [0, 0, 1]]))


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
