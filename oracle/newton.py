"""CPU FP64 restatement of the reference's inexact Newton-CG -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may use this module, as the checker of the device Newton-CG
(``hippymfem_b200.newton``); the product never does.

What it follows (paths relative to the hIPPyMFEM tree):

* :func:`newton_cg_ls` -- ``ReducedSpaceNewtonCG._solve_ls``
  (``hippymfem/algorithms/NewtonCG.py:262-375``): Gauss-Newton for the first ``GN_iter``
  steps, Eisenstat-Walker ``tolcg = min(cg_coarse_tolerance, sqrt(|g| / |g_0|))``,
  the termination codes 1 (gradient), 2 (backtracking), 3 (``(g, dm)``), 4 (forward
  solve failed), the history of each step (``cg_it``, cost, misfit, reg, ``(g, dm)``,
  ``|g|``, ``alpha``, ``tolcg``) -- with the reference's solve tolerances of the CG's
  operator and preconditioner left at their own (``cg_incremental_tolerance = 0``,
  ``cg_preconditioner_tolerance = 0``: here every solve is direct);
* :func:`steihaug_cg` -- ``CGSolverSteihaug._solve``
  (``hippymfem/algorithms/cgsolverSteihaug.py:218-344``) with the explicit
  reorthogonalization against the earlier residuals, and with or without the trust
  region of ``set_TR`` / ``update_x_with_TR`` / ``_tau_to_boundary`` /
  ``_negative_curvature`` (``:117-197``);
* :func:`newton_cg_tr` -- ``ReducedSpaceNewtonCG._solve_tr`` (``NewtonCG.py:377-493``):
  the radius from the first step, the ratio test with ``eta``, the radius updates;
* :func:`armijo` -- ``armijo_backtrack`` (``hippymfem/algorithms/linesearch.py:12-62``);
* :class:`InverseProblem` -- the model the algorithm drives, for the Q2 log-conductivity
  problem on the lattice: the forward and adjoint solves
  (``modeling/PDEVariationalProblem.py:1046-1171``), the cost ``1/(2 sigma^2)|Bu - d|^2 +
  1/2 m^T R m`` (``modeling/misfit.py:65-110``, ``modeling/prior.py:575-586``), the
  gradient ``dR/dm + R m`` and its norm ``sqrt(g^T M^{-1} g)`` (``modeling/model.py:
  219-236``), the reduced Hessian (``modeling/reducedHessian.py:102-131``) and the
  BiLaplacian prior ``R = A M^{-1} A``, ``A = gamma K + delta M`` with
  ``R^{-1} = A^{-1} M A^{-1}`` (``modeling/prior.py:319-373, 894-952``) -- every block
  from :mod:`oracle.q2`'s closed form, every solve by a sparse LU factorization.
"""

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

from . import q2


class InverseProblem:
    def __init__(self, n, pts, data, noise_variance, gamma, delta, f=1.0):
        self.mesh = q2.Lattice(n)
        self.E = self.mesh.edofs()
        nd = self.mesh.ndof
        self.nd = nd
        self.f = f
        self.pat = q2.build_tables(self.E, self.E, nd, nd, True)
        self.ess = self.mesh.boundary_dofs()
        self.mask = np.zeros(nd, bool)
        self.mask[self.ess] = True
        self.B = sp.csr_matrix(q2.observation_matrix(self.mesh, pts))
        self.d = np.asarray(data, dtype=np.float64)
        self.nv = float(noise_variance)
        zero = np.zeros(nd)
        x = self.mesh.node_coords()[:, 0]

        def blk(name, u, logc, p):
            b = q2.element_blocks(self.mesh, self.E, u, np.full(nd, logc), p, (name,))[name]
            return q2.csr(self.pat, q2.scatter(self.pat[2], b, self.pat[3]), (nd, nd))

        self.Ap = (blk("A", zero, math.log(gamma), zero) + blk("Wmm", x, math.log(delta), x)).tocsc()
        self.M = blk("Wmm", x, 0.0, x).tocsc()
        self.Ap_lu = spl.splu(self.Ap)
        self.M_lu = spl.splu(self.M)
        self._point = None

    # ------------------------------------------------------------------ prior
    def R(self, v):
        return self.Ap @ self.M_lu.solve(self.Ap @ v)

    def Rinv(self, v):
        return self.Ap_lu.solve(self.M @ self.Ap_lu.solve(v))

    # ----------------------------------------------------------------- blocks
    def _blocks(self, u, m, p, names):
        blk = q2.element_blocks(self.mesh, self.E, u, m, p, names)
        return {k: q2.csr(self.pat, q2.assemble_block(k, self.pat, blk[k], self.mask),
                          (self.nd, self.nd)) for k in blk}

    def _jacobian_lu(self, m):
        A = self._blocks(np.zeros(self.nd), m, np.zeros(self.nd), ("A",))["A"]
        return spl.splu(A.tocsc())

    def solve_fwd(self, m):
        """One Newton step from u = 0 (the problem is linear in u)."""
        lu = self._jacobian_lu(m)
        zero = np.zeros(self.nd)
        ev = q2.element_vectors(self.mesh, self.E, zero, m, zero, self.f)
        r = q2.assemble_vector(self.E, ev[q2.ADJOINT], self.nd, self.ess)
        return lu.solve(-r)

    def cost(self, u, m):
        r = self.B @ u - self.d
        misfit = 0.5 / self.nv * float(r @ r)
        reg = 0.5 * float(self.R(m) @ m)
        return [misfit + reg, reg, misfit]

    def solve_adj(self, u, m):
        lu = self._jacobian_lu(m)
        rhs = -(self.B.T @ (self.B @ u - self.d)) / self.nv
        rhs[self.ess] = 0.0
        return lu.solve(rhs)

    def gradient(self, u, m, p):
        ev = q2.element_vectors(self.mesh, self.E, u, m, p, self.f)
        g = q2.assemble_vector(self.E, ev[q2.PARAMETER], self.nd) + self.R(m)
        return g, math.sqrt(max(float(g @ self.M_lu.solve(g)), 0.0))

    def set_point(self, u, m, p, gauss_newton):
        names = ("A", "C") if gauss_newton else ("A", "C", "Wum", "Wmm")
        bl = self._blocks(u, m, p, names)
        self._point = (bl, spl.splu(bl["A"].tocsc()), gauss_newton)

    def hessian(self, x):
        bl, lu, gn = self._point
        Wuu = (self.B.T @ self.B) / self.nv
        rhs = bl["C"] @ x
        rhs[self.ess] = 0.0
        uhat = lu.solve(rhs)
        rhs = Wuu @ uhat - (0.0 if gn else bl["Wum"] @ x)
        rhs[self.ess] = 0.0
        phat = lu.solve(rhs)          # A^T = A
        y = bl["C"].T @ phat
        if not gn:
            y = y + bl["Wmm"] @ x - bl["Wum"].T @ uhat
        return y + self.R(x)


def steihaug_cg(A, Binv, b, rel_tolerance, abs_tolerance=1e-12, max_iter=1000,
                reorthogonalize=True, tr=None):
    """Returns ``(x, iterations, actions, reason)``; ``actions`` counts ``A`` products.
    ``tr = (radius, B)``: the steps stay in ``x^T B x <= radius^2``."""
    actions = 0
    x = np.zeros_like(b)
    if tr is not None:
        R2, Bop = tr[0] ** 2, tr[1]

    def bdot(u, v):
        return float(Bop(u) @ v)

    def to_boundary(x, d, rd, dAd):
        a, b_half = bdot(d, d), bdot(d, x)
        c = bdot(x, x) - R2
        disc = np.sqrt(max(b_half * b_half - a * c, 0.0))
        best = None
        for tau in ((-b_half + disc) / a, (-b_half - disc) / a):
            mv = -tau * rd + 0.5 * tau * tau * dAd
            if best is None or mv < best[0]:
                best = (mv, tau)
        return best[1]
    r = b.copy()
    z = Binv(r)
    d = z.copy()
    nom0 = nom = float(d @ r)
    basis = [(r.copy(), z.copy(), nom)] if reorthogonalize else None
    r0 = max(nom * rel_tolerance ** 2, abs_tolerance ** 2)
    if nom <= r0:
        return x, 0, actions, 1
    Ad = A(d)
    actions += 1
    den = float(Ad @ d)
    if den <= 0.0:
        tau = to_boundary(x, d, float(r @ d), den) if tr is not None else 1.0
        return x + tau * d, 0, actions, 2
    it = 1
    while True:
        alpha = nom / den
        xn = x + alpha * d
        if tr is not None and bdot(xn, xn) >= R2:
            a_tau = alpha * alpha * bdot(d, d)
            b_half = alpha * bdot(d, x)
            c_tau = bdot(x, x) - R2
            tau = (-b_half + np.sqrt(max(b_half * b_half - a_tau * c_tau, 0.0))) / a_tau
            return x + (tau * alpha) * d, it, actions, 3
        x = xn
        r = r - alpha * Ad
        if basis is not None:
            for rj, zj, rho in basis:
                r = r - (float(r @ zj) / rho) * rj
        z = Binv(r)
        betanom = float(r @ z)
        if betanom < r0:
            return x, it, actions, 1
        it += 1
        if it > max_iter:
            return x, it, actions, 0
        if basis is not None:
            basis.append((r.copy(), z.copy(), betanom))
        d = (betanom / nom) * d + z
        Ad = A(d)
        actions += 1
        den = float(d @ Ad)
        if den <= 0.0:
            if tr is not None:
                x = x + to_boundary(x, d, float(r @ d), den) * d
            return x, it, actions, 2
        nom = betanom
    del nom0


def armijo(prob, u, m, mhat, mg_mhat, cost_old, c_armijo, max_backtracking, gdm_tolerance):
    alpha, n_back, cost = 1.0, 0, None
    while n_back < max_backtracking:
        m_star = m + alpha * mhat
        u_star = prob.solve_fwd(m_star)
        cost = prob.cost(u_star, m_star)
        if cost[0] < cost_old + alpha * c_armijo * mg_mhat or -mg_mhat <= gdm_tolerance:
            return True, alpha, n_back, cost, u_star, m_star
        n_back += 1
        alpha *= 0.5
    return False, alpha, n_back, cost, u, m


def newton_cg_ls(prob, m0, rel_tolerance=1e-6, abs_tolerance=1e-12, gdm_tolerance=1e-18,
                 max_iter=20, GN_iter=5, cg_coarse_tolerance=0.5, cg_max_iter=100,
                 cg_reorthogonalize=True, c_armijo=1e-4, max_backtracking_iter=10):
    """Returns ``(m, history, reason, converged)``."""
    m = np.array(m0, dtype=np.float64)
    u = prob.solve_fwd(m)
    it, converged, reason = 0, False, 0
    cost_old = prob.cost(u, m)[0]
    gradnorm_ini = float("nan")
    tol = abs_tolerance
    history = []
    while it < max_iter and not converged:
        p = prob.solve_adj(u, m)
        prob.set_point(u, m, p, gauss_newton=it < GN_iter)
        g, gradnorm = prob.gradient(u, m, p)
        if it == 0:
            gradnorm_ini = gradnorm
            tol = max(abs_tolerance, gradnorm_ini * rel_tolerance)
            if gradnorm_ini == 0.0:
                return m, history, 1, True
        if gradnorm < tol and it > 0:
            converged, reason = True, 1
            break
        it += 1
        tolcg = min(cg_coarse_tolerance, math.sqrt(gradnorm / gradnorm_ini))
        mhat, _, actions, _ = steihaug_cg(prob.hessian, prob.Rinv, -g, tolcg,
                                          max_iter=cg_max_iter, reorthogonalize=cg_reorthogonalize)
        mg_mhat = float(g @ mhat)
        accepted, alpha, n_back, cost, u, m = armijo(prob, u, m, mhat, mg_mhat, cost_old,
                                                     c_armijo, max_backtracking_iter,
                                                     gdm_tolerance)
        if accepted:
            cost_old = cost[0]
        history.append({"it": it, "cg_it": actions, "cost": cost[0], "misfit": cost[2],
                        "reg": cost[1], "gdm": mg_mhat, "gradnorm": gradnorm, "alpha": alpha,
                        "tolcg": tolcg})
        if n_back == max_backtracking_iter:
            converged, reason = False, 2
            break
        if -mg_mhat <= gdm_tolerance:
            converged, reason = True, 3
            break
    return m, history, reason, converged


def newton_cg_tr(prob, m0, rel_tolerance=1e-6, abs_tolerance=1e-12, max_iter=20, GN_iter=5,
                 cg_coarse_tolerance=0.5, cg_max_iter=100, cg_reorthogonalize=True, eta=0.05):
    """Returns ``(m, history, reason, converged)``."""
    m = np.array(m0, dtype=np.float64)
    u = prob.solve_fwd(m)
    it, converged, reason = 0, False, 0
    cost_old = cost_new = prob.cost(u, m)[0]
    delta = None
    gradnorm_ini = float("nan")
    tol = abs_tolerance
    history = []
    while it < max_iter and not converged:
        p = prob.solve_adj(u, m)
        prob.set_point(u, m, p, gauss_newton=it < GN_iter)
        g, gradnorm = prob.gradient(u, m, p)
        if it == 0:
            gradnorm_ini = gradnorm
            tol = max(abs_tolerance, gradnorm_ini * rel_tolerance)
        if gradnorm < tol and it > 0:
            converged, reason = True, 1
            break
        it += 1
        tolcg = min(cg_coarse_tolerance, np.sqrt(gradnorm / max(gradnorm_ini, 1e-300)))
        mhat, _, actions, _ = steihaug_cg(prob.hessian, prob.Rinv, -g, tolcg, max_iter=cg_max_iter,
                                          reorthogonalize=cg_reorthogonalize,
                                          tr=None if delta is None else (delta, prob.R))
        if delta is None:
            delta = max(np.sqrt(max(float(prob.R(mhat) @ mhat), 0.0)) * 5.0, 1.0)
        m_star = m + mhat
        u_star = prob.solve_fwd(m_star)
        cost_star = prob.cost(u_star, m_star)
        pred = -(float(g @ mhat) + 0.5 * float(prob.hessian(mhat) @ mhat))
        rho = (cost_old - cost_star[0]) / pred if pred != 0.0 else 0.0
        mhat_R = np.sqrt(max(float(prob.R(mhat) @ mhat), 0.0))
        accept = rho > eta
        if accept:
            m, u = m_star, u_star
            cost_old = cost_new = cost_star[0]
        if rho < 0.25:
            delta *= 0.5
        elif rho > 0.75 and mhat_R >= 0.99 * delta:
            delta *= 2.0
        history.append({"it": it, "cg_it": actions, "cost": cost_new, "gradnorm": gradnorm,
                        "radius": delta, "rho": rho, "accepted": accept, "tolcg": tolcg})
        if delta < 1e-12:
            converged, reason = False, 2
            break
    return m, history, reason, converged
