"""Inexact Newton-CG in the reduced parameter space, on the device.

Semantics of the reference's ``ReducedSpaceNewtonCG`` (algorithms/NewtonCG.py:262-375,
line-search globalization), its Steihaug CG (algorithms/cgsolverSteihaug.py:71-344,
with the explicit reorthogonalization it uses by default) and its Armijo step
(algorithms/linesearch.py:12-62): at Newton step k the system ``H mhat = -g`` is solved
by preconditioned CG (preconditioner ``R^{-1}`` of the prior, identity without one)
truncated at the Eisenstat-Walker tolerance ``min(cg_coarse_tolerance,
sqrt(|g| / |g_0|))``; the first ``GN_iter`` steps use the Gauss-Newton Hessian; the step
is accepted by Armijo backtracking.  Same parameters, defaults and termination codes.
Vectors are FP64 torch tensors; every Hessian action is ``ReducedHessian.mult`` (two
incremental solves on the device).
"""

import math

import torch

from .modeling import ReducedHessian
from .problem import ADJOINT, PARAMETER, STATE


def ReducedSpaceNewtonCG_ParameterList():
    """The reference's parameters and defaults (NewtonCG.py:79-130).  With
    ``cg_reorthogonalize`` the Hessian actions of a Newton step's CG take their
    incremental solves to ``min(cg_incremental_tolerance, tolcg / 1000)`` and the prior's
    solves in its preconditioner to ``min(cg_preconditioner_tolerance, tolcg / 1000)``
    where that is looser than their own; 0 keeps their own."""
    return {"rel_tolerance": 1e-6, "abs_tolerance": 1e-12, "gdm_tolerance": 1e-18,
            "max_iter": 20, "globalization": "LS", "print_level": 0, "GN_iter": 5,
            "cg_coarse_tolerance": 0.5, "cg_max_iter": 100, "cg_reorthogonalize": True,
            "cg_incremental_tolerance": 1e-6, "cg_preconditioner_tolerance": 1e-6,
            "LS": {"c_armijo": 1e-4, "max_backtracking_iter": 10},
            "TR": {"eta": 0.05}}


def CGSolverSteihaug_ParameterList():
    return {"rel_tolerance": 1e-9, "abs_tolerance": 1e-12, "max_iter": 1000,
            "zero_initial_guess": True, "print_level": 0, "reorthogonalize": False}


class _Identity:
    def solve(self, x, b):
        x.copy_(b)
        return x


class _LooserSolves:
    """A solver whose PCG solves stop at ``tol`` while it is used, where that is looser
    than their own tolerance (the prior's R^{-1} = A^{-1} M A^{-1} as a Newton-CG
    preconditioner)."""

    def __init__(self, solver, tol):
        self.solver, self.tol = solver, float(tol)

    def _pcgs(self):
        out = []
        for name in ("Asolver", "Msolver"):
            inner = getattr(self.solver, name, None)
            pcg = getattr(inner, "pcg", None)
            if pcg is not None:
                out.append(pcg)
        return out

    def solve(self, x, b):
        saved = []
        for pcg in self._pcgs():
            own = pcg.parameters["rel_tolerance"]
            if own < self.tol:
                saved.append((pcg, own))
                pcg.parameters["rel_tolerance"] = self.tol
        try:
            return self.solver.solve(x, b)
        finally:
            for pcg, own in saved:
                pcg.parameters["rel_tolerance"] = own


class CGSolverSteihaug:
    """Preconditioned CG with Steihaug truncation: stops on a direction of nonpositive
    curvature, on the relative/absolute residual in the preconditioner's norm, at
    ``max_iter``, or (``set_TR``) on the boundary of the trust region ``x^T B x <=
    radius^2``.  Without a region a nonpositive direction is taken whole at the first
    iteration and not at all later (cgsolverSteihaug.py:177-197); with one the step goes
    along it to the boundary, to the end the quadratic model prefers."""

    reason = ["Maximum Number of Iterations Reached", "Relative/Absolute residual less than tol",
              "Reached a negative direction", "Reached trust region boundary"]

    def __init__(self, parameters=None):
        self.parameters = parameters if parameters is not None else CGSolverSteihaug_ParameterList()
        self.A = None
        self.B_solver = _Identity()
        self.converged = False
        self.iter = 0
        self.reasonid = 0
        self.final_norm = 0.0
        self.TR_radius_2 = None
        self.B_op = None

    def set_operator(self, A):
        self.A = A
        return self

    def set_TR(self, radius, B_op):
        """Restrict the steps to ``x^T B_op x <= radius^2`` (cgsolverSteihaug.py:117-125)."""
        if not self.parameters["zero_initial_guess"]:
            raise ValueError("a trust region requires zero_initial_guess = True")
        self.TR_radius_2 = float(radius) ** 2
        self.B_op = B_op
        return self

    def _Bdot(self, u, v):
        Bu = torch.empty_like(u)
        self.B_op.mult(u, Bu)
        return float(torch.dot(Bu, v))

    def _update_x(self, x, alpha, d):
        """x += alpha d; with a trust region, a step that leaves it stops on its
        boundary instead (returns True)."""
        if self.TR_radius_2 is None:
            x.add_(d, alpha=alpha)
            return False
        x_bk = x.clone()
        x.add_(d, alpha=alpha)
        if self._Bdot(x, x) < self.TR_radius_2:
            return False
        xx = self._Bdot(x_bk, x_bk)
        dd = self._Bdot(d, d)
        dx = self._Bdot(d, x_bk)
        a_tau = alpha * alpha * dd
        b_half = alpha * dx
        c_tau = xx - self.TR_radius_2
        tau = (-b_half + math.sqrt(max(b_half * b_half - a_tau * c_tau, 0.0))) / a_tau
        x.copy_(x_bk).add_(d, alpha=tau * alpha)
        return True

    def _tau_to_boundary(self, x, d, rd, dAd):
        """The step along d from x to the region's boundary, of the two the one with the
        lower model value -tau r.d + tau^2 d.Ad / 2."""
        a = self._Bdot(d, d)
        b_half = self._Bdot(d, x)
        c = self._Bdot(x, x) - self.TR_radius_2
        disc = math.sqrt(max(b_half * b_half - a * c, 0.0))
        best = None
        for tau in ((-b_half + disc) / a, (-b_half - disc) / a):
            mv = -tau * rd + 0.5 * tau * tau * dAd
            if best is None or mv < best[0]:
                best = (mv, tau)
        return best[1]

    def set_preconditioner(self, B_solver):
        self.B_solver = B_solver if B_solver is not None else _Identity()
        return self

    def solve(self, x, b):
        prm = self.parameters
        self.iter, self.converged, self.reasonid = 0, False, 0
        if prm["zero_initial_guess"]:
            r = b.clone()
            x.zero_()
        else:
            r = torch.empty_like(b)
            self.A.mult(x, r)
            r.neg_().add_(b)
        z = torch.empty_like(b)
        self.B_solver.solve(z, r)
        d = z.clone()
        Ad = torch.empty_like(b)
        nom0 = nom = float(torch.dot(d, r))
        basis = [(r.clone(), z.clone(), nom)] if prm["reorthogonalize"] else None
        r0 = max(nom * prm["rel_tolerance"] ** 2, prm["abs_tolerance"] ** 2)
        if nom <= r0:
            self.converged, self.reasonid = True, 1
            self.final_norm = math.sqrt(max(nom, 0.0))
            return self.iter
        self.A.mult(d, Ad)
        den = float(torch.dot(Ad, d))
        if den <= 0.0:
            return self._negative_curvature(x, r, z, d, Ad, first=True)
        self.iter = 1
        betanom = 0.0
        while True:
            alpha = nom / den
            if self._update_x(x, alpha, d):
                self.converged, self.reasonid = True, 3
                self.final_norm = math.sqrt(max(betanom, 0.0))
                break
            r.add_(Ad, alpha=-alpha)
            if basis is not None:
                for rj, zj, rho in basis:
                    r.add_(rj, alpha=-float(torch.dot(r, zj)) / rho)
            self.B_solver.solve(z, r)
            betanom = float(torch.dot(r, z))
            if betanom < r0:
                self.converged, self.reasonid = True, 1
                self.final_norm = math.sqrt(max(betanom, 0.0))
                break
            self.iter += 1
            if self.iter > prm["max_iter"]:
                self.converged, self.reasonid = False, 0
                self.final_norm = math.sqrt(max(betanom, 0.0))
                break
            if basis is not None:
                basis.append((r.clone(), z.clone(), betanom))
            d.mul_(betanom / nom).add_(z)
            self.A.mult(d, Ad)
            den = float(torch.dot(d, Ad))
            if den <= 0.0:
                return self._negative_curvature(x, r, z, d, Ad, first=False)
            nom = betanom
        return self.iter

    def _negative_curvature(self, x, r, z, d, Ad, first):
        self.converged, self.reasonid = True, 2
        if self.TR_radius_2 is not None:
            tau = self._tau_to_boundary(x, d, float(torch.dot(r, d)), float(torch.dot(d, Ad)))
        else:
            tau = 1.0 if first else 0.0
        if tau != 0.0:
            x.add_(d, alpha=tau)
            r.add_(Ad, alpha=-tau)
            self.B_solver.solve(z, r)
        self.final_norm = math.sqrt(max(float(torch.dot(r, z)), 0.0))
        return self.iter


def armijo_backtrack(model, x, x_star, mhat, mg_mhat, cost_old, alpha=1.0, c_armijo=1e-4,
                     max_backtracking=10, gdm_tolerance=None, failures=(RuntimeError,)):
    """Try ``x + alpha mhat``, halving ``alpha`` until the cost decreases enough
    (linesearch.py:12-62); returns ``(accepted, alpha, n_backtrack, cost, fwd_failed)``."""
    n_back, fwd_failed, cost = 0, False, None
    while n_back < max_backtracking:
        x_star[PARAMETER].copy_(x[PARAMETER]).add_(mhat, alpha=alpha)
        x_star[STATE].copy_(x[STATE])
        try:
            model.solveFwd(x_star[STATE], x_star)
            cost = list(model.cost(x_star))
            fwd_failed = False
        except failures:
            cost = [cost_old + 1.0, float("nan"), float("nan")]
            fwd_failed = True
        if (cost[0] < cost_old + alpha * c_armijo * mg_mhat
                or (gdm_tolerance is not None and -mg_mhat <= gdm_tolerance)):
            x[PARAMETER].copy_(x_star[PARAMETER])
            x[STATE].copy_(x_star[STATE])
            return True, alpha, n_back, cost, fwd_failed
        n_back += 1
        alpha *= 0.5
    return False, alpha, n_back, cost, fwd_failed


class ReducedSpaceNewtonCG:
    """``ReducedSpaceNewtonCG(model, parameters=None, callback=None).solve(x)`` with
    ``x = [u, m, p]``; ``m`` is the initial guess and the result."""

    termination_reasons = ["Maximum number of Iteration reached",
                           "Norm of the gradient less than tolerance",
                           "Maximum number of backtracking reached",
                           "Norm of (g, dm) less than tolerance",
                           "Forward solve failed during backtracking"]

    def __init__(self, model, parameters=None, callback=None):
        self.model = model
        self.parameters = parameters if parameters is not None else ReducedSpaceNewtonCG_ParameterList()
        self.callback = callback
        self.it = 0
        self.converged = False
        self.total_cg_iter = 0
        self.ncalls = 0
        self.reason = 0
        self.final_grad_norm = float("nan")
        self.final_cost = float("nan")
        self.history = []

    def solve(self, x):
        g = self.parameters["globalization"]
        if g == "LS":
            return self._solve_ls(x)
        if g == "TR":
            return self._solve_tr(x)
        raise ValueError("unknown globalization %r" % (g,))

    def _solve_tr(self, x):
        """Trust-region globalization (NewtonCG.py:377-493): the Newton step from
        Steihaug CG inside the region ``mhat^T R mhat <= delta^2`` of the prior's
        precision (the first step unrestricted, setting ``delta = max(5 |mhat|_R, 1)``),
        accepted when the actual over the predicted reduction exceeds ``eta``; the radius
        halves below 1/4 and doubles above 3/4 when the step reached the boundary.  Needs a
        prior.  Termination codes as the line search (2: the radius fell below 1e-12)."""
        p = self.parameters
        model = self.model
        if model.prior is None:
            raise ValueError("the trust region is measured with the prior's precision")
        rel_tol, abs_tol = p["rel_tolerance"], p["abs_tolerance"]
        eta = p["TR"]["eta"]
        model.solveFwd(x[STATE], x)
        self.it, self.converged = 0, False
        self.ncalls += 1
        mhat = model.generate_vector(PARAMETER)
        R_mhat = model.generate_vector(PARAMETER)
        mg = model.generate_vector(PARAMETER)
        x_star = [model.generate_vector(STATE), model.generate_vector(PARAMETER), None]
        cost_old = model.cost(x)[0]
        cost_new = cost_old
        delta = None
        gradnorm = gradnorm_ini = float("nan")
        tol = abs_tol
        while self.it < p["max_iter"] and not self.converged:
            model.solveAdj(x[ADJOINT], x)
            model.setPointForHessianEvaluations(x, gauss_newton_approx=(self.it < p["GN_iter"]))
            gradnorm = model.evalGradientParameter(x, mg)
            if self.it == 0:
                gradnorm_ini = gradnorm
                tol = max(abs_tol, gradnorm_ini * rel_tol)
            if gradnorm < tol and self.it > 0:
                self.converged, self.reason = True, 1
                break
            self.it += 1
            tolcg = min(p["cg_coarse_tolerance"], math.sqrt(gradnorm / max(gradnorm_ini, 1e-300)))
            H = ReducedHessian(model)
            solver = CGSolverSteihaug()
            solver.set_operator(H)
            solver.set_preconditioner(model.Rsolver())
            if delta is not None:
                solver.set_TR(delta, model.prior.R)
            solver.parameters.update({"rel_tolerance": tolcg, "max_iter": p["cg_max_iter"],
                                      "zero_initial_guess": True,
                                      "reorthogonalize": bool(p["cg_reorthogonalize"])})
            solver.solve(mhat, -mg)
            self.total_cg_iter += H.ncalls
            cg_it = H.ncalls
            if delta is None:
                model.applyR(mhat, R_mhat)
                delta = max(math.sqrt(max(float(torch.dot(R_mhat, mhat)), 0.0)) * 5.0, 1.0)
            x_star[PARAMETER].copy_(x[PARAMETER]).add_(mhat)
            x_star[STATE].copy_(x[STATE])
            model.solveFwd(x_star[STATE], x_star)
            cost_star = list(model.cost(x_star))
            Hmhat = model.generate_vector(PARAMETER)
            H.mult(mhat, Hmhat)
            pred = -(float(torch.dot(mg, mhat)) + 0.5 * float(torch.dot(Hmhat, mhat)))
            actual = cost_old - cost_star[0]
            rho = actual / pred if pred != 0.0 else 0.0
            model.applyR(mhat, R_mhat)
            mhat_R = math.sqrt(max(float(torch.dot(R_mhat, mhat)), 0.0))
            accept = rho > eta
            if accept:
                x[PARAMETER].copy_(x_star[PARAMETER])
                x[STATE].copy_(x_star[STATE])
                cost_old = cost_new = cost_star[0]
            if rho < 0.25:
                delta *= 0.5
            elif rho > 0.75 and mhat_R >= 0.99 * delta:
                delta *= 2.0
            self.history.append({"it": self.it, "cg_it": cg_it, "cost": cost_new,
                                 "gradnorm": gradnorm, "radius": delta, "rho": rho,
                                 "accepted": accept, "tolcg": tolcg})
            if p["print_level"] >= 0:
                print("newton-TR %2d: cg %3d  cost %.8e  |g| %.3e  radius %.4g  rho %.4g%s"
                      % (self.it, cg_it, cost_new, gradnorm, delta, rho,
                         "" if accept else "  (rejected)"), flush=True)
            if self.callback:
                self.callback(self.it, x)
            if delta < 1e-12:
                self.converged, self.reason = False, 2
                break
        self.final_grad_norm = gradnorm
        self.final_cost = cost_new
        return x

    def _solve_ls(self, x):
        p = self.parameters
        rel_tol, abs_tol = p["rel_tolerance"], p["abs_tolerance"]
        model = self.model
        model.solveFwd(x[STATE], x)
        self.it, self.converged = 0, False
        self.ncalls += 1
        mhat = model.generate_vector(PARAMETER)
        mg = model.generate_vector(PARAMETER)
        x_star = [model.generate_vector(STATE), model.generate_vector(PARAMETER), None]
        cost_old = model.cost(x)[0]
        cost_new = cost_old
        reorth = bool(p["cg_reorthogonalize"])
        gradnorm = gradnorm_ini = float("nan")
        tol = abs_tol
        while self.it < p["max_iter"] and not self.converged:
            model.solveAdj(x[ADJOINT], x)
            model.setPointForHessianEvaluations(x, gauss_newton_approx=(self.it < p["GN_iter"]))
            gradnorm = model.evalGradientParameter(x, mg)
            if self.it == 0:
                gradnorm_ini = gradnorm
                tol = max(abs_tol, gradnorm_ini * rel_tol)
                if gradnorm_ini == 0.0:
                    self.converged, self.reason = True, 1
                    break
            if gradnorm < tol and self.it > 0:
                self.converged, self.reason = True, 1
                break
            self.it += 1
            tolcg = min(p["cg_coarse_tolerance"], math.sqrt(gradnorm / gradnorm_ini))
            H = ReducedHessian(model)
            inc = float(p.get("cg_incremental_tolerance") or 0.0)
            if reorth and inc > 0.0:
                H.set_accuracy(min(inc, 1e-3 * tolcg))
            prec = model.Rsolver() if model.prior is not None else None
            ptol = float(p.get("cg_preconditioner_tolerance") or 0.0)
            if prec is not None and reorth and ptol > 0.0:
                prec = _LooserSolves(prec, min(ptol, 1e-3 * tolcg))
            solver = CGSolverSteihaug()
            solver.set_operator(H)
            solver.set_preconditioner(prec)
            solver.parameters.update({"rel_tolerance": tolcg, "max_iter": p["cg_max_iter"],
                                      "zero_initial_guess": True,
                                      "reorthogonalize": bool(p["cg_reorthogonalize"])})
            solver.solve(mhat, -mg)
            self.total_cg_iter += H.ncalls
            mg_mhat = float(torch.dot(mg, mhat))
            accepted, alpha, n_back, cost, fwd_failed = armijo_backtrack(
                model, x, x_star, mhat, mg_mhat, cost_old, c_armijo=p["LS"]["c_armijo"],
                max_backtracking=p["LS"]["max_backtracking_iter"],
                gdm_tolerance=p["gdm_tolerance"])
            cost_new = cost[0]                      # the last trial's, accepted or not
            if accepted:
                cost_old = cost_new
            self.history.append({"it": self.it, "cg_it": H.ncalls, "cost": cost[0],
                                 "misfit": cost[2], "reg": cost[1], "gdm": mg_mhat,
                                 "gradnorm": gradnorm, "alpha": alpha, "tolcg": tolcg})
            if p["print_level"] >= 0:
                print("newton %2d: cg %3d  cost %.8e (misfit %.6e, reg %.6e)  (g,dm) %+.3e  "
                      "|g| %.3e  alpha %.4g  tolcg %.3e"
                      % tuple(self.history[-1][k] for k in ("it", "cg_it", "cost", "misfit",
                                                             "reg", "gdm", "gradnorm", "alpha",
                                                             "tolcg")), flush=True)
            if self.callback:
                self.callback(self.it, x)
            if n_back == p["LS"]["max_backtracking_iter"]:
                self.converged = False
                self.reason = 4 if fwd_failed else 2
                break
            if -mg_mhat <= p["gdm_tolerance"]:
                self.converged, self.reason = True, 3
                break
        self.final_grad_norm = gradnorm
        self.final_cost = cost_new
        return x
