"""``torch.autograd`` wrappers of the path's hand-written derivative kernels.

The reference differentiates its density with JAX (first and second derivatives in
hippymfem/fem/kernel.py:977-1009, 1343-1405, 1756-1782).  Here every derivative is a
kernel of this library, and these Functions make them usable from ``torch.autograd``:

* ``Residual``: ``r(u, m) = dR/dp``, the weak residual; its vector-Jacobian product is
  ``(A^T rbar, C^T rbar)`` = the assembled vectors ``dR/du`` and ``dR/dm`` evaluated with
  the adjoint slot set to ``rbar`` (one quadrature pass, no matrix formed).
* ``ForwardSolve``: ``u(m)`` with ``R(u, m) = 0`` and the Dirichlet data; its product is
  ``-C^T lambda`` with ``A^T lambda = ubar`` (homogeneous on the Dirichlet nodes) --
  ``solveFwd`` / ``solveAdj`` / ``evalGradientParameter`` of the problem
  (modeling/PDEVariationalProblem.py:1046, 1171, 1365).  With ``recompute=True`` only
  ``m`` is kept and the state is solved again in the backward pass.
* ``Observe``: ``B u`` at the misfit's points (device CSR); its product is ``B^T ybar``.
* ``ReducedGradient``: ``g(m)`` = the gradient of the misfit ``1/(2 sigma^2)|B u(m) - d|^2``
  (modeling/model.py:139-261); its vector-Jacobian product is the reduced Hessian action
  (``ReducedHessian.mult``, modeling/reducedHessian.py:87-131, true Hessian, misfit only),
  so ``torch.autograd.grad(g, m, v)`` is ``H v``.

All tensors are FP64 vectors on the problem's device, in the lattice's node order.
"""

import torch

from .modeling import Model, ReducedHessian
from .problem import ADJOINT, PARAMETER, STATE


class Residual(torch.autograd.Function):
    """``r = Residual.apply(u, m, problem)``: ``dR/dp`` at ``(u, m)`` (no elimination)."""

    @staticmethod
    def forward(ctx, u, m, problem):
        ctx.problem = problem
        ctx.save_for_backward(u, m)
        return problem._residual([u, m, None], ADJOINT).clone()

    @staticmethod
    def backward(ctx, rbar):
        u, m = ctx.saved_tensors
        prob = ctx.problem
        quad = prob._quadrature([u, m, rbar.contiguous()], "vjp")
        _, vecs = prob._assemble(quad, vectors=(STATE, PARAMETER))
        prob._require_finite("the residual's derivatives")
        return vecs[STATE], vecs[PARAMETER], None


class ForwardSolve(torch.autograd.Function):
    """``u = ForwardSolve.apply(m, problem, recompute=False)``."""

    @staticmethod
    def forward(ctx, m, problem, recompute=False):
        u = problem.generate_state()
        problem.solveFwd(u, [u, m, None])
        ctx.problem = problem
        ctx.recompute = bool(recompute)
        if ctx.recompute:
            ctx.save_for_backward(m)
        else:
            ctx.save_for_backward(m, u)
        return u.clone()

    @staticmethod
    def backward(ctx, ubar):
        prob = ctx.problem
        if ctx.recompute:
            (m,) = ctx.saved_tensors
            u = prob.generate_state()
            prob.solveFwd(u, [u, m, None])
        else:
            m, u = ctx.saved_tensors
        lam = prob.generate_adjoint()
        prob.solveAdj(lam, [u, m, None], ubar.contiguous())
        g = prob.generate_parameter()
        prob.evalGradientParameter([u, m, lam], g)
        return -g, None, None


class Observe(torch.autograd.Function):
    """``y = Observe.apply(u, misfit)``: the misfit's observation operator ``B u``."""

    @staticmethod
    def forward(ctx, u, misfit):
        ctx.misfit = misfit
        y = torch.empty(misfit.B.shape[0], dtype=torch.float64, device=u.device)
        misfit.B.mult(u.contiguous(), y)
        return y

    @staticmethod
    def backward(ctx, ybar):
        mis = ctx.misfit
        out = torch.empty(mis.B.shape[1], dtype=torch.float64, device=ybar.device)
        mis.Bt.mult(ybar.contiguous(), out)
        return out, None


def reduced_misfit(m, problem, misfit, recompute=False):
    """``J(m) = 1/(2 sigma^2) |B u(m) - d|^2`` as a differentiable scalar tensor."""
    u = ForwardSolve.apply(m, problem, recompute)
    r = Observe.apply(u, misfit) - misfit.d
    return (0.5 / misfit.noise_variance) * torch.dot(r, r)


class ReducedGradient(torch.autograd.Function):
    """``g = ReducedGradient.apply(m, model)``: the misfit gradient at ``m``; its
    backward applies the reduced (true, misfit-only) Hessian at ``m``."""

    @staticmethod
    def forward(ctx, m, model):
        if not isinstance(model, Model):
            raise TypeError("ReducedGradient needs a Model")
        u, p = model.generate_vector(STATE), model.generate_vector(ADJOINT)
        x = [u, m.detach().clone(), p]
        model.solveFwd(u, x)
        model.solveAdj(p, x)
        g = model.generate_vector(PARAMETER)
        model.evalGradientParameter(x, g)
        ctx.model = model
        ctx.x = x
        return g.clone()

    @staticmethod
    def backward(ctx, gbar):
        model = ctx.model
        model.setPointForHessianEvaluations(ctx.x)
        H = ReducedHessian(model)
        out = model.generate_vector(PARAMETER)
        H.mult(gbar.contiguous(), out)
        return out, None
