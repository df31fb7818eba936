"""Misfit, model and reduced Hessian on top of ``PDEVariationalProblem``.

Mirrors, with the same method names and signs:

* ``DiscreteStateObservation`` / ``PointwiseStateObservation`` --
  hippymfem/modeling/misfit.py:65-125 and the observation operator of
  hippymfem/modeling/pointwiseObservation.py:36-224 (rows of Q2 basis values at the
  points), held as device CSR matrices ``B`` and ``B^T``;
* ``BiLaplacianPrior`` -- hippymfem/modeling/prior.py:894-952 (isotropic, natural BCs);
* ``Model`` -- the block dispatch of hippymfem/modeling/model.py:100-261;
* ``ReducedHessian`` -- hippymfem/modeling/reducedHessian.py:30-131.
"""

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr
from .problem import ADJOINT, PARAMETER, STATE


def targets_in_box(mesh, points):
    """Mask of the targets inside the box: the test ``hm_lattice_observation`` applies,
    ``-1e-12 <= x / h <= n + 1e-12`` on every axis (the same IEEE division), finite."""
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    s = pts / np.asarray(mesh.h, dtype=np.float64)
    n = np.asarray(mesh.n, dtype=np.float64)
    return np.all((s >= -1e-12) & (s <= n + 1e-12), axis=1)


def device_observation_operator(mesh, points, missing="raise"):
    """``B`` on the device (``hm_lattice_observation``): row ``o`` holds the 27 Q2 basis
    values at the o-th target in the element containing it (pointwiseObservation.py:94-170).
    Targets outside the box follow the reference's ``missing`` policy (:53-57, :104-112):
    ``"raise"`` raises ``ValueError``; ``"warn"`` prints a warning and ``"ignore"`` says
    nothing, and both leave those targets out (``B`` has a row per target inside, in
    target order; their indices are ``B.owned_targets``)."""
    if missing not in ("raise", "warn", "ignore"):
        raise ValueError("missing must be 'raise', 'warn' or 'ignore', got %r" % (missing,))
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
    inside = targets_in_box(mesh, pts)
    owned = np.nonzero(inside)[0]
    if owned.size < pts.shape[0]:
        bad = pts[~inside]
        msg = ("%d observation target(s) are outside the mesh, e.g. %s"
               % (bad.shape[0], bad[:3].tolist()))
        if missing == "raise":
            raise ValueError(msg)
        if missing == "warn":
            print("warning: " + msg, flush=True)
        pts = np.ascontiguousarray(pts[owned])
    npts = pts.shape[0]
    dev = mesh.device
    P = torch.as_tensor(pts, device=dev)
    indptr = torch.empty(npts + 1, dtype=torch.int32, device=dev)
    indices = torch.empty(max(27 * npts, 1), dtype=torch.int32, device=dev)
    values = torch.empty(max(27 * npts, 1), dtype=torch.float64, device=dev)
    work = torch.empty(lib.hm_lattice_observation_workspace_bytes(npts), dtype=torch.uint8,
                       device=dev)
    rc = lib.hm_lattice_observation(mesh.handle, ptr(P), npts, ptr(indptr), ptr(indices),
                                    ptr(values), ptr(work), stream_ptr())
    if rc == _lib.HM_ERR_RANGE:   # targets_in_box applies the kernel's own test
        raise ValueError("observation targets outside the mesh")
    check(rc, "hm_lattice_observation")
    B = DeviceCSR.from_device(indptr, indices[:27 * npts], values[:27 * npts],
                              (npts, mesh.ndof))
    B.owned_targets = owned
    return B


def observation_operator(mesh, points, missing="raise"):
    """Host (scipy) copy of ``device_observation_operator(mesh, points, missing)``."""
    return device_observation_operator(mesh, points, missing).to_scipy()


class DeviceCSR:
    """A general (rectangular) CSR matrix on the device, applied by ``hm_csr_spmv``;
    ``transpose()`` by ``hm_csr_transpose``."""

    def __init__(self, M, device):
        M = sp.csr_matrix(M)
        M.sort_indices()
        self.shape = M.shape
        self.indptr = torch.as_tensor(M.indptr.astype(np.int32), device=device)
        self.indices = torch.as_tensor(M.indices.astype(np.int32), device=device)
        self.values = torch.as_tensor(M.data.astype(np.float64), device=device)

    @classmethod
    def from_device(cls, indptr, indices, values, shape):
        self = cls.__new__(cls)
        self.shape = (int(shape[0]), int(shape[1]))
        self.indptr, self.indices, self.values = indptr, indices, values
        return self

    @property
    def nnz(self):
        return int(self.values.numel())

    def transpose(self):
        nrow, ncol = self.shape
        dev = self.values.device
        nnz = self.nnz
        tindptr = torch.empty(ncol + 1, dtype=torch.int32, device=dev)
        tindices = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        tvalues = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
        work = torch.empty(lib.hm_csr_transpose_workspace_bytes(ncol), dtype=torch.uint8,
                           device=dev)
        check(lib.hm_csr_transpose(nrow, ncol, nnz, ptr(self.indptr), ptr(self.indices),
                                   ptr(self.values), ptr(tindptr), ptr(tindices), ptr(tvalues),
                                   ptr(work), stream_ptr()), "hm_csr_transpose")
        return DeviceCSR.from_device(tindptr, tindices[:nnz], tvalues[:nnz], (ncol, nrow))

    def to_scipy(self):
        return sp.csr_matrix((self.values.cpu().numpy(), self.indices.cpu().numpy(),
                              self.indptr.cpu().numpy()), shape=self.shape)

    def mult(self, x, y, alpha=1.0, beta=0.0):
        check(lib.hm_csr_spmv(self.shape[0], ptr(self.indptr), ptr(self.indices),
                              ptr(self.values), ptr(x), ptr(y), float(alpha), float(beta),
                              stream_ptr()), "hm_csr_spmv")
        return y


class DiscreteStateObservation:
    """Gaussian misfit ``1/(2 sigma^2) |B u - d|^2`` (misfit.py:65-110)."""

    def __init__(self, B, data=None, noise_variance=None, device="cuda"):
        if noise_variance is None:
            raise ValueError("noise_variance must be specified")
        if noise_variance == 0:
            raise ZeroDivisionError("noise_variance must not be 0; use 1.0 for a deterministic "
                                    "inverse problem")
        self.B = B if isinstance(B, DeviceCSR) else DeviceCSR(B, device)
        self.Bt = self.B.transpose()
        self._Bh = None
        nobs = self.B.shape[0]
        if isinstance(data, torch.Tensor):
            self.d = data.to(device=device, dtype=torch.float64).clone()
        elif data is not None:
            self.d = torch.as_tensor(np.asarray(data, dtype=np.float64), device=device)
        else:
            self.d = torch.zeros(nobs, dtype=torch.float64, device=device)
        self.Bu = torch.zeros(nobs, dtype=torch.float64, device=device)
        self.noise_variance = float(noise_variance)

    @property
    def Bh(self):
        """Host (scipy) copy of ``B``."""
        if self._Bh is None:
            self._Bh = self.B.to_scipy()
        return self._Bh

    def cost(self, x):
        self.B.mult(x[STATE], self.Bu)
        self.Bu.sub_(self.d)
        return 0.5 / self.noise_variance * float(torch.dot(self.Bu, self.Bu))

    def grad(self, i, x, out):
        if i == STATE:
            self.B.mult(x[STATE], self.Bu)
            self.Bu.sub_(self.d)
            self.Bt.mult(self.Bu, out, alpha=1.0 / self.noise_variance)
        elif i == PARAMETER:
            out.zero_()
        else:
            raise IndexError("grad index %r" % (i,))
        return out

    def setLinearizationPoint(self, x, gauss_newton_approx=False):
        return self

    def block_is_zero(self, i, j):
        return not (i == STATE and j == STATE)

    def apply_ij(self, i, j, dir, out):
        if i == STATE and j == STATE:
            self.B.mult(dir, self.Bu)
            self.Bt.mult(self.Bu, out, alpha=1.0 / self.noise_variance)
        else:
            out.zero_()
        return out


def PointwiseStateObservation(Vh, obs_points, data=None, noise_variance=None, missing="raise"):
    """Misfit for pointwise observations of the state at ``obs_points`` (``data`` per
    target inside the mesh; ``missing`` as for ``device_observation_operator``)."""
    mesh = Vh.mesh
    return DiscreteStateObservation(device_observation_operator(mesh, obs_points, missing),
                                    data, noise_variance, device=mesh.device)


class _BlockSolver:
    """``x = M^{-1} b`` for an assembled SPD block (Jacobi-PCG, from zero)."""

    def __init__(self, block, rel_tolerance, max_iter):
        from .sparse import PCGSolver
        self.pcg = PCGSolver(block, rel_tolerance=rel_tolerance, max_iter=max_iter)

    def solve(self, x, b):
        x.zero_()
        self.pcg.solve(x, b)
        return x


class _BilaplacianR:
    """``R = A M^{-1} A`` applied matrix-free (prior.py:319-350)."""

    def __init__(self, A, Msolver):
        self.A, self.Msolver = A, Msolver
        self._t1 = torch.empty(A.nrow, dtype=torch.float64, device=A.values.device)
        self._t2 = torch.empty_like(self._t1)

    def mult(self, x, y):
        self.A.mult(x, self._t1)
        self.Msolver.solve(self._t2, self._t1)
        self.A.mult(self._t2, y)
        return y

    multTranspose = mult


class _BilaplacianRsolver:
    """``R^{-1} = A^{-1} M A^{-1}`` (prior.py:353-373)."""

    def __init__(self, Asolver, M):
        self.Asolver, self.M = Asolver, M
        self._t1 = torch.empty(M.nrow, dtype=torch.float64, device=M.values.device)
        self._t2 = torch.empty_like(self._t1)

    def solve(self, x, b):
        self.Asolver.solve(self._t1, b)
        self.M.mult(self._t1, self._t2)
        self.Asolver.solve(x, self._t2)
        return x


class BiLaplacianPrior:
    """Matern-class Gaussian prior with precision ``R = A M^{-1} A``,
    ``A = gamma div(Theta grad) + delta M`` with natural boundary conditions, plus with
    ``robin_bc`` the boundary term ``beta M_boundary``, ``beta = sqrt(gamma delta) /
    1.42``: BiLaplacianPrior of modeling/prior.py:894-952.  ``Theta``: ``None``
    (isotropic), a scalar, or a constant diagonal tensor (a 3-vector or a diagonal 3 x 3
    array); a tensor with off-diagonal entries or a spatially varying one, and the lumped
    mass, are not part of this prior.

    The operators come from the fused assembly kernel on the lattice's pattern: ``gamma
    K`` is the Jacobian block ``A`` at the constant field ``m = log gamma``, and
    ``delta M`` the block ``W_mm`` at ``u = p = x`` (so that ``grad u . grad p = 1``) and
    ``m = log delta``; no Dirichlet elimination.  A diagonal ``Theta`` scales the
    element sizes of the stiffness lattice to ``h / sqrt(theta)`` (the derivative terms
    take ``theta / h^2``) with ``m = log gamma + log(theta_x theta_y theta_z) / 2``
    restoring ``|J|``; the Robin term is added by ``hm_lattice_add_boundary_mass``.
    Solves with ``A`` and ``M`` are Jacobi-PCG to ``rel_tol``."""

    def __init__(self, Vh, gamma, delta, Theta=None, mean=None, rel_tol=1e-12, max_iter=1000,
                 robin_bc=False, lumped_mass=False):
        import math

        import numpy as np

        from .mesh import BoxMesh
        from .pattern import LatticePattern
        from .sparse import CSRBlock

        if lumped_mass:
            raise NotImplementedError("the lumped mass is not part of this prior")
        if not (gamma > 0 and delta > 0):
            raise ValueError("gamma and delta must be positive")
        theta = self._theta(Theta)
        self.Vh = Vh
        mesh = Vh.mesh
        self.gamma, self.delta, self.robin_bc = float(gamma), float(delta), bool(robin_bc)
        self.Theta = theta
        pat = LatticePattern(mesh)

        status = torch.zeros(1, dtype=torch.int32, device=mesh.device)
        quad = torch.empty((mesh.quad_bytes() + 7) // 8, dtype=torch.float64, device=mesh.device)

        def block(msh, name, u, logc, p):
            # msh: the lattice of the prior's mesh, or its rescaled copy (same pattern)
            const = Vh.vector()
            const.fill_(float(logc))
            check(lib.hm_lattice_quadrature(msh.handle, ptr(u), ptr(const), ptr(p), _lib.HM_FP64,
                                            ptr(quad), ptr(status), stream_ptr()),
                  "hm_lattice_quadrature")
            vals = pat.new_values()
            check(lib.hm_lattice_assemble(
                msh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr), None, 0.0,
                ptr(vals) if name == "A" else None, None, None,
                ptr(vals) if name == "Wmm" else None, None, None, None, 0, stream_ptr()),
                "hm_lattice_assemble")
            if int(status.item()) & _lib.HM_STATUS_NONFINITE:
                raise RuntimeError("non-finite values in the prior's operators")
            return vals

        x = torch.as_tensor(mesh.node_coords()[:, 0], device=mesh.device).contiguous()
        zero = Vh.vector()
        logg = math.log(self.gamma)
        stiff = mesh
        if theta is not None and np.all(theta == theta[0]):
            logg += math.log(theta[0])                      # isotropic: gamma theta
        elif theta is not None:
            logg += 0.5 * float(np.sum(np.log(theta)))
            stiff = BoxMesh(mesh.n, tuple(Ld / math.sqrt(t) for Ld, t in zip(mesh.L, theta)),
                            device=mesh.device)
        K = block(stiff, "A", zero, logg, zero)
        Md = block(mesh, "Wmm", x, math.log(self.delta), x)
        M1 = block(mesh, "Wmm", x, 0.0, x)
        K.add_(Md)
        if self.robin_bc:
            beta = math.sqrt(self.gamma * self.delta) / 1.42
            check(lib.hm_lattice_add_boundary_mass(mesh.handle, beta, ptr(K), stream_ptr()),
                  "hm_lattice_add_boundary_mass")
        self.A = CSRBlock(pat, K)
        self.M = CSRBlock(pat, M1)
        self.Msolver = _BlockSolver(self.M, rel_tol, max_iter)
        self.Asolver = _BlockSolver(self.A, rel_tol, max_iter)
        self.R = _BilaplacianR(self.A, self.Msolver)
        self.Rsolver = _BilaplacianRsolver(self.Asolver, self.M)
        self.mean = mean.clone() if mean is not None else Vh.vector()

    @staticmethod
    def _theta(Theta):
        """``None`` or the three diagonal entries of a constant ``Theta``."""
        import numbers

        import numpy as np

        if Theta is None:
            return None
        if isinstance(Theta, numbers.Number):
            t = np.full(3, float(Theta))
        else:
            a = np.asarray(Theta, dtype=float)
            if a.shape == (3,):
                t = a.copy()
            elif a.shape == (3, 3):
                if np.any(a - np.diag(np.diag(a))):
                    raise NotImplementedError("Theta with off-diagonal entries is not part of "
                                              "this prior (the lattice kernels assemble "
                                              "axis-aligned diffusion)")
                t = np.diag(a).copy()
            else:
                raise NotImplementedError("Theta must be a scalar, a 3-vector or a constant "
                                          "diagonal 3 x 3 array")
        if not np.all(t > 0):
            raise ValueError("Theta must be positive definite")
        return t

    def init_vector(self, x=None, dim=0):
        return self.Vh.vector()

    def cost(self, m):
        """``1/2 (m - mean)^T R (m - mean)`` (prior.py:575-580)."""
        d = m - self.mean
        Rd = torch.empty_like(d)
        self.R.mult(d, Rd)
        return 0.5 * float(torch.dot(Rd, d))

    def grad(self, m, out):
        """``R (m - mean)`` (prior.py:582-586)."""
        self.R.mult(m - self.mean, out)
        return out


class Model:
    """``Model(problem, prior, misfit)``: the block dispatch of model.py:201-261; the prior
    may be ``None`` (a misfit-only model: no regularization cost, gradient or ``R``)."""

    def __init__(self, problem, prior, misfit):
        self.problem = problem
        self.prior = prior
        self.misfit = misfit
        self.gauss_newton_approx = False
        self.n_fwd_solve = self.n_adj_solve = self.n_inc_solve = 0

    def generate_vector(self, component="ALL"):
        gen = {STATE: self.problem.generate_state, PARAMETER: self.problem.generate_parameter,
               ADJOINT: self.problem.generate_adjoint}
        if component == "ALL":
            return [gen[i]() for i in (STATE, PARAMETER, ADJOINT)]
        return gen[component]()

    def cost(self, x):
        """``[total, regularization, misfit]`` at ``x`` (model.py:213-217)."""
        misfit = self.misfit.cost(x)
        reg = self.prior.cost(x[PARAMETER]) if self.prior is not None else 0.0
        return [misfit + reg, reg, misfit]

    def solveFwd(self, out, x):
        self.n_fwd_solve += 1
        return self.problem.solveFwd(out, x)

    def solveAdj(self, out, x):
        self.n_adj_solve += 1
        rhs = self.problem.generate_state()
        self.misfit.grad(STATE, x, rhs)
        rhs.neg_()
        return self.problem.solveAdj(out, x, rhs)

    def evalGradientParameter(self, x, mg, misfit_only=False):
        """The cost's gradient in ``mg`` (model.py:219-236); returns its norm, the
        discrete L2 norm ``sqrt(g^T M^{-1} g)`` with a prior, the Euclidean one
        without."""
        self.problem.evalGradientParameter(x, mg)
        if self.prior is None:
            return float(torch.sqrt(torch.dot(mg, mg)))
        if not misfit_only:
            tmp = self.problem.generate_parameter()
            self.prior.grad(x[PARAMETER], tmp)
            mg.add_(tmp)
        g = self.problem.generate_parameter()
        self.prior.Msolver.solve(g, mg)
        return max(float(torch.dot(g, mg)), 0.0) ** 0.5

    def setPointForHessianEvaluations(self, x, gauss_newton_approx=False):
        self.gauss_newton_approx = bool(gauss_newton_approx)
        self.problem.setLinearizationPoint(x, self.gauss_newton_approx)
        self.misfit.setLinearizationPoint(x, self.gauss_newton_approx)
        return self

    def solveFwdIncremental(self, sol, rhs, rel_tolerance=None):
        self.n_inc_solve += 1
        return self.problem.solveIncremental(sol, rhs, False, rel_tolerance=rel_tolerance)

    def solveAdjIncremental(self, sol, rhs, rel_tolerance=None):
        self.n_inc_solve += 1
        return self.problem.solveIncremental(sol, rhs, True, rel_tolerance=rel_tolerance)

    def applyC(self, dm, out):
        return self.problem.apply_ij(ADJOINT, PARAMETER, dm, out)

    def applyCt(self, dp, out):
        return self.problem.apply_ij(PARAMETER, ADJOINT, dp, out)

    def applyWuu(self, du, out):
        self.misfit.apply_ij(STATE, STATE, du, out)
        return out

    def _second_order(self, i, j, d, out):
        if self.gauss_newton_approx:
            out.zero_()
            return out
        return self.problem.apply_ij(i, j, d, out)

    def applyWum(self, dm, out):
        return self._second_order(STATE, PARAMETER, dm, out)

    def applyWmu(self, du, out):
        return self._second_order(PARAMETER, STATE, du, out)

    def applyWmm(self, dm, out):
        return self._second_order(PARAMETER, PARAMETER, dm, out)

    def applyR(self, dm, out):
        if self.prior is None:
            out.zero_()
            return out
        return self.prior.R.mult(dm, out)

    def Rsolver(self):
        """The solver of the prior's precision (the Newton-CG preconditioner)."""
        if self.prior is None:
            raise ValueError("a misfit-only model has no prior precision")
        return self.prior.Rsolver


class ReducedHessian:
    """Matrix-free reduced Hessian at the point set on the model (reducedHessian.py)."""

    def __init__(self, model, misfit_only=False):
        self.model = model
        self.gauss_newton_approx = model.gauss_newton_approx
        self.misfit_only = bool(misfit_only)
        self.ncalls = 0
        self.rhs_fwd = model.generate_vector(STATE)
        self.rhs_adj = model.generate_vector(ADJOINT)
        self.rhs_adj2 = model.generate_vector(ADJOINT)
        self.uhat = model.generate_vector(STATE)
        self.phat = model.generate_vector(ADJOINT)
        self.yhelp = model.generate_vector(PARAMETER)
        self.accuracy = None
        self.iterations = []

    def set_accuracy(self, tolerance):
        self.accuracy = float(tolerance) if tolerance else None
        return self

    def _incremental(self, adjoint, sol, rhs):
        solve = self.model.solveAdjIncremental if adjoint else self.model.solveFwdIncremental
        solve(sol, rhs, rel_tolerance=self.accuracy)
        self.iterations.append(self.model.problem.last_solve.iterations)
        return sol

    def mult(self, x, y):
        if self.gauss_newton_approx:
            self.GNHessian(x, y)
        else:
            self.TrueHessian(x, y)
        self.ncalls += 1
        return y

    multTranspose = mult

    def inner(self, x, y):
        Hx = self.model.generate_vector(PARAMETER)
        self.mult(x, Hx)
        return float(torch.dot(Hx, y))

    def _applyCt(self, dp, out):
        # C^T dp as dR/dm from the point's fields where the problem offers it
        prob = self.model.problem
        if hasattr(prob, "transposed_product"):
            return prob.transposed_product(PARAMETER, ADJOINT, dp, out)
        return self.model.applyCt(dp, out)

    def GNHessian(self, x, y):
        self.model.applyC(x, self.rhs_fwd)
        self._incremental(False, self.uhat, self.rhs_fwd)
        self.model.applyWuu(self.uhat, self.rhs_adj)
        self._incremental(True, self.phat, self.rhs_adj)
        self._applyCt(self.phat, y)
        if not self.misfit_only:
            self.model.applyR(x, self.yhelp)
            y.add_(self.yhelp)
        return y

    def TrueHessian(self, x, y):
        # C x, W_um x and W_mm x in one pass over the point's fields where the problem
        # offers it (reducedHessian.py:102-131 takes them as three block products)
        prob = self.model.problem
        fwd = (prob.directional_products(x) if hasattr(prob, "directional_products")
               and not self.model.gauss_newton_approx else None)
        if fwd is not None:
            self.rhs_fwd.copy_(fwd[ADJOINT])
        else:
            self.model.applyC(x, self.rhs_fwd)
        self._incremental(False, self.uhat, self.rhs_fwd)
        self.model.applyWuu(self.uhat, self.rhs_adj)
        if fwd is not None:
            self.rhs_adj.sub_(fwd[STATE])
        else:
            self.model.applyWum(x, self.rhs_adj2)
            self.rhs_adj.sub_(self.rhs_adj2)
        self._incremental(True, self.phat, self.rhs_adj)
        if fwd is not None:
            y.copy_(fwd[PARAMETER])
        else:
            self.model.applyWmm(x, y)
        self._applyCt(self.phat, self.yhelp)
        y.add_(self.yhelp)
        if fwd is not None and hasattr(prob, "transposed_product"):
            prob.transposed_product(PARAMETER, STATE, self.uhat, self.yhelp)
        else:
            self.model.applyWmu(self.uhat, self.yhelp)
        y.sub_(self.yhelp)
        if not self.misfit_only:
            self.model.applyR(x, self.yhelp)
            y.add_(self.yhelp)
        return y
