"""Assembled blocks on the device and the FP64 Jacobi-PCG of the incremental solves.

``CSRBlock`` stands where the reference holds a ``HypreParMatrix`` built over the
scatter pattern (hippymfem/fem/parmat.py:106-171): its ``Mult``/``MultTranspose`` are
``hm_csr_spmv`` / ``hm_csr_spmv_t``.  ``pcg`` replaces the hypre PCG behind
``KrylovSolver.solve`` (hippymfem/algorithms/linSolvers.py:709); the preconditioner is
Jacobi (BoomerAMG is out of scope).
"""

import ctypes

import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr


class CSRBlock:
    """A square block in a (shared) device pattern, FP64 values."""

    def __init__(self, pattern, values):
        self.pattern = pattern
        self.values = values
        self.nrow = pattern.nrow
        self.ncol = pattern.ncol

    def Height(self):
        return self.nrow

    def Width(self):
        return self.ncol

    def mult(self, x, y, alpha=1.0, beta=0.0, stream=None):
        """``y = alpha A x + beta y``."""
        p = self.pattern
        check(lib.hm_csr_spmv(self.nrow, ptr(p.indptr), ptr(p.indices), ptr(self.values), ptr(x),
                              ptr(y), float(alpha), float(beta), stream_ptr(stream)), "hm_csr_spmv")
        return y

    def mult_transpose(self, x, y, alpha=1.0, beta=0.0, stream=None):
        """``y = alpha A^T x + beta y`` (a gather through the transpose map)."""
        p = self.pattern
        if p.tpos is None:
            raise ValueError("the pattern was built without its transpose map")
        check(lib.hm_csr_spmv_t(self.nrow, ptr(p.indptr), ptr(p.indices), ptr(p.tpos),
                                ptr(self.values), ptr(x), ptr(y), float(alpha), float(beta),
                                stream_ptr(stream)), "hm_csr_spmv_t")
        return y

    Mult = mult
    MultTranspose = mult_transpose

    def diagonal(self, out=None, stream=None):
        out = out if out is not None else torch.empty(self.nrow, dtype=torch.float64,
                                                      device=self.values.device)
        check(lib.hm_csr_diag(self.nrow, ptr(self.pattern.indptr), ptr(self.values), ptr(out),
                              stream_ptr(stream)), "hm_csr_diag")
        return out

    def to_scipy(self):
        import scipy.sparse as sp

        p = self.pattern
        return sp.csr_matrix((self.values.cpu().numpy(), p.indices.cpu().numpy(),
                              p.indptr.cpu().numpy()), shape=(self.nrow, self.ncol))


class MatrixFreeJacobian:
    """The Jacobian ``A(m)`` applied from the quadrature data of a point, with its
    elimination (``apply_ij_at`` for the (ADJOINT, STATE) pair).  Keeps the operator's
    data (D of the point in the layout the operator streams, plus its scratch); applies
    that share one instance must run in one stream."""

    def __init__(self, mesh, quad, ess_marker, precision=_lib.HM_FP64, stream=None,
                 quad_precision=None):
        self.mesh, self.ess, self.precision = mesh, ess_marker, precision
        qp = precision if quad_precision is None else quad_precision
        self.nrow = self.ncol = mesh.ndof
        nbytes = lib.hm_lattice_jacobian_bytes(mesh.handle, precision)
        self.jac = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device=mesh.device)
        check(lib.hm_lattice_jacobian_prepare(mesh.handle, ptr(quad), qp, ptr(self.jac), precision,
                                              stream_ptr(stream)), "hm_lattice_jacobian_prepare")
        # the diagonal (Jacobi) is taken now, so the point's quadrature data need not be kept
        self._diag = torch.empty(self.nrow, dtype=torch.float64, device=mesh.device)
        check(lib.hm_lattice_diag_A(mesh.handle, ptr(quad), qp, ptr(ess_marker),
                                    ptr(self._diag), stream_ptr(stream)), "hm_lattice_diag_A")

    def mult(self, x, y, stream=None):
        check(lib.hm_lattice_apply_A(self.mesh.handle, ptr(self.jac), self.precision,
                                     ptr(self.ess), ptr(x), ptr(y), stream_ptr(stream)),
              "hm_lattice_apply_A")
        return y

    Mult = mult
    # the Jacobian of this density is symmetric (A^T = A)
    mult_transpose = MultTranspose = mult

    def diagonal(self, out=None, stream=None):
        if out is None:
            return self._diag.clone()
        out.copy_(self._diag)
        return out


class PCGResult:
    __slots__ = ("iterations", "relres", "converged")

    def __init__(self, iterations, relres, converged):
        self.iterations, self.relres, self.converged = iterations, relres, converged

    def __repr__(self):
        return "PCGResult(iterations=%d, relres=%.3e, converged=%s)" % (
            self.iterations, self.relres, self.converged)


class PCGSolver:
    """Jacobi-PCG for ``A x = b``, FP64 throughout, on the device.

    ``operator`` is a ``CSRBlock`` or a ``MatrixFreeJacobian``; the workspace and the
    diagonal are allocated once and kept (the reference keeps its solver objects and
    AMG hierarchies per operator the same way)."""

    def __init__(self, operator, rel_tolerance=1e-12, max_iter=20000, check_every=16,
                 raise_on_fail=True):
        self.parameters = {"rel_tolerance": float(rel_tolerance), "max_iter": int(max_iter),
                           "check_every": int(check_every)}
        self.raise_on_fail = raise_on_fail
        self.last = None
        self.set_operator(operator)

    def set_operator(self, operator):
        self.op = operator
        n = operator.nrow
        dev = (operator.values.device if isinstance(operator, CSRBlock)
               else operator.mesh.device)
        self.diag = operator.diagonal()
        nbytes = lib.hm_pcg_workspace_bytes(n)
        self.work = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device=dev)
        return self

    def solve(self, x, b, stream=None):
        op = self.op
        it, rr = ctypes.c_int(), ctypes.c_double()
        prm = self.parameters
        if isinstance(op, CSRBlock):
            p = op.pattern
            args = (ptr(p.indptr), ptr(p.indices), ptr(op.values), None, None, _lib.HM_FP64, None)
        else:
            args = (None, None, None, op.mesh.handle, ptr(op.jac), op.precision, ptr(op.ess))
        rc = lib.hm_pcg(op.nrow, *args, ptr(self.diag), ptr(b), ptr(x),
                        prm["rel_tolerance"], prm["max_iter"], prm["check_every"], ptr(self.work),
                        ctypes.byref(it), ctypes.byref(rr), stream_ptr(stream))
        self.last = PCGResult(it.value, rr.value, rc == _lib.HM_OK)
        if rc == _lib.HM_ERR_NOCONV and not self.raise_on_fail:
            return x
        check(rc, "hm_pcg")
        return x


class MixedPCGSolver:
    """Mixed-precision solve of ``A x = b`` with the lattice's matrix-free Jacobian:
    conjugate gradients whose recurrence runs in FP32, re-anchored to the FP64 true
    residual whenever it has fallen by ``reliable_delta`` (``hm_pcg_mixed``).  It takes
    the place of the reference's refined single-precision solves
    (modeling/PDEVariationalProblem.py:1220-1329) with the same goal and stall rule.
    ``operator`` is the FP64 ``MatrixFreeJacobian``; the FP32 operator is derived from
    the same point."""

    def __init__(self, operator, quad, rel_tolerance=1e-12, reliable_delta=0.1,
                 max_updates=200, max_iter=20000, check_every=16, raise_on_fail=True):
        if not isinstance(operator, MatrixFreeJacobian):
            raise TypeError("the mixed-precision solve needs the matrix-free Jacobian")
        self.op = operator
        self.op32 = MatrixFreeJacobian(operator.mesh, quad, operator.ess, _lib.HM_FP32,
                                       quad_precision=operator.precision)
        self.parameters = {"rel_tolerance": float(rel_tolerance),
                           "reliable_delta": float(reliable_delta),
                           "max_updates": int(max_updates), "max_iter": int(max_iter),
                           "check_every": int(check_every)}
        self.raise_on_fail = raise_on_fail
        self.diag = operator.diagonal()
        nbytes = lib.hm_pcg_mixed_workspace_bytes(operator.nrow)
        self.work = torch.empty((nbytes + 7) // 8, dtype=torch.float64,
                                device=operator.mesh.device)
        self.last = None
        self.last_updates = 0

    def solve(self, x, b, stream=None):
        op, prm = self.op, self.parameters
        it, nup, rr = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        rc = lib.hm_pcg_mixed(op.mesh.handle, ptr(op.jac), ptr(self.op32.jac), ptr(op.ess),
                              ptr(self.diag), ptr(b), ptr(x), prm["rel_tolerance"],
                              prm["reliable_delta"], prm["max_updates"], prm["max_iter"],
                              prm["check_every"], ptr(self.work), ctypes.byref(it),
                              ctypes.byref(nup), ctypes.byref(rr), stream_ptr(stream))
        self.last = PCGResult(it.value, rr.value, rc == _lib.HM_OK)
        self.last_updates = nup.value
        if rc == _lib.HM_ERR_NOCONV and not self.raise_on_fail:
            return x
        check(rc, "hm_pcg_mixed")
        return x


class SolvePlan:
    """A resident solve workspace for one lattice and its Dirichlet nodes
    (``hm_pcg_plan_*``): the operator storage of a point (FP64, plus FP32 for the
    mixed-precision solve), the Jacobi diagonal, fixed right-hand side and solution
    buffers and the PCG workspace.  ``set_point`` loads a point's quadrature data;
    ``solve`` copies the right-hand side in, solves from zero and copies the solution
    out.  Solves in a stream other than the legacy default stream replay a CUDA graph of
    each batch of ``check_every`` iterations, captured on first use.  One host thread at
    a time; the reference keeps its solver objects per operator the same way."""

    def __init__(self, mesh, ess_marker, precision="fp64", rel_tolerance=1e-8, max_iter=20000,
                 check_every=16, reliable_delta=0.1, max_updates=200, multigrid=False):
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.mesh, self.ess, self.precision = mesh, ess_marker, precision
        self.parameters = {"rel_tolerance": float(rel_tolerance), "max_iter": int(max_iter),
                           "check_every": int(check_every), "reliable_delta": float(reliable_delta),
                           "max_updates": int(max_updates)}
        dev, n, h = mesh.device, mesh.ndof, mesh.handle

        def buf(nbytes):
            return torch.empty((int(nbytes) + 7) // 8, dtype=torch.float64, device=dev)

        self.jac64 = buf(lib.hm_lattice_jacobian_bytes(h, _lib.HM_FP64))
        self.jac32 = (buf(lib.hm_lattice_jacobian_bytes(h, _lib.HM_FP32))
                      if precision == "mixed" else None)
        self.diag = torch.empty(n, dtype=torch.float64, device=dev)
        self.b = torch.zeros(n, dtype=torch.float64, device=dev)
        self.x = torch.zeros(n, dtype=torch.float64, device=dev)
        self.work = buf(lib.hm_pcg_mixed_workspace_bytes(n) if precision == "mixed"
                        else lib.hm_pcg_workspace_bytes(n))
        self.nbytes = sum(t.numel() * 8 for t in (self.jac64, self.jac32, self.diag, self.b,
                                                  self.x, self.work) if t is not None)
        self._plan = ctypes.c_void_p()
        check(lib.hm_pcg_plan_create(h, ptr(self.jac64), ptr(self.jac32), ptr(ess_marker),
                                     ptr(self.diag), ptr(self.b), ptr(self.x), ptr(self.work),
                                     int(check_every), ctypes.byref(self._plan)),
              "hm_pcg_plan_create")
        self.last = None
        self.last_updates = 0
        self.mg = None
        if multigrid:
            if precision != "fp64":
                raise ValueError("the multigrid plan is FP64")
            self.mg = Multigrid(mesh)
            self.nbytes += self.mg.work.numel() * 8
            check(lib.hm_pcg_plan_set_mg(self._plan, self.mg._mg), "hm_pcg_plan_set_mg")

    def set_point(self, quad, stream=None):
        """Load the operator of a point from its FP64 quadrature data."""
        h, sp = self.mesh.handle, stream_ptr(stream)
        check(lib.hm_lattice_jacobian_prepare(h, ptr(quad), _lib.HM_FP64, ptr(self.jac64),
                                              _lib.HM_FP64, sp), "hm_lattice_jacobian_prepare")
        if self.jac32 is not None:
            check(lib.hm_lattice_jacobian_prepare(h, ptr(quad), _lib.HM_FP64, ptr(self.jac32),
                                                  _lib.HM_FP32, sp), "hm_lattice_jacobian_prepare")
        check(lib.hm_lattice_diag_A(h, ptr(quad), _lib.HM_FP64, ptr(self.ess), ptr(self.diag), sp),
              "hm_lattice_diag_A")
        if self.mg is not None:
            self.mg.setup(self.jac64, self.ess, self.diag, stream)
        return self

    def solve(self, out, rhs, stream=None):
        """``out = A^{-1} rhs`` (rhs zero on the Dirichlet nodes)."""
        prm = self.parameters
        if rhs is not self.b:
            self.b.copy_(rhs)
        it, nup, rr = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        rc = lib.hm_pcg_plan_solve(self._plan, prm["rel_tolerance"], prm["reliable_delta"],
                                   prm["max_updates"], prm["max_iter"], ctypes.byref(it),
                                   ctypes.byref(nup), ctypes.byref(rr), stream_ptr(stream))
        self.last = PCGResult(it.value, rr.value, rc == _lib.HM_OK)
        self.last_updates = nup.value
        check(rc, "hm_pcg_plan_solve")
        if out is not None and out is not self.x:
            out.copy_(self.x)
        return out

    def close(self):
        if self._plan:
            lib.hm_pcg_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()
        if getattr(self, "mg", None) is not None:
            self.mg.close()

    def __del__(self):
        try:
            self.close()
        except Exception:                                   # noqa: BLE001
            pass


class SolveGroup:
    """Several FP64 ``SolvePlan``s of one lattice size solved together
    (``hm_pcg_group_*``): each full batch of iterations of all plans is one CUDA graph,
    one branch per plan, and one host synchronisation per batch checks them all.  Every
    solution is bit for bit the plan's own solve's.  The plans' tolerances and iteration
    limits are taken from the first plan."""

    def __init__(self, plans):
        if not plans:
            raise ValueError("a solve group needs at least one plan")
        if any(p.jac32 is not None for p in plans):
            raise ValueError("solve groups take FP64 plans")
        self.plans = list(plans)
        arr = (ctypes.c_void_p * len(plans))(*[p._plan.value for p in plans])
        self._g = ctypes.c_void_p()
        check(lib.hm_pcg_group_create(arr, len(plans), ctypes.byref(self._g)),
              "hm_pcg_group_create")
        self.last = None

    def solve(self, outs, rhss, stream=None):
        """``outs[i] = A_i^{-1} rhss[i]`` for plan i (right-hand sides zero on the
        Dirichlet nodes); returns the per-plan ``PCGResult``s."""
        k = len(self.plans)
        if len(outs) != k or len(rhss) != k:
            raise ValueError("one right-hand side and one output per plan")
        for p, rhs in zip(self.plans, rhss):
            if rhs is not p.b:
                p.b.copy_(rhs)
        prm = self.plans[0].parameters
        its = (ctypes.c_int * k)()
        rr = (ctypes.c_double * k)()
        rc = lib.hm_pcg_group_solve(self._g, prm["rel_tolerance"], prm["max_iter"], its, rr,
                                    stream_ptr(stream))
        self.last = [PCGResult(its[i], rr[i], rc == _lib.HM_OK) for i in range(k)]
        for i, p in enumerate(self.plans):
            p.last = self.last[i]
        check(rc, "hm_pcg_group_solve")
        for p, out in zip(self.plans, outs):
            if out is not None and out is not p.x:
                out.copy_(p.x)
        return self.last

    def close(self):
        if self._g:
            lib.hm_pcg_group_destroy(self._g)
            self._g = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:                                   # noqa: BLE001
            pass


def default_smoothing_degree(mesh):
    """Chebyshev degree of the smoother when the caller gives none: 1 from a million dofs
    up, 2 below.  Measured on a B200 (FP64 multigrid-PCG to rtol 1e-12): at 64^3 degree 1
    takes 12 iterations and 7.3 ms against 8 and 7.9 ms (45 against 58 iterations, 33.5
    against 42.3 ms at sigma 1); at 32^3, where a cycle's launches dominate, degree 2 is
    faster (2.1 against 2.6 ms)."""
    return 1 if mesh.ndof >= 1_000_000 else 2


MG_PRECISIONS = ("fp64", "fp32")


class Multigrid:
    """The lattice Jacobian's geometric multigrid V-cycle (``hm_mg_*``): hierarchy and
    level storage on one workspace; ``setup`` loads a point's FP64 operator data (again
    whenever the point changes); ``apply(r, z)`` is ``z = V(r)``.  ``precision="fp32"``
    runs the cycle on single-precision copies of the level data (formed at every set-up;
    ``r`` and ``z`` stay FP64): a preconditioner of the FP64 CG, which keeps the solve's
    accuracy."""

    def __init__(self, mesh, degree=None, coarse_degree=24, precision="fp64"):
        if degree is None:
            degree = default_smoothing_degree(mesh)
        self.mesh = mesh
        nbytes = lib.hm_mg_workspace_bytes(mesh.handle)
        self.work = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device=mesh.device)
        self.work32 = None
        self.precision = "fp64"
        self._mg = ctypes.c_void_p()
        check(lib.hm_mg_create(mesh.handle, ptr(self.work), int(degree), int(coarse_degree),
                               ctypes.byref(self._mg)), "hm_mg_create")
        self.levels = lib.hm_mg_levels(self._mg)
        self.set_precision(precision)

    @staticmethod
    def workspace_bytes(mesh, precision="fp64"):
        """Device bytes of a V-cycle's storage in ``precision``."""
        nbytes = lib.hm_mg_workspace_bytes(mesh.handle)
        if precision == "fp32":
            nbytes += lib.hm_mg_single_workspace_bytes(mesh.handle)
        return nbytes

    def set_precision(self, precision, stream=None):
        """The cycle in ``"fp64"`` or ``"fp32"``; after a set-up the FP32 copies are
        formed at once (on ``stream``)."""
        if precision not in MG_PRECISIONS:
            raise ValueError("the multigrid precision must be one of %s" % (MG_PRECISIONS,))
        if precision == "fp32":
            if self.work32 is None:
                nbytes = lib.hm_mg_single_workspace_bytes(self.mesh.handle)
                self.work32 = torch.empty((nbytes + 3) // 4, dtype=torch.float32,
                                          device=self.mesh.device)
            check(lib.hm_mg_set_single(self._mg, ptr(self.work32), stream_ptr(stream)),
                  "hm_mg_set_single")
        else:
            check(lib.hm_mg_set_single(self._mg, None, stream_ptr(stream)), "hm_mg_set_single")
        self.precision = precision
        return self

    def setup(self, jac64, ess, diag, stream=None):
        check(lib.hm_mg_setup(self._mg, ptr(jac64), ptr(ess), ptr(diag), stream_ptr(stream)),
              "hm_mg_setup")
        return self

    def apply(self, r, z, stream=None):
        check(lib.hm_mg_apply(self._mg, ptr(r), ptr(z), stream_ptr(stream)), "hm_mg_apply")
        return z

    def set_tail_nodes(self, max_nodes):
        """Levels of at most ``max_nodes`` nodes run as one CTA-wide kernel (0: none)."""
        check(lib.hm_mg_set_tail_nodes(self._mg, int(max_nodes)), "hm_mg_set_tail_nodes")
        return self

    def set_fused(self, fused):
        """Degree-1 smoothing steps fused with their operator pass (the default), or
        launched step by step; the same arithmetic either way."""
        check(lib.hm_mg_set_fused(self._mg, int(bool(fused))), "hm_mg_set_fused")
        return self

    def close(self):
        if self._mg:
            lib.hm_mg_destroy(self._mg)
            self._mg = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:                                   # noqa: BLE001
            pass


class MGPCGSolver:
    """PCG for ``A x = b`` with the matrix-free FP64 Jacobian, preconditioned by the
    geometric multigrid V-cycle -- in place of the reference's BoomerAMG-preconditioned
    hypre PCG (algorithms/linSolvers.py:243-828, 709).  It runs as a solve plan on the
    operator's own storage (``hm_pcg_plan_*`` with ``hm_pcg_plan_set_mg``): in a stream
    other than the legacy default stream every batch of iterations, V-cycles included,
    replays a captured CUDA graph.  ``x`` is overwritten (the solve starts from zero).
    ``mg_precision="fp32"`` runs the V-cycle in single precision; the CG recurrence, its
    inner products and the stopping test stay FP64, so the tolerance means the same.  The
    FP32 cycle's rounding is relative to the smooth part of its correction, so at high
    contrast (condition numbers near 1e7) it can stop carrying the solve: a solve with it
    that stalls, or whose FP64 true residual ends above ten times the tolerance, is solved
    again with the FP64 cycle, which the solver keeps from then on (``fallbacks`` counts
    them), as the reference finishes a refined solve in double (``_solve_in_double``,
    modeling/PDEVariationalProblem.py:1331)."""

    def __init__(self, operator, rel_tolerance=1e-12, max_iter=2000, check_every=4,
                 degree=None, coarse_degree=24, raise_on_fail=True, mg_precision="fp64"):
        if not isinstance(operator, MatrixFreeJacobian) or operator.precision != _lib.HM_FP64:
            raise TypeError("the multigrid solve needs the FP64 matrix-free Jacobian")
        self.op = operator
        self.parameters = {"rel_tolerance": float(rel_tolerance), "max_iter": int(max_iter),
                           "check_every": int(check_every)}
        self.raise_on_fail = raise_on_fail
        mesh = operator.mesh
        self.mg = Multigrid(mesh, degree, coarse_degree, precision=mg_precision)
        self.mg.setup(operator.jac, operator.ess, operator._diag)
        n = operator.nrow
        self.b = torch.zeros(n, dtype=torch.float64, device=mesh.device)
        self.x = torch.zeros(n, dtype=torch.float64, device=mesh.device)
        nbytes = lib.hm_pcg_workspace_bytes(n)
        self.work = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device=mesh.device)
        self._plan = ctypes.c_void_p()
        self._make_plan()
        self._y = None
        self.fallbacks = 0
        self.last = None

    def _make_plan(self):
        """A solve plan on the operator's storage with this solver's V-cycle (again after
        the cycle's precision changes: a plan keeps the launches it captured)."""
        if self._plan:
            lib.hm_pcg_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()
        op = self.op
        check(lib.hm_pcg_plan_create(op.mesh.handle, ptr(op.jac), None, ptr(op.ess), ptr(op._diag),
                                     ptr(self.b), ptr(self.x), ptr(self.work),
                                     self.parameters["check_every"], ctypes.byref(self._plan)),
              "hm_pcg_plan_create")
        check(lib.hm_pcg_plan_set_mg(self._plan, self.mg._mg), "hm_pcg_plan_set_mg")

    def _run(self, stream):
        prm = self.parameters
        it, nup, rr = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        rc = lib.hm_pcg_plan_solve(self._plan, prm["rel_tolerance"], 0.1, 1, prm["max_iter"],
                                   ctypes.byref(it), ctypes.byref(nup), ctypes.byref(rr),
                                   stream_ptr(stream))
        self.last = PCGResult(it.value, rr.value, rc == _lib.HM_OK)
        return rc

    def _carried(self, stream):
        """The FP64 true residual of the FP32-cycle solve within ten times the tolerance."""
        if self._y is None:
            self._y = torch.empty_like(self.x)
        with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
            self.op.mult(self.x, self._y)
            self._y.sub_(self.b)
            res, bnorm = torch.stack((self._y.norm(), self.b.norm())).tolist()   # one read
        return res <= 10.0 * self.parameters["rel_tolerance"] * bnorm

    def solve(self, x, b, stream=None):
        self.b.copy_(b)
        rc = self._run(stream)
        if self.mg.precision == "fp32" and rc in (_lib.HM_OK, _lib.HM_ERR_NOCONV) and (
                rc != _lib.HM_OK or not self._carried(stream)):
            self.mg.set_precision("fp64", stream)
            self.mg.work32 = None
            self._make_plan()
            self.fallbacks += 1
            rc = self._run(stream)
        if rc == _lib.HM_ERR_NOCONV and not self.raise_on_fail:
            x.copy_(self.x)
            return x
        check(rc, "hm_pcg_plan_solve")
        x.copy_(self.x)
        return x

    def __del__(self):
        try:
            if self._plan:
                lib.hm_pcg_plan_destroy(self._plan)
                self._plan = ctypes.c_void_p()
        except Exception:                                   # noqa: BLE001
            pass
