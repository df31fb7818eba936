"""The forward problem of the log-conductivity diffusion density on the Q2 lattice.

Keeps the reference's problem/form API -- method names, slot indices, the essential-dof
policy per block and the exception types -- so that callers of
``hippymfem.modeling.PDEVariationalProblem`` (modeling/PDEVariationalProblem.py:127-2016)
can switch.  The density is fixed to ``exp(m) grad u . grad p - f p``
(benchmarks/bench_newton_device.py:392 with a constant source ``f``); every derivative
the reference takes by JAX AD is a hand-written CUDA kernel here:

* quadrature data of a point (``hm_lattice_quadrature``): what ``_eval_field`` and the
  pointwise derivatives of the quadrature route compute (hippymfem/fem/kernel.py:378-394,
  1431-1485);
* one fused, write-once assembly (``hm_lattice_assemble``) for every block of a
  linearization point and the assembled vectors, in place of ``element_matrices_many``
  + ``scatter_many`` (kernel.py:2048, hippymfem/fem/csrassemble.py:286);
* the incremental solves by an FP64 Jacobi-PCG on the device (``hm_pcg``).

Vectors are FP64 CUDA tensors of the lattice's dof count (one rank: local = true dofs).
"""

import ctypes

import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr
from .mesh import DirichletBC
from .pattern import LatticePattern
from .sparse import CSRBlock, MatrixFreeJacobian, MGPCGSolver, MixedPCGSolver, PCGSolver

STATE, PARAMETER, ADJOINT = 0, 1, 2
NVAR = 3

_BLOCKS = {(ADJOINT, STATE): "A", (ADJOINT, PARAMETER): "C", (STATE, PARAMETER): "Wum",
           (PARAMETER, PARAMETER): "Wmm"}


class _Snapshot:
    """A copy of a vector, to recognise it again by its values (object identity and
    storage addresses are reused once a tensor is freed)."""

    __slots__ = ("t",)

    def __init__(self, t):
        self.t = None if t is None else t.detach().clone()

    def matches(self, t):
        if self.t is None or t is None:
            return self.t is None and t is None
        return self.t.shape == t.shape and bool(torch.equal(self.t, t))


class PDEVariationalProblem:
    """Stationary forward problem ``-div(e^m grad u) = f`` on a Q2 ``BoxMesh``.

    Parameters
    ----------
    Vh : sequence of 3 ``Q2Space`` on one mesh, ``[STATE, PARAMETER, ADJOINT]``.
    f : constant source.
    bc, bc0 : ``DirichletBC`` (homogeneous; ``bc0`` defaults to ``bc``).
    is_fwd_linear : the density is linear in ``u``; ``W_uu`` is never assembled.
    solver_tolerance : relative tolerance of the forward, adjoint and incremental
        solves (the reference's ``KrylovSolver`` default is 1e-12,
        hippymfem/algorithms/linSolvers.py:65).
    matrix_free_solves : solve with the lattice's matrix-free Jacobian instead of the
        assembled ``A`` (same operator, no SpMV over 135 M nonzeros at 64^3).
    check_finite : read the device status word after each assembly and raise
        ``RuntimeError`` on non-finite values (``require_finite_arrays``,
        modeling/PDEVariationalProblem.py:1844-1892); one synchronisation each.
    preconditioner : ``"jacobi"`` or ``"mg"`` (the lattice's geometric multigrid V-cycle,
        in place of the reference's BoomerAMG; FP64 matrix-free solves, Dirichlet nodes
        on the whole boundary).
    solver_precision : ``"fp64"``, or ``"mixed"``: with ``"jacobi"``, PCG whose
        recurrence runs in FP32 with the FP32 matrix-free operator, re-anchored to the
        FP64 true residual each time it falls by ``reliable_delta``, to the same
        tolerance (in place of the reference's ``_refined_solve``, :1220-1329); with
        ``"mg"``, the FP64 CG preconditioned by the V-cycle run in FP32.  Implies
        ``matrix_free_solves``.
    """

    def __init__(self, Vh, f=1.0, bc=None, bc0=None, is_fwd_linear=True, solver_tolerance=1e-12,
                 matrix_free_solves=False, check_finite=True, max_iter=50000,
                 solver_precision="fp64", reliable_delta=0.1, preconditioner="jacobi"):
        if len(Vh) != NVAR:
            raise ValueError("Vh must have %d entries" % NVAR)
        self.Vh = list(Vh)
        self.mesh = Vh[STATE].mesh
        if any(V.mesh is not self.mesh for V in self.Vh):
            raise ValueError("all three spaces must live on one mesh")
        self.f = float(f)
        self.bc = bc if bc is not None else DirichletBC(Vh[STATE])
        self.bc0 = bc0 if bc0 is not None else self.bc
        self.is_fwd_linear = bool(is_fwd_linear)
        if not self.is_fwd_linear:
            raise NotImplementedError("the log-conductivity density is linear in the state")
        self.solver_tolerance = float(solver_tolerance)
        if solver_precision not in ("fp64", "mixed"):
            raise ValueError("solver_precision must be 'fp64' or 'mixed'")
        self.solver_precision = solver_precision
        self.reliable_delta = float(reliable_delta)
        if preconditioner not in ("jacobi", "mg"):
            raise ValueError("preconditioner must be 'jacobi' or 'mg'")
        self.preconditioner = preconditioner
        self.matrix_free_solves = (bool(matrix_free_solves) or solver_precision == "mixed"
                                   or preconditioner == "mg")
        self.check_finite = bool(check_finite)
        self.max_iter = int(max_iter)
        self.precision = _lib.HM_FP64
        self._pattern = None
        self._status = torch.zeros(1, dtype=torch.int32, device=self.mesh.device)
        self._quad = {}
        self._dir_cache = None
        self._jac_cache = None
        self.A = self.At = self.C = self.Wuu = self.Wum = self.Wmm = self.Ct = self.Wmu = None
        self._lin_point = None
        self._lin_vectors = None
        self._same_word = None
        self.gauss_newton_approx = False
        self.solver = self.solver_fwd_inc = self.solver_adj_inc = None
        self.n_calls = {"forward": 0, "adjoint": 0, "incremental_forward": 0,
                        "incremental_adjoint": 0}
        self.last_solve = None

    # ----------------------------------------------------------------- vectors
    def generate_state(self):
        return self.Vh[STATE].vector()

    def generate_parameter(self):
        return self.Vh[PARAMETER].vector()

    def generate_adjoint(self):
        return self.Vh[ADJOINT].vector()

    def init_parameter(self, m):
        return m

    @property
    def pattern(self):
        if self._pattern is None:
            self._pattern = LatticePattern(self.mesh)
        return self._pattern

    # ------------------------------------------------------------- quadrature
    def _locals(self, x):
        out = []
        for i in range(NVAR):
            v = x[i] if i < len(x) and x[i] is not None else None
            out.append(v if v is not None else self.Vh[i].vector())
        return out

    def _quadrature(self, x, slot="point", mhat=None):
        """Quadrature data of ``x`` into the buffer named ``slot`` (kept for reuse); with
        ``mhat`` the data of the directional derivative along ``mhat``."""
        u, m, p = self._locals(x)
        nbytes = self.mesh.quad_bytes(self.precision)
        buf = self._quad.get(slot)
        if buf is None or buf.numel() * 8 < nbytes:
            buf = self._quad[slot] = torch.empty((nbytes + 7) // 8, dtype=torch.float64,
                                                 device=self.mesh.device)
        if self.check_finite:
            self._status.zero_()
        if mhat is None:
            check(lib.hm_lattice_quadrature(self.mesh.handle, ptr(u), ptr(m), ptr(p),
                                            self.precision, ptr(buf), ptr(self._status),
                                            stream_ptr()), "hm_lattice_quadrature")
        else:
            check(lib.hm_lattice_quadrature_dir(self.mesh.handle, ptr(u), ptr(m), ptr(p),
                                                ptr(mhat), self.precision, ptr(buf),
                                                ptr(self._status), stream_ptr()),
                  "hm_lattice_quadrature_dir")
        return buf

    def _direct_vectors(self, x, slots, f=None, mhat=None, zero_ess=False):
        """The assembled vectors of ``slots`` at ``x`` (``hm_lattice_vectors``: straight
        from the fields, no pointwise-data workspace); with ``mhat`` the second-order
        products along it (no source)."""
        u, m, p = self._locals(x)
        n = len(slots)
        need = lib.hm_lattice_vectors_workspace_bytes(self.mesh.handle, n)
        buf = self._quad.get("vectors")
        if buf is None or buf.numel() * 8 < need:
            buf = self._quad["vectors"] = torch.empty((need + 7) // 8, dtype=torch.float64,
                                                      device=self.mesh.device)
        vecs = {s_: self.Vh[s_].vector() for s_ in slots}
        if self.check_finite:
            self._status.zero_()
        check(lib.hm_lattice_vectors(
            self.mesh.handle, ptr(u), ptr(m), ptr(p), ptr(mhat),
            0.0 if mhat is not None else (self.f if f is None else float(f)),
            ptr(self.bc0.marker), ptr(vecs.get(STATE)), ptr(vecs.get(PARAMETER)),
            ptr(vecs.get(ADJOINT)), int(bool(zero_ess)), ptr(buf), ptr(self._status),
            stream_ptr()), "hm_lattice_vectors")
        return vecs

    def _require_finite(self, what):
        if self.check_finite and int(self._status.item()) & _lib.HM_STATUS_NONFINITE:
            raise RuntimeError("non-finite values in %s" % what)

    def _assemble(self, quad, blocks=(), vectors=(), zero_ess_vectors=False, f=None):
        """One fused launch: the CSR values of ``blocks`` (names of ``_BLOCKS``) and the
        assembled vectors of the slots in ``vectors`` (source ``f``: the problem's)."""
        pat = self.pattern if blocks else None
        vals = {b: pat.new_values() for b in blocks}
        vecs = {s: self.Vh[s].vector() for s in vectors}
        check(lib.hm_lattice_assemble(
            self.mesh.handle, ptr(quad), self.precision,
            ptr(pat.indptr) if pat is not None else None, ptr(self.bc0.marker),
            self.f if f is None else float(f),
            ptr(vals.get("A")), ptr(vals.get("C")), ptr(vals.get("Wum")), ptr(vals.get("Wmm")),
            ptr(vecs.get(STATE)), ptr(vecs.get(PARAMETER)), ptr(vecs.get(ADJOINT)),
            int(bool(zero_ess_vectors)), stream_ptr()), "hm_lattice_assemble")
        return {b: CSRBlock(pat, v) for b, v in vals.items()}, vecs

    # ------------------------------------------------------------ assembly
    def _residual(self, x, var=ADJOINT, ess=None):
        """``dR/d(var)`` at ``x`` (modeling/PDEVariationalProblem.py:423), essential
        entries of ``ess`` zeroed."""
        cached = self._lin_vectors.get(var) if self._lin_vectors else None
        if cached is not None and not self.check_finite and self._point_complete(x):
            # the point's vector where x is the point, else from the fields: decided on
            # the device, without waiting for it
            out = self._vectors_at(x, var, cached)
        elif cached is not None and self._at_linearization_point(x):
            out = cached.clone()
        else:
            vecs = self._direct_vectors(x, (var,))
            self._require_finite("the residual")
            out = vecs[var]
        if ess is not None and len(ess):
            out.masked_fill_(self.mesh.ess_marker(ess).bool(), 0.0)
        return out

    def _point_complete(self, x):
        loc = self._locals(x)
        return (self._lin_point is not None and all(v is not None for v in loc)
                and all(v is not None for v in self._lin_point)
                and all(a.shape == b.shape for a, b in zip(loc, self._lin_point)))

    def _vectors_at(self, x, var, kept):
        """``hm_lattice_vectors_at``: the kept vector of slot ``var`` where ``x`` equals
        the linearization point value for value, else the vector from the fields."""
        u, m, p = self._locals(x)
        u0, m0, p0 = self._lin_point
        need = lib.hm_lattice_vectors_workspace_bytes(self.mesh.handle, 1)
        buf = self._quad.get("vectors")
        if buf is None or buf.numel() * 8 < need:
            buf = self._quad["vectors"] = torch.empty((need + 7) // 8, dtype=torch.float64,
                                                      device=self.mesh.device)
        if self._same_word is None:
            self._same_word = torch.zeros(1, dtype=torch.int32, device=self.mesh.device)
        out = self.Vh[var].vector()
        kept_s = kept if var == STATE else None
        kept_m = kept if var == PARAMETER else None
        kept_a = kept if var == ADJOINT else None
        check(lib.hm_lattice_vectors_at(
            self.mesh.handle, ptr(u), ptr(m), ptr(p), ptr(u0), ptr(m0), ptr(p0),
            ptr(kept_s), ptr(kept_m), ptr(kept_a), float(self.f),
            ptr(out) if var == STATE else None, ptr(out) if var == PARAMETER else None,
            ptr(out) if var == ADJOINT else None, ptr(buf), ptr(self._same_word),
            ptr(self._status), stream_ptr()), "hm_lattice_vectors_at")
        return out

    def _at_linearization_point(self, x):
        """``x`` holds the values of the current linearization point (compared on the
        device, value for value)."""
        if self._lin_point is None:
            return False
        for a, b in zip(self._locals(x), self._lin_point):
            if (a is None) != (b is None):
                return False
            if a is not None and not (a.shape == b.shape and bool(torch.equal(a, b))):
                return False
        return True

    def _block(self, i, j, x):
        """Block ``(i, j)`` at ``x`` with its elimination policy (``_block``, :448)."""
        name = _BLOCKS.get((i, j))
        if name is None:
            raise ValueError("no assembled block (%d, %d) for this density" % (i, j))
        quad = self._quadrature(x, "block")
        blocks, _ = self._assemble(quad, blocks=(name,))
        self._require_finite("block (%d, %d)" % (i, j))
        return blocks[name]

    def _jacobian(self, x):
        """The assembled Jacobian ``A`` and its transpose (``A`` itself: the density is
        symmetric in u and p), reused while ``m`` has not moved (:542)."""
        m = x[PARAMETER]
        if self._jac_cache is not None and self._jac_cache[0].matches(m):
            return self._jac_cache[1], self._jac_cache[1]
        quad = self._quadrature([None, m, None], "jacobian")
        A = self._make_jacobian(quad)
        self._jac_cache = (_Snapshot(m), A, quad)
        self.solver = None
        return A, A

    def _make_jacobian(self, quad):
        if self.matrix_free_solves:
            # the matrix-free operator keeps its own copy of the point's data
            self._require_finite("the Jacobian")
            return MatrixFreeJacobian(self.mesh, quad, self.bc0.marker, self.precision)
        blocks, _ = self._assemble(quad, blocks=("A",))
        self._require_finite("the Jacobian")
        return blocks["A"]

    def _get_solver(self, A):
        if self.preconditioner == "mg":
            mgp = "fp32" if self.solver_precision == "mixed" else "fp64"
            return MGPCGSolver(A, rel_tolerance=self.solver_tolerance, max_iter=self.max_iter,
                               mg_precision=mgp)
        if self.solver_precision == "mixed":
            return MixedPCGSolver(A, self._jac_cache[2], rel_tolerance=self.solver_tolerance,
                                  reliable_delta=self.reliable_delta, max_iter=self.max_iter)
        return PCGSolver(A, rel_tolerance=self.solver_tolerance, max_iter=self.max_iter)

    # ---------------------------------------------------------------- solves
    def solveFwd(self, out, x):
        """One Newton step from the boundary data: exact for a linear problem (:1046)."""
        self.n_calls["forward"] += 1
        A, _ = self._jacobian(x)
        u0 = self.Vh[STATE].vector()
        r = self._residual([u0, x[PARAMETER], None], ADJOINT, self.bc.ess_tdof)
        if self.solver is None or self.solver.op is not A:
            self.solver = self._get_solver(A)
        du = self.Vh[STATE].vector()
        r.neg_()
        self.solver.solve(du, r)
        self.last_solve = self.solver.last
        out.copy_(u0 + du)
        return out

    def solveAdj(self, out, x, adj_rhs):
        """``A^T p = adj_rhs`` with the homogeneous condition (:1171)."""
        self.n_calls["adjoint"] += 1
        A, At = self._jacobian(x)
        if self.solver is None or self.solver.op is not A:
            self.solver = self._get_solver(A)
        rhs = adj_rhs.clone()
        self.bc0.zero(rhs)
        out.zero_()
        self.solver.solve(out, rhs)
        self.last_solve = self.solver.last
        return out

    def evalGradientParameter(self, x, out):
        """``out = dR/dm`` at ``x``; equals ``C^T p`` but needs no matrix (:1365)."""
        out.copy_(self._residual(x, PARAMETER))
        return out

    # ------------------------------------------------------ linearization point
    def setLinearizationPoint(self, x, gauss_newton_approx=False, matrix_free=False):
        """Assemble the blocks of the incremental solves and the Hessian (:1372) in one
        fused pass: ``C`` always, ``W_um`` and ``W_mm`` unless Gauss-Newton, ``A`` when
        ``m`` moved; ``W_uu`` is zero for this density and never formed.  With
        ``matrix_free`` only the quadrature data is kept and every product is taken
        from it (``apply_ij_at``)."""
        self._lin_point = [v.clone() if v is not None else None for v in self._locals(x)]
        self._lin_vectors = None
        self.C = self.Wuu = self.Wum = self.Wmm = self.Ct = self.Wmu = None
        self.gauss_newton_approx = bool(gauss_newton_approx)
        self._mf = bool(matrix_free)
        m = x[PARAMETER]
        need_A = self._jac_cache is None or not self._jac_cache[0].matches(m)
        quad = self._quadrature(self._lin_point, "linpoint")
        names = []
        if need_A and not self.matrix_free_solves:
            names.append("A")
        if not self._mf:
            names.append("C")
            if not gauss_newton_approx:
                names += ["Wum", "Wmm"]
        # the vectors of the assembled blocks come with them (their row sums, summed in
        # the same pass): dR/dp with C, dR/du with W_um, dR/dm with W_mm, kept for a
        # residual or gradient asked for at this same point
        vnames = tuple(v for v, b in ((ADJOINT, "C"), (STATE, "Wum"), (PARAMETER, "Wmm"))
                       if b in names) if self.precision == _lib.HM_FP64 else ()
        blocks, vecs = (self._assemble(quad, blocks=tuple(names), vectors=vnames) if names
                        else ({}, {}))
        self._require_finite("linearization point")
        self._lin_vectors = vecs
        if need_A:
            A = blocks["A"] if "A" in blocks else self._make_jacobian(quad)
            self._jac_cache = (_Snapshot(m), A, quad)
            self.solver = None
        self.A, self.At = self._jac_cache[1], self._jac_cache[1]
        self.C = blocks.get("C")
        self.Wum = blocks.get("Wum")
        self.Wmm = blocks.get("Wmm")
        # the incremental solvers are made at the first incremental solve of the point
        # (a point whose gradient alone is asked for never pays for their set-up)
        self.solver_fwd_inc = self.solver_adj_inc = None
        return self

    def solveIncremental(self, out, rhs, is_adj, rel_tolerance=None):
        """The incremental forward or adjoint solve, right-hand side zeroed on the
        essential dofs (:1583)."""
        r = rhs.clone()
        self.bc0.zero(r)
        out.zero_()
        self.n_calls["incremental_adjoint" if is_adj else "incremental_forward"] += 1
        if self.solver_fwd_inc is None or self.solver_fwd_inc.op is not self.A:
            self.solver_fwd_inc = self._get_solver(self.A)
            self.solver_adj_inc = self.solver_fwd_inc      # A^T = A: one solver serves both
        solver = self.solver_adj_inc if is_adj else self.solver_fwd_inc
        prm = solver.parameters
        own = None
        if rel_tolerance is not None and prm["rel_tolerance"] < float(rel_tolerance):
            own, prm["rel_tolerance"] = prm["rel_tolerance"], float(rel_tolerance)
        try:
            solver.solve(out, r)
        finally:
            if own is not None:
                prm["rel_tolerance"] = own
        self.last_solve = solver.last
        return out

    # ------------------------------------------------------------- derivatives
    def block_is_zero(self, i, j):
        if self.A is None or {i, j} == {STATE, ADJOINT}:
            return False
        if (i, j) == (STATE, STATE):
            return True                       # linear in the state
        if self.gauss_newton_approx and ADJOINT not in (i, j):
            return True
        return False

    def apply_ij(self, i, j, dir, out):
        """Apply the ``(i, j)`` second-derivative block to ``dir`` (:1629)."""
        if self.A is None:
            raise RuntimeError("setLinearizationPoint must be called first")
        if getattr(self, "_mf", False) and {i, j} != {STATE, ADJOINT}:
            return self.apply_ij_at(i, j, self._lin_point, dir, out)
        table = {(ADJOINT, STATE): (self.A, False), (STATE, ADJOINT): (self.A, True),
                 (ADJOINT, PARAMETER): (self.C, False), (PARAMETER, ADJOINT): (self.C, True),
                 (STATE, STATE): (self.Wuu, False), (STATE, PARAMETER): (self.Wum, False),
                 (PARAMETER, STATE): (self.Wum, True), (PARAMETER, PARAMETER): (self.Wmm, False)}
        if (i, j) not in table:
            raise ValueError("no block (%d, %d)" % (i, j))
        mat, transpose = table[(i, j)]
        if mat is None:
            out.zero_()
            return out
        if out.numel() != mat.nrow or dir.numel() != mat.ncol:
            raise ValueError("apply_ij(%d, %d): block is %d x %d, got dir of size %d and out "
                             "of size %d" % (i, j, mat.nrow, mat.ncol, dir.numel(), out.numel()))
        if transpose:
            mat.mult_transpose(dir, out)
        else:
            mat.mult(dir, out)
        return out

    def _dir_products(self, x, mhat):
        """``C mhat``, ``W_um mhat`` and ``W_mm mhat`` at ``x`` from one pass over the
        fields (``hm_lattice_vectors`` with ``mhat``, no source), with the row
        eliminations of C and W_um; kept for the next products along the same ``mhat``
        at the same point."""
        c = self._dir_cache
        if c is not None and all(a.matches(v) for a, v in zip(c[0], list(x) + [mhat])):
            return c[1]
        vecs = self._direct_vectors(x, (ADJOINT, STATE, PARAMETER), mhat=mhat, zero_ess=True)
        self._require_finite("the second-order products")
        self._dir_cache = (tuple(_Snapshot(v) for v in list(x) + [mhat]), vecs)
        return vecs

    def directional_products(self, mhat):
        """``{ADJOINT: C mhat, STATE: W_um mhat, PARAMETER: W_mm mhat}`` at the
        linearization point in one pass over its fields (the row eliminations of C and
        W_um applied), or None where the point has no FP64 fields to take them from.  The
        Hessian action's three products along its direction, faster than three products
        of the assembled blocks, equal to rounding."""
        if self._lin_point is None or any(v is None for v in self._lin_point):
            return None
        vecs = self._direct_vectors(self._lin_point, (ADJOINT, STATE, PARAMETER), mhat=mhat,
                                    zero_ess=True)
        self._require_finite("the second-order products")
        return vecs

    def transposed_product(self, i, j, dir, out):
        """``C^T dir`` (i, j = PARAMETER, ADJOINT) or ``W_mu dir`` (PARAMETER, STATE) at
        the linearization point as ``dR/dm`` with the direction in the adjoint or state
        slot: faster than the transposed product of the assembled block, equal to
        rounding; through ``apply_ij`` where the point has no FP64 fields."""
        if self._lin_point is None or any(v is None for v in self._lin_point):
            return self.apply_ij(i, j, dir, out)
        return self.apply_ij_at(i, j, self._lin_point, dir, out)

    def apply_ij_at(self, i, j, x, dir, out):
        """The ``(i, j)`` block at ``x`` applied to ``dir`` without forming the block
        (:1672): the Jacobian pair through the matrix-free operator; the second-order
        blocks from the vector kernels -- ``C``, ``W_um``, ``W_mm`` times a parameter
        direction from the directional quadrature data, ``C^T p`` and ``W_mu u`` as
        ``dR/dm`` with the direction in the adjoint or state slot (eliminated rows
        zeroed first)."""
        if {i, j} == {STATE, ADJOINT}:
            quad = self._quadrature([None, x[PARAMETER], None], "apply")
            MatrixFreeJacobian(self.mesh, quad, self.bc0.marker, self.precision).mult(dir, out)
            return out
        if (i, j) == (STATE, STATE) or (self.gauss_newton_approx and ADJOINT not in (i, j)):
            out.zero_()
            return out
        x = self._locals(x)
        if j == PARAMETER:
            if (i, j) not in ((ADJOINT, PARAMETER), (STATE, PARAMETER), (PARAMETER, PARAMETER)):
                raise ValueError("no block (%d, %d)" % (i, j))
            out.copy_(self._dir_products(x, dir)[i])
            return out
        if (i, j) not in ((PARAMETER, ADJOINT), (PARAMETER, STATE)):
            raise ValueError("no block (%d, %d)" % (i, j))
        d = dir.masked_fill(self.bc0.mask, 0.0)
        y = [x[STATE], x[PARAMETER], d] if j == ADJOINT else [d, x[PARAMETER], x[ADJOINT]]
        vecs = self._direct_vectors(y, (PARAMETER,))
        self._require_finite("the second-order products")
        out.copy_(vecs[PARAMETER])
        return out
