"""The lattice path on a caller's own dof numbering, the element-matrix export and the
C-ABI Hessian action.

* :class:`CallerNumbering` -- a caller whose Q2 space numbers its dofs otherwise than the
  lattice (MFEM: its element-to-dof table, ``hippymfem/fem/elementbatch.py:528-565``, in
  MFEM's element-local order) gets every vector and every block in its numbering: its
  own CSR pattern (the arrays ``hm_pattern_build`` gives for its table, which are the
  reference's ``ScatterPattern`` arrays, ``fem/pattern.py:548-663``) and the values
  mapped into it by one deterministic gather per block.
* :func:`element_matrices` -- the ``(count, 27, 27)`` element matrices of a point
  (``QuadratureKernel.element_matrices``, ``hippymfem/fem/kernel.py:1964-2068``) in a
  caller-chosen element-local order; not on the fused path.
* :class:`AssembledHessian` -- ``ReducedHessian.mult`` (``modeling/reducedHessian.py:
  87-131``) as one C-ABI object over the assembled blocks and a solve plan.
"""

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, hptr, lib, ptr, stream_ptr
from .pattern import build_tables


class CallerNumbering:
    """The caller's numbering of the lattice's Q2 dofs.

    ``cdofs``: ``(ne, 27)`` element dof table, elements in the lattice order
    ``e = ex + nx (ey + ny ez)``; ``local[a]``: the caller's element-local slot of
    lattice-local dof ``a = a1 + 3 a2 + 9 a3`` (``None``: the same order)."""

    def __init__(self, mesh, cdofs, local=None):
        self.mesh = mesh
        dev = mesh.device
        cdofs = np.ascontiguousarray(cdofs, dtype=np.int64)
        if cdofs.shape != (mesh.ne, 27):
            raise ValueError("the element dof table must be (%d, 27)" % mesh.ne)
        loc = None if local is None else np.ascontiguousarray(local, dtype=np.int32)
        if loc is not None and loc.shape != (27,):
            raise ValueError("local must hold 27 slots")
        perm = np.empty(mesh.ndof, dtype=np.int32)
        check(lib.hm_lattice_dof_permutation(mesh.handle, hptr(cdofs), hptr(loc), hptr(perm)),
              "hm_lattice_dof_permutation")
        self.perm_host = perm
        self.perm = torch.as_tensor(perm, device=dev)                  # lattice -> caller
        inv = np.empty_like(perm)
        inv[perm] = np.arange(mesh.ndof, dtype=np.int32)
        self.iperm = torch.as_tensor(inv, device=dev)                  # caller -> lattice
        indptr, indices, slot, nnz = build_tables(cdofs, cdofs, mesh.ndof, mesh.ndof)
        if nnz != mesh.nnz:
            raise ValueError("the caller's pattern has %d entries, the lattice's %d"
                             % (nnz, mesh.nnz))
        self.indptr_host, self.indices_host, self.slot_host = indptr, indices, slot
        self.indptr = torch.as_tensor(indptr, device=dev)
        self.indices = torch.as_tensor(indices, device=dev)
        self.src_pos = torch.empty(mesh.nnz, dtype=torch.int32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        check(lib.hm_lattice_caller_map(mesh.handle, ptr(self.perm), ptr(self.indptr),
                                        ptr(self.indices), ptr(self.src_pos), ptr(status),
                                        stream_ptr()), "hm_lattice_caller_map")
        if int(status.item()) & _lib.HM_STATUS_RANGE:
            raise ValueError("the caller's pattern does not match the lattice's entries")

    def _gather(self, idx, src, out):
        if out is None:
            out = torch.empty(idx.numel(), dtype=torch.float64, device=src.device)
        check(lib.hm_gather_f64(idx.numel(), ptr(idx), ptr(src), ptr(out), stream_ptr()),
              "hm_gather_f64")
        return out

    def to_lattice(self, v, out=None):
        """A vector in the caller's numbering -> the lattice's."""
        return self._gather(self.perm, v, out)

    def to_caller(self, v, out=None):
        """A vector in the lattice's numbering -> the caller's."""
        return self._gather(self.iperm, v, out)

    def values_to_caller(self, vals, out=None):
        """Block values on the lattice pattern -> the caller's CSR ``data`` (its
        ``indptr``/``indices`` are :attr:`indptr`/:attr:`indices`)."""
        return self._gather(self.src_pos, vals, out)


def element_matrices(mesh, quad, precision=_lib.HM_FP64, names=("A", "C", "Wum", "Wmm"), e0=0,
                     count=None, local=None):
    """``{name: (count, 27, 27)}`` element matrices of the point whose quadrature data is
    ``quad`` (rows: test dof, columns: trial dof), at ``[e][local[a]][local[b]]``."""
    count = mesh.ne - e0 if count is None else int(count)
    out = {n: torch.empty((count, 27, 27), dtype=torch.float64, device=mesh.device)
           for n in names}
    loc = None if local is None else np.ascontiguousarray(local, dtype=np.int32)
    check(lib.hm_lattice_element_blocks(mesh.handle, ptr(quad), precision, int(e0), count,
                                        hptr(loc), ptr(out.get("A")), ptr(out.get("C")),
                                        ptr(out.get("Wum")), ptr(out.get("Wmm")), stream_ptr()),
          "hm_lattice_element_blocks")
    return out


class AssembledHessian:
    """``hm_hessian``: the misfit part of the reduced Hessian at an assembled point.

    ``pattern``: the lattice pattern (with its transpose map); ``C``, ``Wum``, ``Wmm``:
    CSR value tensors (``Wum = Wmm = None``: Gauss-Newton); ``misfit``: a
    ``DiscreteStateObservation`` (its ``B``, ``Bt`` and noise variance) or ``None``;
    ``plan``: a ``SolvePlan`` of the point's Jacobian."""

    def __init__(self, mesh, pattern, C, Wum, Wmm, misfit, marker, plan):
        self.mesh = mesh
        nobs = 0 if misfit is None else int(misfit.B.shape[0])
        self._keep = (pattern, C, Wum, Wmm, misfit, marker, plan)
        self.work = torch.empty(lib.hm_hessian_workspace_bytes(mesh.ndof, nobs) // 8 + 1,
                                dtype=torch.float64, device=mesh.device)
        B = misfit.B if misfit is not None else None
        Bt = misfit.Bt if misfit is not None else None
        h = ctypes.c_void_p()
        check(lib.hm_hessian_create(
            mesh.handle, ptr(pattern.indptr), ptr(pattern.indices), ptr(pattern.tpos), ptr(C),
            ptr(Wum), ptr(Wmm), nobs,
            ptr(B.indptr) if B is not None else None, ptr(B.indices) if B is not None else None,
            ptr(B.values) if B is not None else None,
            ptr(Bt.indptr) if Bt is not None else None, ptr(Bt.indices) if Bt is not None else None,
            ptr(Bt.values) if Bt is not None else None,
            float(misfit.noise_variance) if misfit is not None else 0.0,
            ptr(marker), plan._plan, ptr(self.work), ctypes.byref(h)), "hm_hessian_create")
        self.handle = h
        self.iterations = (0, 0)

    def mult(self, x, y, rel_tolerance=1e-12, max_iter=20000):
        it = (ctypes.c_int * 2)()
        check(lib.hm_hessian_apply(self.handle, ptr(x), ptr(y), float(rel_tolerance),
                                   int(max_iter), it, stream_ptr()), "hm_hessian_apply")
        self.iterations = (it[0], it[1])
        return y

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and lib is not None:
            lib.hm_hessian_destroy(h)
            self.handle = None
