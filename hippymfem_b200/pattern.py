"""Sparsity patterns of the element-assembly map.

* :func:`build_tables` -- the host build for any pair of dof tables, identical arrays
  to the reference's ``patternbuild.build_tables`` (hippymfem/fem/patternbuild.py:209-253)
  through ``hm_pattern_build``;
* :class:`LatticePattern` -- the pattern of a Q2 x Q2 block on a ``BoxMesh``, built on
  the device arithmetically (``hm_lattice_pattern``): ``indptr``/``indices`` in hypre's
  diagonal-first order, the entry->slot map on request and the transpose map used to
  apply a block transposed.  Replaces ``ScatterPattern`` / ``get_pattern``
  (hippymfem/fem/pattern.py:375-663, 1094).
"""

import ctypes

import numpy as np
import torch

from ._lib import check, hptr, lib, ptr, stream_ptr


def build_tables(tdofs, cdofs, nrow, ncol, diag_first=None, nthreads=0):
    """``(indptr, indices, slot, nnz)`` of the entries ``(e, a, b)`` -> row
    ``tdofs[e, a]``, column ``cdofs[e, b]``; int32 arrays as the reference keeps them.
    ``diag_first`` defaults to the reference's rule: a square shape leads with the
    diagonal (``ScatterPattern._diag_first``, hippymfem/fem/pattern.py:419)."""
    tdofs = np.ascontiguousarray(tdofs, dtype=np.int64)
    cdofs = np.ascontiguousarray(cdofs, dtype=np.int64)
    if tdofs.ndim != 2 or cdofs.ndim != 2 or tdofs.shape[0] != cdofs.shape[0]:
        raise ValueError("dof tables must be (ne, nd) with the same element count")
    ne, ndt = tdofs.shape
    ndr = cdofs.shape[1]
    if diag_first is None:
        diag_first = nrow == ncol
    indptr = np.empty(int(nrow) + 1, dtype=np.int32)
    nnz = ctypes.c_int64()
    args = (hptr(tdofs), hptr(cdofs), ne, ndt, ndr, int(nrow), int(ncol), int(bool(diag_first)),
            int(nthreads))
    check(lib.hm_pattern_build(*args, hptr(indptr), None, 0, None, ctypes.byref(nnz)),
          "hm_pattern_build")
    indices = np.empty(nnz.value, dtype=np.int32)
    slot = np.empty(ne * ndt * ndr, dtype=np.int32)
    check(lib.hm_pattern_build(*args, hptr(indptr), hptr(indices), nnz.value, hptr(slot),
                               ctypes.byref(nnz)), "hm_pattern_build")
    return indptr, indices, slot, int(nnz.value)


class LatticePattern:
    """Device CSR pattern of a Q2 x Q2 block on a ``BoxMesh`` (every block of the
    linearization point shares it: the parameter is Q2 on the same lattice)."""

    def __init__(self, mesh, with_slot=False, with_transpose=True, stream=None):
        self.mesh = mesh
        dev = mesh.device
        self.nrow = self.ncol = mesh.ndof
        self.nnz = mesh.nnz
        self.indptr = torch.empty(mesh.ndof + 1, dtype=torch.int32, device=dev)
        self.indices = torch.empty(mesh.nnz, dtype=torch.int32, device=dev)
        self.slot = (torch.empty(mesh.ne * 729, dtype=torch.int32, device=dev)
                     if with_slot else None)
        s = stream_ptr(stream)
        check(lib.hm_lattice_pattern(mesh.handle, ptr(self.indptr), ptr(self.indices),
                                     ptr(self.slot), s), "hm_lattice_pattern")
        self.tpos = None
        if with_transpose:
            self.tpos = torch.empty(mesh.nnz, dtype=torch.int32, device=dev)
            check(lib.hm_lattice_transpose_map(mesh.handle, ptr(self.indptr), ptr(self.tpos), s),
                  "hm_lattice_transpose_map")

    def new_values(self):
        return torch.empty(self.nnz, dtype=torch.float64, device=self.mesh.device)
