"""The Q2 hexahedral lattice: mesh, function space and Dirichlet markers.

``BoxMesh`` is the structured counterpart of the reference's ``MeshBatches`` /
``ElementGroup`` / ``SpaceTables`` (hippymfem/fem/elementbatch.py:159-565) for a uniform
box: geometry, basis tables and element dof tables are arithmetic inside the kernels,
so the mesh holds a host-side handle and nothing on the device.  Numbering:

* elements ``e = ex + nx (ey + ny ez)``;
* Q2 dofs lexicographic on the ``(2nx+1) x (2ny+1) x (2nz+1)`` node lattice;
* element-local dof ``a = a1 + 3 a2 + 9 a3`` is node ``(2ex+a1, 2ey+a2, 2ez+a3)``.
"""

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib


class BoxMesh:
    """Uniform ``nx x ny x nz`` hexahedral mesh of ``[0, Lx] x [0, Ly] x [0, Lz]``."""

    def __init__(self, n, L=(1.0, 1.0, 1.0), device=None):
        self.n = tuple(int(v) for v in (n if np.ndim(n) else (n, n, n)))
        self.L = tuple(float(v) for v in L)
        self.N = tuple(2 * v + 1 for v in self.n)
        self.h = tuple(Lv / nv for Lv, nv in zip(self.L, self.n))
        self.device = torch.device(device if device is not None else "cuda")
        h = ctypes.c_void_p()
        check(lib.hm_lattice_create(*self.n, *self.L, ctypes.byref(h)), "hm_lattice_create")
        self.handle = h
        ne, nd, nnz, qb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib.hm_lattice_sizes(h, _lib.HM_FP64, ctypes.byref(ne), ctypes.byref(nd),
                                   ctypes.byref(nnz), ctypes.byref(qb)))
        self.ne, self.ndof, self.nnz = ne.value, nd.value, nnz.value
        self._ess = {}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and lib is not None:
            lib.hm_lattice_destroy(h)
            self.handle = None

    def quad_bytes(self, precision=_lib.HM_FP64):
        qb = ctypes.c_int64()
        check(lib.hm_lattice_sizes(self.handle, precision, None, None, None, ctypes.byref(qb)))
        return qb.value

    # -------------------------------------------------------------- host helpers
    def node_coords(self):
        """``(ndof, 3)`` float64 host array of node coordinates."""
        Nx, Ny, _ = self.N
        i = np.arange(self.ndof)
        ix, iy, iz = i % Nx, (i // Nx) % Ny, i // (Nx * Ny)
        return np.stack([ix * self.h[0] / 2, iy * self.h[1] / 2, iz * self.h[2] / 2], -1)

    def edofs(self):
        """``(ne, 27)`` int64 host element dof table (for checks and the general path)."""
        nx, ny, nz = self.n
        Nx, Ny, _ = self.N
        e = np.arange(self.ne)
        ex, ey, ez = e % nx, (e // nx) % ny, e // (nx * ny)
        a = np.arange(27)
        a1, a2, a3 = a % 3, (a // 3) % 3, a // 9
        return ((2 * ex[:, None] + a1) + Nx * ((2 * ey[:, None] + a2)
                                               + Ny * (2 * ez[:, None] + a3))).astype(np.int64)

    def boundary_dofs(self):
        Nx, Ny, Nz = self.N
        i = np.arange(self.ndof)
        ix, iy, iz = i % Nx, (i // Nx) % Ny, i // (Nx * Ny)
        b = (ix == 0) | (ix == Nx - 1) | (iy == 0) | (iy == Ny - 1) | (iz == 0) | (iz == Nz - 1)
        return np.flatnonzero(b).astype(np.int64)

    def ess_marker(self, ess):
        """uint8 device marker of a set of essential dofs (cached on the array's id)."""
        if ess is None:
            return None
        key = id(ess)
        got = self._ess.get(key)
        if got is None or got[0] is not ess:
            m = torch.zeros(self.ndof, dtype=torch.uint8, device=self.device)
            if len(ess):
                m[torch.as_tensor(np.asarray(ess, dtype=np.int64), device=self.device)] = 1
            got = self._ess[key] = (ess, m)
        return got[1]


class Q2Space:
    """The Q2 H1 space on a ``BoxMesh``: what ``FunctionSpace.H1(mesh, 2)`` gives the
    reference (hippymfem/fem/spaces.py); vectors are FP64 CUDA tensors."""

    order = 2

    def __init__(self, mesh):
        self.mesh = mesh
        self.ndof = mesh.ndof

    def vector(self):
        return torch.zeros(self.ndof, dtype=torch.float64, device=self.mesh.device)

    def project(self, fn):
        """Nodal interpolation of ``fn(x) -> (ndof,)`` (``FunctionSpace.project``)."""
        vals = np.asarray(fn(self.mesh.node_coords()), dtype=np.float64)
        return torch.as_tensor(vals, device=self.mesh.device)


class DirichletBC:
    """Homogeneous essential condition on the whole boundary of a Q2 lattice space
    (``DirichletBC(space, None, "all")``, hippymfem/fem/bcs.py:115)."""

    def __init__(self, space, value=None, bdr_attributes="all"):
        if bdr_attributes != "all":
            raise NotImplementedError("only the whole boundary is supported")
        if value not in (None, 0, 0.0):
            raise NotImplementedError("only homogeneous conditions are supported")
        self.space = space
        self.ess_tdof = space.mesh.boundary_dofs()
        self.ess = self.ess_tdof
        self.marker = space.mesh.ess_marker(self.ess_tdof)
        self.mask = self.marker.bool()

    def zero(self, v):
        """Zero the essential entries of ``v`` in place (``zero_essential``)."""
        return v.masked_fill_(self.mask, 0.0)

    apply = zero
