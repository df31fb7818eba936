"""Assembly sharded over several GPUs (one process each): z-slabs of node rows.

The reference's true-dof route (``fem/tdofassemble.py:5-35, 657-724``) assembles element
blocks on each rank's element partition and sends the partial sums of the rows on a
partition boundary to their owners.  The fused lattice kernel computes every CSR value
of a row from the fields of the elements around it, so the exchange moves to the inputs:
a rank owns the node planes ``[2 z0, 2 z1)`` (the last one also the top plane ``2 nz``)
of the element planes ``[z0, z1)`` of its slab, receives the node values of two planes
below (from the rank under it) and one plane above (from the rank over it), and
assembles its slab plus one element layer below as a lattice of its own.  Its owned rows
are then complete and unclipped (their stencils stay inside that lattice), and, rows
being numbered plane by plane, they are one stretch of the local CSR arrays and one
stretch of the global ones, with the same columns shifted by a constant node offset.

``SlabPartition`` holds the geometry, ``exchange_planes`` the halo exchange over
``torch.distributed`` (NCCL for device tensors, gloo for host tensors), and
``assemble_slab`` runs an assembler on the local lattice and returns the owned stretch,
``hypre_arrays`` the row pointers and global columns hypre takes with it.
``device_slab_assembler`` is the fused CUDA assembler (``hm_lattice_quadrature`` +
``hm_lattice_assemble`` on the local lattice)."""

import numpy as np
import torch
import torch.distributed as dist

BLOCKS = ("A", "C", "Wum", "Wmm")


def stencil_count(i, N):
    """Columns of the 1D stencil of node i on an axis of N nodes (3 or 5)."""
    if i & 1:
        return 3
    return min(i + 2, N - 1) - max(i - 2, 0) + 1


def stencil_prefix(i, N):
    """1D (row, column) pairs of the rows before node i."""
    return sum(stencil_count(k, N) for k in range(i))


def plane_csr_offset(N, k):
    """CSR offset of the first row of node plane k of the lattice pattern (rows in node
    order, x fastest): the pairs of all rows of the planes below."""
    Nx, Ny, Nz = N
    return stencil_prefix(k, Nz) * stencil_prefix(Nx, Nx) * stencil_prefix(Ny, Ny)


def exact_length(h, n):
    """A box length L with L / n == h exactly (so that a lattice of n elements built from
    L has the element size h bit for bit)."""
    L = n * h
    for _ in range(64):
        q = L / n
        if q == h:
            return L
        L = np.nextafter(L, np.inf if q < h else -np.inf)
    raise ValueError("no length gives element size %r over %d elements" % (h, n))


class SlabPartition:
    """z-slabs of an ``(nx, ny, nz)`` lattice of the box ``L`` over ``world`` ranks: rank
    r takes the element planes ``[cut[r], cut[r + 1])``, ``cut[r] = round(r nz / world)``
    (at least one element plane each)."""

    def __init__(self, n, L, world):
        self.n = tuple(int(v) for v in n)
        self.L = tuple(float(v) for v in L)
        self.world = int(world)
        nz = self.n[2]
        if not 1 <= self.world <= nz:
            raise ValueError("%d ranks for %d element planes" % (self.world, nz))
        self.cut = [int(round(r * nz / self.world)) for r in range(self.world + 1)]
        self.N = tuple(2 * v + 1 for v in self.n)
        self.h = tuple(Lv / nv for Lv, nv in zip(self.L, self.n))
        self.plane = self.N[0] * self.N[1]            # nodes per plane

    def elements(self, rank):
        return self.cut[rank], self.cut[rank + 1]

    def owned_planes(self, rank):
        """Global node planes ``[k0, k1)`` whose rows (and vector entries) rank owns."""
        z0, z1 = self.elements(rank)
        return 2 * z0, (2 * z1 + 1 if rank == self.world - 1 else 2 * z1)

    def local_elements(self, rank):
        """Element planes of rank's lattice: its slab and one layer below."""
        z0, z1 = self.elements(rank)
        return max(z0 - 1, 0), z1

    def local_planes(self, rank):
        ze0, ze1 = self.local_elements(rank)
        return 2 * ze0, 2 * ze1 + 1

    def local_box(self, rank):
        """``(n, L)`` of rank's lattice, with the global element size exactly."""
        ze0, ze1 = self.local_elements(rank)
        nzl = ze1 - ze0
        return ((self.n[0], self.n[1], nzl),
                (self.L[0], self.L[1], exact_length(self.h[2], nzl)))

    def owned_local_rows(self, rank):
        """Rows ``[r0, r1)`` of rank's lattice that it owns."""
        k0, k1 = self.owned_planes(rank)
        l0, _ = self.local_planes(rank)
        return (k0 - l0) * self.plane, (k1 - l0) * self.plane

    def owned_global_rows(self, rank):
        k0, k1 = self.owned_planes(rank)
        return k0 * self.plane, k1 * self.plane

    def owned_global_csr(self, rank):
        """CSR value range ``[s0, s1)`` of the global pattern that rank's rows cover."""
        k0, k1 = self.owned_planes(rank)
        return plane_csr_offset(self.N, k0), plane_csr_offset(self.N, k1)


def exchange_planes(owned, part, rank, group=None):
    """Rank's local node values from its owned planes ``owned`` (shape ``(planes,
    nodes per plane)``, any dtype the backend carries): two planes from the rank below
    and one from the rank above, by point-to-point messages.  Every rank calls it."""
    k0, k1 = part.owned_planes(rank)
    l0, l1 = part.local_planes(rank)
    assert owned.shape[0] == k1 - k0
    below, above = k0 - l0, l1 - k1                   # 0 or 2, 0 or 1
    out = torch.empty((l1 - l0,) + tuple(owned.shape[1:]), dtype=owned.dtype,
                      device=owned.device)
    out[below:below + owned.shape[0]] = owned
    ops = []
    if rank > 0:                                      # my first plane: the rank below's top halo
        ops.append(dist.P2POp(dist.isend, owned[:1].contiguous(), rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, out[:below], rank - 1, group))
    if rank < part.world - 1:                         # my top two planes: the rank above's
        ops.append(dist.P2POp(dist.isend, owned[-2:].contiguous(), rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, out[below + owned.shape[0]:], rank + 1, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return out


def assemble_slab(part, rank, u, m, p, ess, assembler, f=1.0, group=None):
    """Rank's stretch of the global blocks and vectors.

    ``u, m, p`` (FP64) and ``ess`` (Dirichlet markers, 0/1): rank's owned planes, shape
    ``(planes, nodes per plane)``.  ``assembler(n, L, u, m, p, ess, f)`` assembles a
    lattice with the folded elimination and returns ``(indptr, blocks, vectors)``:
    ``blocks[name]`` the CSR values of A, C, W_um, W_mm, ``vectors[slot]`` dR/du, dR/dm,
    dR/dp (slots STATE, PARAMETER, ADJOINT; zeroed on the Dirichlet nodes except dR/dm).
    Returns ``(blocks, vectors, (s0, s1), (g0, g1))``: the owned values, the owned
    vector entries, and their ranges in the global CSR values and dofs."""
    loc = [exchange_planes(t, part, rank, group).reshape(-1) for t in (u, m, p)]
    e = exchange_planes(ess.to(torch.int32), part, rank, group).reshape(-1)
    n, L = part.local_box(rank)
    indptr, blocks, vectors = assembler(n, L, loc[0], loc[1], loc[2], e, f)
    r0, r1 = part.owned_local_rows(rank)
    a, b = int(indptr[r0]), int(indptr[r1])
    owned_blocks = {k: v[a:b] for k, v in blocks.items()}
    owned_vectors = {k: v[r0:r1] for k, v in vectors.items()}
    s0, s1 = part.owned_global_csr(rank)
    assert s1 - s0 == b - a, "local and global row stretches differ"
    return owned_blocks, owned_vectors, (s0, s1), part.owned_global_rows(rank)


def hypre_arrays(part, rank, local_indptr, local_indices):
    """The arrays the reference hands hypre for rank's rows (``fem/parmat.py:106-171``,
    ``HypreParMatrix(comm, nrow, rglob, cglob, [I, J, D, rows])``): ``I`` the row
    pointers of the owned rows from 0 (int32), ``J`` their global column indices (int64:
    the local lattice's columns shifted by its first node plane), and ``rows`` the
    partition ``[first row, last row + 1]``; ``D`` is the owned stretch that
    ``assemble_slab`` returns.  Works on numpy arrays or tensors."""
    r0, r1 = part.owned_local_rows(rank)
    l0, _ = part.local_planes(rank)
    ip = local_indptr[r0:r1 + 1]
    a, b = int(ip[0]), int(ip[-1])
    if isinstance(ip, torch.Tensor):
        I = (ip - a).to(torch.int32)
        J = local_indices[a:b].to(torch.int64) + l0 * part.plane
    else:
        I = (np.asarray(ip, dtype=np.int64) - a).astype(np.int32)
        J = np.asarray(local_indices[a:b], dtype=np.int64) + l0 * part.plane
    g0, g1 = part.owned_global_rows(rank)
    return I, J, np.array([g0, g1], dtype=np.int64)


def device_slab_assembler(n, L, u, m, p, ess, f=1.0):
    """The fused CUDA assembly of a lattice (the tensors on its device)."""
    from . import _lib
    from ._lib import check, lib, ptr, stream_ptr
    from .mesh import BoxMesh
    from .pattern import LatticePattern

    dev = u.device
    mesh = BoxMesh(n, L, device=dev)
    pat = LatticePattern(mesh, with_transpose=False)
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    marker = ess.to(device=dev, dtype=torch.uint8).contiguous()
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(u), ptr(m), ptr(p), _lib.HM_FP64,
                                    ptr(quad), ptr(status), stream_ptr()), "hm_lattice_quadrature")
    blocks = {k: torch.empty(mesh.nnz, dtype=torch.float64, device=dev) for k in BLOCKS}
    vecs = [torch.empty(mesh.ndof, dtype=torch.float64, device=dev) for _ in range(3)]
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr),
                                  ptr(marker), float(f), *(ptr(blocks[k]) for k in BLOCKS),
                                  *(ptr(v) for v in vecs), 1, stream_ptr()), "hm_lattice_assemble")
    if int(status.item()) != 0:
        raise RuntimeError("non-finite values in the fields")
    return pat.indptr, blocks, {0: vecs[0], 1: vecs[1], 2: vecs[2]}
