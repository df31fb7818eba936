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
    """Rank's rows of the assembled global matrix as a row-partitioned ParCSR: ``I`` the
    row pointers of the owned rows from 0 (int32), ``J`` their global column indices
    (int64: the local lattice's columns shifted by its first node plane) and ``rows``
    the partition ``[first row, last row + 1]``; the values ``D`` are the owned stretch
    that ``assemble_slab`` returns.  These are the arguments of
    ``mfem.HypreParMatrix(comm, nrow, rglob, cglob, [I, J, D, rows])``, but not what the
    reference's ``local_par_matrix`` (``fem/parmat.py:106-171``) passes: there each rank
    hands hypre a block-diagonal matrix over its own local dofs and the true-dof route
    (``fem/tdofassemble.py``) forms ``P^T A P`` from it.  Here the rows are already the
    assembled global rows (an owned row holds columns of the neighbouring slabs), in the
    lattice's node numbering and partitioned by z-slab node planes, so the result replaces
    the whole true-dof assembly, and the vectors it multiplies must use the same slab
    partition and numbering (``SlabPartition.owned_global_rows``).  Works on numpy
    arrays or tensors."""
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


_SLAB_CACHE = {}


def device_slab_assembler(n, L, u, m, p, ess, f=1.0, check_finite=True):
    """The fused CUDA assembly of a lattice (the tensors on its device).  The mesh, its
    pattern and the buffers are kept per (n, L, device), so a Newton loop assembles again
    without rebuilding the pattern or allocating; the returned blocks and vectors are
    those buffers, overwritten by the next call on the same lattice.  With
    ``check_finite`` the status word is read (one synchronisation)."""
    from . import _lib
    from ._lib import check, lib, ptr, stream_ptr
    from .mesh import BoxMesh
    from .pattern import LatticePattern

    dev = u.device
    key = (tuple(n), tuple(L), str(dev))
    c = _SLAB_CACHE.get(key)
    if c is None:
        mesh = BoxMesh(n, L, device=dev)
        c = _SLAB_CACHE[key] = {
            "mesh": mesh, "pat": LatticePattern(mesh, with_transpose=False),
            "quad": torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=dev),
            "status": torch.zeros(1, dtype=torch.int32, device=dev),
            "blocks": {k: torch.empty(mesh.nnz, dtype=torch.float64, device=dev) for k in BLOCKS},
            "vecs": [torch.empty(mesh.ndof, dtype=torch.float64, device=dev) for _ in range(3)]}
    mesh, pat, quad, status = c["mesh"], c["pat"], c["quad"], c["status"]
    blocks, vecs = c["blocks"], c["vecs"]
    marker = ess.to(device=dev, dtype=torch.uint8).contiguous()
    status.zero_()
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(u), ptr(m), ptr(p), _lib.HM_FP64,
                                    ptr(quad), ptr(status), stream_ptr()), "hm_lattice_quadrature")
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr),
                                  ptr(marker), float(f), *(ptr(blocks[k]) for k in BLOCKS),
                                  *(ptr(v) for v in vecs), 1, stream_ptr()), "hm_lattice_assemble")
    if check_finite and int(status.item()) != 0:
        raise RuntimeError("non-finite values in the fields")
    return pat.indptr, blocks, {0: vecs[0], 1: vecs[1], 2: vecs[2]}


# ------------------------------------------------------------- sharded Hessian action
# The reduced-Hessian action (modeling/reducedHessian.py:87-131) over the same z-slabs.
# Every operator of the action is a vector assembly on rank's lattice (its slab and one
# element layer below) from node values on its planes: the Jacobian apply, the second-
# order products from the directional data (C mhat, W_um mhat, W_mm mhat), the
# transposed ones as dR/dm with the direction in the adjoint or state slot, and the
# misfit's W_uu from the observations inside rank's elements.  So one exchange of the
# input's halo planes (exchange_planes) precedes each, and the owned rows of its result
# are complete -- the hypre ParCSR halo of the reference's true-dof route
# (fem/tdofassemble.py:657-724, common/parvector.py:107-146) moved to the inputs.  The
# incremental solves are Jacobi-PCG over the slabs; each inner product is the sum, in
# plane order, of per-node-plane partial sums gathered from all ranks, so the action is
# bit for bit the same on any number of ranks (a plane's partial is computed alike
# wherever it lives).

def plane_partials(a, b):
    """Per-node-plane partial sums of a . b for owned-plane arrays (planes, nodes)."""
    return (a * b).sum(dim=1)


def sharded_dot_t(part, a, b, group=None):
    """a . b over all ranks' owned planes, summed plane by plane in order, as a 0-d
    tensor on the vectors' device (no host synchronisation)."""
    pp = plane_partials(a, b)
    if part.world == 1:
        return pp.sum()
    sizes = [part.owned_planes(r)[1] - part.owned_planes(r)[0] for r in range(part.world)]
    width = max(sizes)
    mine = torch.zeros(width, dtype=pp.dtype, device=pp.device)
    mine[:pp.numel()] = pp
    bufs = [torch.empty(width, dtype=pp.dtype, device=pp.device) for _ in sizes]
    dist.all_gather(bufs, mine, group=group)
    return torch.cat([b[:s] for b, s in zip(bufs, sizes)]).sum()


def sharded_dot(part, a, b, group=None):
    """a . b over all ranks' owned planes, summed plane by plane in order."""
    return float(sharded_dot_t(part, a, b, group))


class ShardedHessian:
    """The misfit part of ``ReducedHessian.mult`` (TrueHessian; ``gauss_newton``:
    GNHessian) at the point ``(u, m, p)`` over the slabs of ``part``; every vector is
    rank's owned planes, shape ``(planes, nodes per plane)``.

    ``ops``: rank's local operators, an object with
    ``set_point(u, m, p, ess)`` (local node values), ``apply_A(x) -> y`` (the eliminated
    Jacobian), ``diag_A() -> d``, ``dir_products(mhat) -> (C mhat, W_um mhat, W_mm mhat)``
    (rows of C and W_um zeroed on the Dirichlet nodes), ``grad_m(u, p) -> dR/dm`` at
    ``(u, m, p)`` with the point's ``m``, and ``wuu(x) -> W_uu x`` -- all on rank's
    local lattice (vectors of its local planes, flattened)."""

    def __init__(self, part, rank, ops, u, m, p, ess, rtol=1e-12, max_iter=20000,
                 gauss_newton=False, group=None, check_every=8):
        self.part, self.rank, self.ops, self.group = part, rank, ops, group
        self.check_every = max(1, int(check_every))
        self.rtol, self.max_iter, self.gauss_newton = float(rtol), int(max_iter), gauss_newton
        self.shape = tuple(u.shape)
        self.ess = ess.to(torch.bool)
        loc = [self.halo(t) for t in (u, m, p)]
        self.ess_local = self.halo(ess.to(torch.int32)).to(torch.bool)
        self.u, self.m, self.p = loc
        ops.set_point(loc[0], loc[1], loc[2], self.ess_local)
        self.diag = self.own(ops.diag_A())
        self.iterations = []

    def halo(self, owned):
        return exchange_planes(owned, self.part, self.rank, self.group).reshape(-1)

    def own(self, local):
        r0, r1 = self.part.owned_local_rows(self.rank)
        return local[r0:r1].reshape(self.shape)

    def apply_A(self, x):
        return self.own(self.ops.apply_A(self.halo(x)))

    def dot(self, a, b):
        return sharded_dot(self.part, a, b, self.group)

    def dot_t(self, a, b):
        return sharded_dot_t(self.part, a, b, self.group)

    def solve(self, b):
        """A x = b (b zero on the Dirichlet nodes) by Jacobi-PCG from zero to ||r|| <=
        rtol ||b||; the iteration count is kept.  The scalars stay on the vectors'
        device; convergence is read every ``check_every`` iterations and frozen on the
        device when reached (the step length is zero from then on), so the result and
        the count are those of a check after every iteration."""
        x = torch.zeros_like(b)
        bb = self.dot_t(b, b)
        if float(bb) == 0.0:
            self.iterations.append(0)
            return x
        r = b.clone()
        z = r / self.diag
        d = z.clone()
        rz = self.dot_t(r, z)
        tol2 = (self.rtol * self.rtol) * bb
        zero = torch.zeros((), dtype=b.dtype, device=b.device)
        done = torch.zeros((), dtype=torch.bool, device=b.device)
        conv = torch.zeros((), dtype=torch.int64, device=b.device)
        for it in range(1, self.max_iter + 1):
            q = self.apply_A(d)
            alpha = torch.where(done, zero, rz / self.dot_t(d, q))
            x.add_(alpha * d)
            r.sub_(alpha * q)
            newly = (~done) & (self.dot_t(r, r) <= tol2)
            conv = torch.where(newly, torch.full_like(conv, it), conv)
            done = done | newly
            if it % self.check_every == 0 and bool(done):
                break
            z = r / self.diag
            rz_new = self.dot_t(r, z)
            d = z + torch.where(done, zero, rz_new / rz) * d
            rz = torch.where(done, rz, rz_new)
        if not bool(done):
            raise RuntimeError("sharded PCG did not reach rtol %g in %d iterations"
                               % (self.rtol, self.max_iter))
        self.iterations.append(int(conv))
        return x

    def mult(self, x):
        """y = H x on rank's owned planes (collective: every rank calls it)."""
        ops = self.ops
        xl = self.halo(x)
        c, wum, wmm = (self.own(v) for v in ops.dir_products(xl))
        uhat = self.solve(c.masked_fill(self.ess, 0.0))
        rhs = self.own(ops.wuu(self.halo(uhat)))
        if not self.gauss_newton:
            rhs = rhs - wum
        phat = self.solve(rhs.masked_fill(self.ess, 0.0))
        y = self.own(ops.grad_m(self.u, self.halo(phat.masked_fill(self.ess, 0.0))))
        if not self.gauss_newton:
            y = y + wmm - self.own(ops.grad_m(self.halo(uhat), self.p))
        return y


def local_points(part, rank, points):
    """The observation targets inside rank's local elements, in its lattice's
    coordinates, and their indices (the element of a target as the global lattice
    assigns it)."""
    pts = np.asarray(points, dtype=np.float64)
    ze0, ze1 = part.local_elements(rank)
    hz = part.h[2]
    ez = np.clip(np.floor(pts[:, 2] / hz).astype(np.int64), 0, part.n[2] - 1)
    keep = np.flatnonzero((ez >= ze0) & (ez < ze1))
    loc = pts[keep].copy()
    loc[:, 2] -= ze0 * hz
    return loc, keep


class DeviceSlabOps:
    """``ShardedHessian``'s local operators on the GPU: rank's lattice as a ``BoxMesh``
    and the library's kernels (the matrix-free Jacobian from the point's quadrature data,
    the assembled vectors straight from the fields, the device observation operator)."""

    def __init__(self, part, rank, points, noise_variance, device):
        from .mesh import BoxMesh
        from .modeling import device_observation_operator
        n, L = part.local_box(rank)
        self.mesh = BoxMesh(n, L, device=device)
        loc, _ = local_points(part, rank, points)
        self.nobs = len(loc)
        self.B = device_observation_operator(self.mesh, loc) if self.nobs else None
        self.Bt = self.B.transpose() if self.nobs else None
        self.inv_noise = 1.0 / float(noise_variance)
        self.quad = torch.empty(self.mesh.quad_bytes() // 8, dtype=torch.float64, device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.work = None

    def _quadrature(self, u, m, p, mhat=None):
        from . import _lib
        from ._lib import check, lib, ptr, stream_ptr
        if mhat is None:
            check(lib.hm_lattice_quadrature(self.mesh.handle, ptr(u), ptr(m), ptr(p), _lib.HM_FP64,
                                            ptr(self.quad), ptr(self.status), stream_ptr()))
        else:
            check(lib.hm_lattice_quadrature_dir(self.mesh.handle, ptr(u), ptr(m), ptr(p), ptr(mhat),
                                                _lib.HM_FP64, ptr(self.quad), ptr(self.status),
                                                stream_ptr()))

    def set_point(self, u, m, p, ess):
        from .sparse import MatrixFreeJacobian
        self.u, self.m, self.p = u.contiguous(), m.contiguous(), p.contiguous()
        self.marker = ess.to(torch.uint8).contiguous()
        self.mask = ess
        self._quadrature(self.u, self.m, self.p)
        self.A = MatrixFreeJacobian(self.mesh, self.quad, self.marker)

    def apply_A(self, x):
        y = torch.empty_like(x)
        return self.A.mult(x.contiguous(), y)

    def diag_A(self):
        return self.A.diagonal()

    def _direct(self, u, m, p, mhat, slots):
        """The vectors of ``slots`` straight from the fields (``hm_lattice_vectors``, no
        source term): STATE 0, PARAMETER 1, ADJOINT 2."""
        from ._lib import check, lib, ptr, stream_ptr
        if self.work is None:
            self.work = torch.empty(lib.hm_lattice_vectors_workspace_bytes(self.mesh.handle, 3) // 8,
                                    dtype=torch.float64, device=self.quad.device)
        out = {s: torch.empty(self.mesh.ndof, dtype=torch.float64, device=self.quad.device)
               for s in slots}
        check(lib.hm_lattice_vectors(self.mesh.handle, ptr(u), ptr(m), ptr(p), ptr(mhat), 0.0,
                                     None, ptr(out.get(0)), ptr(out.get(1)), ptr(out.get(2)), 0,
                                     ptr(self.work), ptr(self.status), stream_ptr()),
              "hm_lattice_vectors")
        return out

    def dir_products(self, mhat):
        v = self._direct(self.u, self.m, self.p, mhat.contiguous(), (0, 1, 2))
        return (v[2].masked_fill(self.mask, 0.0), v[0].masked_fill(self.mask, 0.0), v[1])

    def grad_m(self, u, p):
        return self._direct(u.contiguous(), self.m, p.contiguous(), None, (1,))[1]

    def wuu(self, x):
        if not self.nobs:
            return torch.zeros_like(x)
        bu = torch.empty(self.nobs, dtype=torch.float64, device=x.device)
        self.B.mult(x.contiguous(), bu)
        y = torch.empty_like(x)
        self.Bt.mult(bu, y, alpha=self.inv_noise)
        return y
