"""Sharded assembly over z-slabs with gloo ranks on the CPU: the halo exchange of the
input planes, the local lattices and the owned row stretches, with the oracle as each
rank's assembler, reproduce the global assembly's blocks and vectors bit for bit and
cover them exactly once.  CPU only."""

import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import q2

N_ELEM = (3, 4, 7)
BOX = (1.0, 0.8, 1.3)
F = 1.3


def _fields(mesh):
    rng = np.random.default_rng(21)
    u, p = rng.standard_normal(mesh.ndof), rng.standard_normal(mesh.ndof)
    m = 0.4 * rng.standard_normal(mesh.ndof)
    ess = np.zeros(mesh.ndof, np.int32)
    ess[mesh.boundary_dofs()] = 1
    return u, m, p, ess


def _oracle_assembler(n, L, u, m, p, ess, f):
    mo = q2.Lattice(n, L)
    E = mo.edofs()
    nd = mo.ndof
    pat = q2.build_tables(E, E, nd, nd, True)
    u, m, p = (np.asarray(t, dtype=np.float64) for t in (u, m, p))
    mask = np.asarray(ess).astype(bool)
    blk = q2.element_blocks(mo, E, u, m, p)
    blocks = {k: q2.assemble_block(k, pat, blk[k], mask) for k in blk}
    ev = q2.element_vectors(mo, E, u, m, p, f)
    vecs = {}
    for s in (q2.STATE, q2.PARAMETER, q2.ADJOINT):
        v = q2.assemble_vector(E, ev[s], nd)
        if s != q2.PARAMETER:
            v[mask] = 0.0
        vecs[s] = v
    return pat[0], blocks, vecs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    from hippymfem_b200.shard import SlabPartition, assemble_slab

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mesh = q2.Lattice(N_ELEM, BOX)
        part = SlabPartition(N_ELEM, BOX, world)
        u, m, p, ess = _fields(mesh)
        k0, k1 = part.owned_planes(rank)
        own = [torch.as_tensor(a.reshape(mesh.N[2], -1)[k0:k1].copy()) for a in (u, m, p, ess)]
        blocks, vecs, csr, dofs = assemble_slab(part, rank, *own, _oracle_assembler, f=F)
        out.put((rank, {k: np.asarray(v) for k, v in blocks.items()},
                 {k: np.asarray(v) for k, v in vecs.items()}, csr, dofs))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_reproduce_the_global_assembly(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = sorted((out.get(timeout=300) for _ in range(world)), key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        if pr.is_alive():
            pr.kill()
    assert all(pr.exitcode == 0 for pr in procs)

    mesh = q2.Lattice(N_ELEM, BOX)
    u, m, p, ess = _fields(mesh)
    indptr, blocks, vecs = _oracle_assembler(N_ELEM, BOX, u, m, p, ess, F)
    nnz = int(indptr[-1])
    s_prev, g_prev = 0, 0
    for rank, b, v, (s0, s1), (g0, g1) in got:
        assert s0 == s_prev and g0 == g_prev            # stretches tile the global arrays
        assert s0 == indptr[g0] and s1 == indptr[g1]
        for k in blocks:
            assert np.array_equal(b[k], blocks[k][s0:s1]), (rank, k)
        for s in vecs:
            assert np.array_equal(v[s], vecs[s][g0:g1]), (rank, s)
        s_prev, g_prev = s1, g1
    assert s_prev == nnz and g_prev == mesh.ndof


def test_partition_geometry():
    from hippymfem_b200.shard import SlabPartition, exact_length, plane_csr_offset

    part = SlabPartition((5, 6, 9), (1.0, 1.0, 0.7), 4)
    assert part.cut == [0, 2, 4, 7, 9]
    planes = [part.owned_planes(r) for r in range(4)]
    assert planes[0][0] == 0 and planes[-1][1] == 19
    assert all(planes[r][1] == planes[r + 1][0] for r in range(3))
    assert part.local_planes(0) == (0, 5) and part.local_planes(2) == (6, 15)
    for r in range(4):
        (n, L) = part.local_box(r)
        assert L[2] / n[2] == part.h[2]
    assert exact_length(0.7 / 9, 3) / 3 == 0.7 / 9
    mo = q2.Lattice((5, 6, 9), (1.0, 1.0, 0.7))
    E = mo.edofs()
    indptr = q2.build_tables(E, E, mo.ndof, mo.ndof, True)[0]
    plane = mo.N[0] * mo.N[1]
    for k in range(mo.N[2] + 1):
        assert plane_csr_offset(mo.N, k) == indptr[k * plane]
    with pytest.raises(ValueError):
        SlabPartition((2, 2, 3), (1, 1, 1), 4)


@pytest.mark.parametrize("world", [1, 2, 4])
def test_hypre_arrays_are_the_global_rows(world):
    """Each rank's row pointers and global columns (from its local lattice's pattern)
    are the global pattern's rows, diagonal first as hypre keeps them."""
    from hippymfem_b200.shard import SlabPartition, hypre_arrays

    n, L = (4, 3, 8), (1.0, 0.6, 1.1)
    part = SlabPartition(n, L, world)
    mo = q2.Lattice(n, L)
    E = mo.edofs()
    gptr, gind = q2.build_tables(E, E, mo.ndof, mo.ndof, True)[:2]
    for r in range(world):
        nl, Ll = part.local_box(r)
        ml = q2.Lattice(nl, Ll)
        El = ml.edofs()
        lptr, lind = q2.build_tables(El, El, ml.ndof, ml.ndof, True)[:2]
        I, J, rows = hypre_arrays(part, r, lptr, lind)
        g0, g1 = rows
        assert I.dtype == np.int32 and J.dtype == np.int64
        assert np.array_equal(I, gptr[g0:g1 + 1] - gptr[g0])
        assert np.array_equal(J, gind[gptr[g0]:gptr[g1]])
        assert np.all(J[I[:-1]] == np.arange(g0, g1))          # diagonal first


def test_hypre_arrays_from_tensors_match_numpy():
    from hippymfem_b200.shard import SlabPartition, hypre_arrays

    n, L = (3, 3, 6), (1.0, 1.0, 1.0)
    part = SlabPartition(n, L, 3)
    nl, Ll = part.local_box(1)
    ml = q2.Lattice(nl, Ll)
    El = ml.edofs()
    lptr, lind = q2.build_tables(El, El, ml.ndof, ml.ndof, True)[:2]
    In, Jn, rn = hypre_arrays(part, 1, lptr, lind)
    It, Jt, rt = hypre_arrays(part, 1, torch.as_tensor(lptr), torch.as_tensor(lind))
    assert It.dtype == torch.int32 and Jt.dtype == torch.int64
    assert np.array_equal(It.numpy(), In) and np.array_equal(Jt.numpy(), Jn)
    assert np.array_equal(rt, rn)
