"""The reduced-Hessian action sharded over z-slabs, with gloo ranks on the CPU.

Each rank runs ``ShardedHessian`` on its slab with the oracle as its local operators
(the assembled local blocks of its lattice, its slab and one element layer below); the
halos travel by ``exchange_planes`` and the inner products by per-plane partial sums.
The action on 2 and 3 ranks equals the one-rank action bit for bit, and the oracle's
``TrueHessian`` (and ``GNHessian``) restatement on the whole lattice to the solve
tolerance.  CPU only.
"""

import datetime
import os
import socket

import numpy as np
import pytest
import scipy.sparse as sp
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import q2

N_ELEM = (3, 4, 7)
BOX = (1.0, 0.8, 1.3)
NOBS = 40
NOISE = 1e-3


def _data():
    mesh = q2.Lattice(N_ELEM, BOX)
    rng = np.random.default_rng(41)
    u, p = rng.standard_normal(mesh.ndof), rng.standard_normal(mesh.ndof)
    m = 0.4 * rng.standard_normal(mesh.ndof)
    x = rng.standard_normal(mesh.ndof)
    ess = np.zeros(mesh.ndof, np.int32)
    ess[mesh.boundary_dofs()] = 1
    pts = 0.05 + 0.9 * rng.random((NOBS, 3)) * np.asarray(BOX)
    return mesh, u, m, p, x, ess, pts


class OracleSlabOps:
    """Rank's local operators from the oracle: the assembled blocks of its lattice with
    the folded elimination, the vector assembly, and the rows of the global observation
    operator whose targets lie in its elements (columns shifted to its lattice)."""

    def __init__(self, part, rank, pts):
        from hippymfem_b200.shard import local_points

        n, L = part.local_box(rank)
        self.mesh = q2.Lattice(n, L)
        self.E = self.mesh.edofs()
        nd = self.mesh.ndof
        self.pat = q2.build_tables(self.E, self.E, nd, nd, True)
        Bg = sp.csr_matrix(q2.observation_matrix(q2.Lattice(N_ELEM, BOX), pts))
        _, keep = local_points(part, rank, pts)
        l0, _ = part.local_planes(rank)
        Bk = Bg[keep].tocoo()
        self.B = sp.csr_matrix((Bk.data, (Bk.row, Bk.col - l0 * part.plane)),
                               shape=(len(keep), nd))
        self.Bt = self.B.T.tocsr()

    def set_point(self, u, m, p, ess):
        self.u, self.m, self.p = (np.asarray(t, dtype=np.float64) for t in (u, m, p))
        self.mask = np.asarray(ess).astype(bool)
        blk = q2.element_blocks(self.mesh, self.E, self.u, self.m, self.p)
        nd = self.mesh.ndof
        self.blocks = {k: q2.csr(self.pat, q2.assemble_block(k, self.pat, blk[k], self.mask),
                                 (nd, nd)) for k in blk}

    def apply_A(self, x):
        return torch.as_tensor(self.blocks["A"] @ np.asarray(x))

    def diag_A(self):
        return torch.as_tensor(self.blocks["A"].diagonal().copy())

    def dir_products(self, mhat):
        mh = np.asarray(mhat)
        return tuple(torch.as_tensor(self.blocks[k] @ mh) for k in ("C", "Wum", "Wmm"))

    def grad_m(self, u, p):
        ev = q2.element_vectors(self.mesh, self.E, np.asarray(u), self.m, np.asarray(p), 0.0)
        return torch.as_tensor(q2.assemble_vector(self.E, ev[q2.PARAMETER], self.mesh.ndof))

    def wuu(self, x):
        return torch.as_tensor(self.Bt @ (self.B @ np.asarray(x)) / NOISE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    from hippymfem_b200.shard import ShardedHessian, SlabPartition

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        mesh, u, m, p, x, ess, pts = _data()
        part = SlabPartition(N_ELEM, BOX, world)
        k0, k1 = part.owned_planes(rank)
        own = [torch.as_tensor(a.reshape(mesh.N[2], -1)[k0:k1].copy()) for a in (u, m, p, ess, x)]
        ops = OracleSlabOps(part, rank, pts)
        res = []
        for gn in (False, True):
            H = ShardedHessian(part, rank, ops, *own[:4], rtol=1e-13, gauss_newton=gn)
            y = H.mult(own[4])
            res.append((y.numpy().reshape(-1), H.iterations))
        out.put((rank, res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = {}
    try:
        for _ in range(world):
            r, res = out.get(timeout=240)
            got[r] = res
    finally:
        for pr in procs:
            pr.join(timeout=60)
            if pr.exitcode is None:
                pr.kill()
    assert all(pr.exitcode == 0 for pr in procs)
    # per variant (true, Gauss-Newton): the global vector and rank 0's solve counts
    return [(np.concatenate([got[r][v][0] for r in range(world)]), got[0][v][1])
            for v in range(2)]


def test_sharded_hessian_action_is_the_one_rank_action():
    one = _run(1)
    mesh, u, m, p, x, ess, pts = _data()
    assert one[0][0].shape == (mesh.ndof,)
    for world in (2, 3):
        many = _run(world)
        for (yw, itw), (y1, it1) in zip(many, one):
            assert itw == it1
            assert np.array_equal(yw, y1), world
    for gn, (y1, _) in zip((False, True), one):
        _check_oracle(mesh, u, m, p, x, ess, pts, gn, y1)


def _check_oracle(mesh, u, m, p, x, ess, pts, gn, y1):
    # the oracle's restatement on the whole lattice (Jacobi-PCG to 1e-13 there too)
    E = mesh.edofs()
    nd = mesh.ndof
    mask = ess.astype(bool)
    pat = q2.build_tables(E, E, nd, nd, True)
    blk = q2.element_blocks(mesh, E, u, m, p)
    blocks = {k: q2.csr(pat, q2.assemble_block(k, pat, blk[k], mask), (nd, nd)) for k in blk}
    B = q2.observation_matrix(mesh, pts)
    Wuu = (B.T @ B) / NOISE
    if gn:
        blocks = dict(blocks, Wum=0 * blocks["Wum"], Wmm=0 * blocks["Wmm"])
    yref, _ = q2.hessian_apply(blocks, x, np.flatnonzero(mask), Wuu=Wuu, rtol=1e-13)
    assert np.linalg.norm(y1 - yref) <= 1e-10 * np.linalg.norm(yref)
