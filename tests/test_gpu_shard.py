"""The CUDA slab assembler of the sharded assembly on one GPU: three ranks emulated one
after the other (each given its local planes of the global fields, no collectives),
their owned stretches against the global assembly, bit for bit.  GPU."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_slab_stretches_equal_the_global_assembly(cuda):
    from hippymfem_b200.shard import SlabPartition, device_slab_assembler

    n, L, world = (6, 5, 9), (1.0, 0.8, 1.3), 3
    part = SlabPartition(n, L, world)
    Nx, Ny, Nz = part.N
    nd = Nx * Ny * Nz
    rng = np.random.default_rng(3)
    u, p = (torch.as_tensor(rng.standard_normal(nd), device=cuda) for _ in range(2))
    m = torch.as_tensor(0.3 * rng.standard_normal(nd), device=cuda)
    i = np.arange(nd)
    ix, iy, iz = i % Nx, (i // Nx) % Ny, i // (Nx * Ny)
    b = (ix == 0) | (ix == Nx - 1) | (iy == 0) | (iy == Ny - 1) | (iz == 0) | (iz == Nz - 1)
    ess = torch.as_tensor(b.astype(np.int32), device=cuda)
    gi, gb, gv = device_slab_assembler(n, L, u, m, p, ess, 1.3)
    covered = 0
    for r in range(world):
        l0, l1 = part.local_planes(r)
        sl = slice(l0 * part.plane, l1 * part.plane)
        nl, Ll = part.local_box(r)
        li, lb, lv = device_slab_assembler(nl, Ll, u[sl].contiguous(), m[sl].contiguous(),
                                           p[sl].contiguous(), ess[sl].contiguous(), 1.3)
        r0, r1 = part.owned_local_rows(r)
        a, c = int(li[r0]), int(li[r1])
        s0, s1 = part.owned_global_csr(r)
        g0, g1 = part.owned_global_rows(r)
        assert s0 == int(gi[g0]) and s1 == int(gi[g1])
        for k in gb:
            assert torch.equal(lb[k][a:c], gb[k][s0:s1]), (r, k)
        for s in gv:
            assert torch.equal(lv[s][r0:r1], gv[s][g0:g1]), (r, s)
        covered += s1 - s0
    assert covered == gb["A"].numel()


def test_device_slab_operators_give_the_hessian_action(cuda):
    """ShardedHessian with the CUDA slab operators (matrix-free Jacobian, the vectors
    straight from the fields, device observation operator) on one rank:
    the oracle's TrueHessian restatement to the solve tolerance.  The decomposition over
    several ranks is tested with gloo on the CPU (bit for bit against one rank)."""
    from hippymfem_b200.shard import DeviceSlabOps, ShardedHessian, SlabPartition
    from oracle import q2

    n, L = (6, 5, 7), (1.0, 0.8, 1.3)
    mo = q2.Lattice(n, L)
    rng = np.random.default_rng(43)
    u, p = rng.standard_normal(mo.ndof), rng.standard_normal(mo.ndof)
    m = 0.4 * rng.standard_normal(mo.ndof)
    x = rng.standard_normal(mo.ndof)
    ess = np.zeros(mo.ndof, np.int32)
    ess[mo.boundary_dofs()] = 1
    pts = 0.05 + 0.9 * rng.random((30, 3)) * np.asarray(L)
    part = SlabPartition(n, L, 1)
    shape = (mo.N[2], -1)
    own = [torch.as_tensor(a.reshape(shape).copy(), device=cuda) for a in (u, m, p, ess, x)]
    ops = DeviceSlabOps(part, 0, pts, 1e-3, cuda)
    H = ShardedHessian(part, 0, ops, *own[:4], rtol=1e-13)
    y = H.mult(own[4]).reshape(-1).cpu().numpy()
    E = mo.edofs()
    nd = mo.ndof
    mask = ess.astype(bool)
    pat = q2.build_tables(E, E, nd, nd, True)
    blk = q2.element_blocks(mo, E, u, m, p)
    blocks = {k: q2.csr(pat, q2.assemble_block(k, pat, blk[k], mask), (nd, nd)) for k in blk}
    B = q2.observation_matrix(mo, pts)
    yref, _ = q2.hessian_apply(blocks, x, np.flatnonzero(mask), Wuu=(B.T @ B) / 1e-3, rtol=1e-13)
    assert np.linalg.norm(y - yref) <= 1e-9 * np.linalg.norm(yref)
