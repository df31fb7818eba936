"""Parity at the benchmark configuration: the 64^3 Q2 lattice (262,144 elements,
2,146,689 dofs, 135,005,697 entries per block) with the benchmark's fields -- the seeded
log-conductivity (seed 0), u and p standard normal (seed 11), f = 1, the whole boundary
eliminated.  GPU.

* values: every block and vector on ~2000 rows covering every clipping class (corner,
  edge, face and interior nodes, both node parities, tile edges) against the oracle,
  which assembles those rows from the elements around them (``oracle.q2.assembled_rows``)
  -- 1e-12 relative to the block's largest sampled entry;
* pattern: the full ``indptr``/``indices`` against the host builder ``hm_pattern_build``
  on the lattice's element dof table (pinned to the reference's own pattern passes by
  the golden fixtures);
* size-independent properties over all rows: ``A`` annihilates the constants on every
  row whose stencil misses the boundary, ``A`` and ``Wmm`` are symmetric.
"""

import numpy as np
import pytest
import torch

from oracle import q2

pytestmark = pytest.mark.gpu

BLOCKS = ("A", "C", "Wum", "Wmm")
TOL = 1e-12
N = 64


def _sample_rows(nd, Nn, rng):
    """Rows of every clipping class: each axis at the two boundaries, the nodes next to
    them, a tile edge (4k / 4k + 3) and the middle, in all combinations; plus random rows."""
    axis = np.array([0, 1, 2, 3, 4, 7, 63, 64, Nn - 4, Nn - 3, Nn - 2, Nn - 1])
    i, j, k = np.meshgrid(axis, axis, axis, indexing="ij")
    classes = (i + Nn * (j + Nn * k)).reshape(-1)
    pick = rng.choice(classes, 1200, replace=False)
    rand = rng.choice(nd, 800, replace=False)
    return np.unique(np.concatenate([pick, rand]))


@pytest.fixture(scope="module")
def bench64(cuda):
    from hippymfem_b200 import BoxMesh, DirichletBC, LatticePattern, Q2Space
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.synthetic import log_conductivity

    mesh = BoxMesh(N, device=cuda)
    bc = DirichletBC(Q2Space(mesh))
    pat = LatticePattern(mesh, with_transpose=True)
    nd, nnz = mesh.ndof, mesh.nnz
    m_h = log_conductivity(mesh.node_coords(), seed=0)
    rng = np.random.default_rng(11)
    u_h, p_h = rng.standard_normal(nd), rng.standard_normal(nd)
    U, M, P = (torch.as_tensor(x, device=cuda) for x in (u_h, m_h, p_h))
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    vals = {b: torch.full((nnz,), float("nan"), dtype=torch.float64, device=cuda) for b in BLOCKS}
    vecs = [torch.full((nd,), float("nan"), dtype=torch.float64, device=cuda) for _ in range(3)]
    s = stream_ptr()
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(U), ptr(M), ptr(P), _lib.HM_FP64, ptr(quad),
                                    ptr(status), s))
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr),
                                  ptr(bc.marker), 1.0, *(ptr(vals[b]) for b in BLOCKS),
                                  *(ptr(v) for v in vecs), 0, s))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    del quad
    mo = q2.Lattice(N)
    ess = np.zeros(nd, bool)
    ess[mo.boundary_dofs()] = True
    return dict(mesh=mesh, mo=mo, pat=pat, vals=vals, vecs=vecs, u=u_h, m=m_h, p=p_h, ess=ess)


def test_sampled_rows_match_the_oracle_at_64_cubed(bench64):
    mesh, mo, pat = bench64["mesh"], bench64["mo"], bench64["pat"]
    nd = mesh.ndof
    rows = _sample_rows(nd, mo.N[0], np.random.default_rng(64))
    assert len(rows) >= 1900
    ip = pat.indptr.cpu().numpy().astype(np.int64)
    starts, ends = ip[rows], ip[rows + 1]
    pos = np.concatenate([np.arange(a, b) for a, b in zip(starts, ends)])
    row_of = np.repeat(rows, ends - starts)
    pos_d = torch.as_tensor(pos, device=pat.indices.device)
    cols = pat.indices[pos_d].cpu().numpy().astype(np.int64)
    keys = row_of * nd + cols
    order = np.argsort(keys)
    ref_b, ref_v = q2.assembled_rows(mo, bench64["u"], bench64["m"], bench64["p"], rows,
                                     bench64["ess"], 1.0)
    for b in BLOCKS:
        got = bench64["vals"][b][pos_d].cpu().numpy()
        rk, rv = ref_b[b]
        assert np.array_equal(keys[order], rk), b          # same columns in every row
        err = np.abs(got[order] - rv).max() / np.abs(rv).max()
        assert np.isfinite(got).all(), b
        assert err <= TOL, (b, err)
    rows_d = torch.as_tensor(rows, device=pat.indices.device)
    for s in range(3):
        got = bench64["vecs"][s][rows_d].cpu().numpy()
        err = np.abs(got - ref_v[s]).max() / np.abs(ref_v[s]).max()
        assert err <= TOL, (s, err)


def test_full_pattern_matches_the_host_build_at_64_cubed(bench64):
    from hippymfem_b200 import build_tables

    mesh, pat = bench64["mesh"], bench64["pat"]
    indptr, indices, _, nnz = build_tables(mesh.edofs(), mesh.edofs(), mesh.ndof, mesh.ndof)
    assert nnz == mesh.nnz == 135005697
    assert np.array_equal(pat.indptr.cpu().numpy(), indptr)
    assert np.array_equal(pat.indices.cpu().numpy(), indices)


def test_properties_over_all_rows_at_64_cubed(bench64):
    """A times the constants vanishes on every row whose columns avoid the boundary (the
    constants are in the kernel of the un-eliminated operator); A and Wmm are symmetric
    (A^T == A is what the problem layer relies on)."""
    mesh, pat, vals = bench64["mesh"], bench64["pat"], bench64["vals"]
    dev = pat.indptr.device
    ip = pat.indptr.long()
    counts = ip[1:] - ip[:-1]
    row_of = torch.repeat_interleave(torch.arange(mesh.ndof, device=dev), counts)
    ess = torch.as_tensor(bench64["ess"], device=dev)
    touches = torch.zeros(mesh.ndof, dtype=torch.int32, device=dev).index_add_(
        0, row_of, ess[pat.indices.long()].int()) > 0
    A = vals["A"]
    rowsum = torch.zeros(mesh.ndof, dtype=torch.float64, device=dev).index_add_(0, row_of, A)
    scale = A.abs().max()
    free = ~touches
    assert int(free.sum()) > 0.8 * mesh.ndof
    assert float(rowsum[free].abs().max() / scale) <= 1e-13
    tpos = pat.tpos.long()
    for b in ("A", "Wmm"):
        v = vals[b]
        err = float((v - v[tpos]).abs().max() / v.abs().max())
        assert err <= 1e-14, (b, err)
