"""The constant-exact single-precision blocks (consistent_block, kernel.py:1503-1571) on
the device against the oracle's restatement.  GPU.

The corrected FP32 blocks must be exact on the constants to FP64 rounding -- the
assembled A annihilates them (1e-13 relative), and C, Wum, Wmm reproduce the FP64
blocks' row and column sums -- while every entry stays within the single-precision
error of the FP64 block and within it of the oracle's consistent blocks; A and Wmm are
symmetric to the bit; the folded elimination is the fused kernel's.
"""

import numpy as np
import pytest
import torch

from oracle import q2

pytestmark = pytest.mark.gpu

BLOCKS = ("A", "C", "Wum", "Wmm")


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _run(mesh, u, m, p, marker=None):
    from hippymfem_b200 import LatticePattern
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    dev = mesh.device
    pat = LatticePattern(mesh, with_transpose=True)
    U, M, P = (torch.as_tensor(v, device=dev) for v in (u, m, p))
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(U), ptr(M), ptr(P), _lib.HM_FP64, ptr(quad),
                                    ptr(status), stream_ptr()))
    work = torch.empty(lib.hm_lattice_consistent_workspace_bytes(mesh.handle) // 8,
                       dtype=torch.float64, device=dev)
    cons = {b: torch.full((mesh.nnz,), float("nan"), dtype=torch.float64, device=dev)
            for b in BLOCKS}
    check(lib.hm_lattice_assemble_consistent(mesh.handle, ptr(quad), ptr(marker),
                                             *(ptr(cons[b]) for b in BLOCKS), ptr(work),
                                             stream_ptr()), "hm_lattice_assemble_consistent")
    f64 = {b: pat.new_values() for b in BLOCKS}
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr),
                                  ptr(marker), 1.0, *(ptr(f64[b]) for b in BLOCKS),
                                  None, None, None, 0, stream_ptr()))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return pat, {b: v.cpu().numpy() for b, v in cons.items()}, \
        {b: v.cpu().numpy() for b, v in f64.items()}


def test_consistent_blocks_are_exact_on_the_constants(cuda):
    from hippymfem_b200 import BoxMesh

    n, L = (5, 4, 6), (1.0, 0.8, 1.2)
    mesh = BoxMesh(n, L)
    mo = q2.Lattice(n, L)
    rng = np.random.default_rng(31)
    u, p = rng.standard_normal(mesh.ndof), rng.standard_normal(mesh.ndof)
    m = 0.6 * rng.standard_normal(mesh.ndof)
    pat, cons, f64 = _run(mesh, u, m, p)
    ip = pat.indptr.cpu().numpy().astype(np.int64)
    ind = pat.indices.cpu().numpy()
    tpos = pat.tpos.cpu().numpy()
    row_of = np.repeat(np.arange(mesh.ndof), np.diff(ip))
    E = mo.edofs()
    ptab = q2.build_tables(E, E, mesh.ndof, mesh.ndof, True)
    ocons = q2.consistent_blocks(mo, E, u, m, p)
    o32 = q2.element_blocks_fp32(mo, E, u, m, p)
    for b in BLOCKS:
        c, r = cons[b], f64[b]
        assert np.isfinite(c).all(), b
        scale = np.abs(r).max()
        rows_c = np.bincount(row_of, weights=c, minlength=mesh.ndof)
        rows_r = np.bincount(row_of, weights=r, minlength=mesh.ndof)
        cols_c = np.bincount(ind, weights=c, minlength=mesh.ndof)
        cols_r = np.bincount(ind, weights=r, minlength=mesh.ndof)
        assert np.abs(rows_c - rows_r).max() <= 1e-13 * scale, (b, "rows")
        assert np.abs(cols_c - cols_r).max() <= 1e-13 * scale, (b, "columns")
        if b == "A":
            assert np.abs(rows_c).max() <= 1e-13 * scale
        # within single precision of FP64 and of the oracle's consistent blocks
        ref = q2.scatter(ptab[2], ocons[b], ptab[3])
        plain = q2.scatter(ptab[2], o32[b], ptab[3])
        err32 = _rel(plain, r)
        assert _rel(c, r) <= 10 * err32 + 1e-12, (b, _rel(c, r), err32)
        assert _rel(c, ref) <= 10 * err32 + 1e-12, (b, _rel(c, ref))
        # the plain single-precision block misses the constants by its rounding
        rows_p = np.bincount(row_of, weights=plain, minlength=mesh.ndof)
        assert np.abs(rows_p - rows_r).max() > 1e3 * np.abs(rows_c - rows_r).max() + 1e-300, b
    for b in ("A", "Wmm"):
        assert np.array_equal(cons[b], cons[b][tpos]), b


def test_consistent_blocks_elimination(cuda):
    from hippymfem_b200 import BoxMesh, DirichletBC, Q2Space

    n = (4, 5, 3)
    mesh = BoxMesh(n)
    rng = np.random.default_rng(32)
    u, m, p = rng.standard_normal(mesh.ndof), 0.3 * rng.standard_normal(mesh.ndof), \
        rng.standard_normal(mesh.ndof)
    marker = DirichletBC(Q2Space(mesh)).marker
    pat, free, _ = _run(mesh, u, m, p)
    _, elim, _ = _run(mesh, u, m, p, marker)
    ess = marker.cpu().numpy().astype(bool)
    ip = pat.indptr.cpu().numpy().astype(np.int64)
    ind = pat.indices.cpu().numpy()
    row_of = np.repeat(np.arange(mesh.ndof), np.diff(ip))
    for b in BLOCKS:
        want = free[b].copy()
        rows, cols, diag = q2.ELIMINATION[b]
        kill = np.zeros_like(want, dtype=bool)
        if rows:
            kill |= ess[row_of]
        if cols:
            kill |= ess[ind]
        want[kill] = 0.0
        if diag is not None:
            want[kill & (row_of == ind) & ess[row_of]] = diag
        assert np.array_equal(elim[b], want), b
