"""The fused CUDA assembly against the oracle: every block and vector of a
linearization point, with and without the folded elimination, FP64 to 1e-12 relative,
bit-reproducible; the FP32 variant within its stated bound.  GPU."""

import numpy as np
import pytest
import torch

from oracle import q2

pytestmark = pytest.mark.gpu

BLOCKS = ("A", "C", "Wum", "Wmm")
TOL = 1e-12          # FP64 values, relative to the block's largest entry
TOL_FP32 = 2e-5      # FP32 contractions, FP64 values


def _point(nd, seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    u, m, p = (rng.standard_normal(nd) for _ in range(3))
    return u, scale * m, p


def _device_assemble(mesh, pat, u, m, p, ess=None, f=1.0, precision=0, blocks=BLOCKS,
                     vectors=(0, 1, 2), zero_ess=False):
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    dev = mesh.device
    U, M, P = (torch.as_tensor(v, device=dev) for v in (u, m, p))
    quad = torch.empty(mesh.quad_bytes(precision) // 8, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(U), ptr(M), ptr(P), precision, ptr(quad),
                                    ptr(status), stream_ptr()))
    vals = {b: torch.full((mesh.nnz,), np.nan, dtype=torch.float64, device=dev) for b in blocks}
    vecs = {s: torch.full((mesh.ndof,), np.nan, dtype=torch.float64, device=dev) for s in vectors}
    marker = mesh.ess_marker(ess) if ess is not None else None
    check(lib.hm_lattice_assemble(
        mesh.handle, ptr(quad), precision, ptr(pat.indptr), ptr(marker), float(f),
        ptr(vals.get("A")), ptr(vals.get("C")), ptr(vals.get("Wum")), ptr(vals.get("Wmm")),
        ptr(vecs.get(0)), ptr(vecs.get(1)), ptr(vecs.get(2)), int(zero_ess), stream_ptr()))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return ({b: v.cpu().numpy() for b, v in vals.items()},
            {s: v.cpu().numpy() for s, v in vecs.items()}, quad)


def _oracle(mesh_o, u, m, p, ess_mask=None, f=1.0):
    E = mesh_o.edofs()
    pat = q2.build_tables(E, E, mesh_o.ndof, mesh_o.ndof, True)
    blk = q2.element_blocks(mesh_o, E, u, m, p)
    vals = {}
    for b in BLOCKS:
        if ess_mask is None:
            vals[b] = q2.scatter(pat[2], blk[b], pat[3])
        else:
            vals[b] = q2.assemble_block(b, pat, blk[b], ess_mask)
    ev = q2.element_vectors(mesh_o, E, u, m, p, f)
    vecs = {s: q2.assemble_vector(E, ev[s], mesh_o.ndof) for s in range(3)}
    return vals, vecs


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("n,L", [((4, 3, 5), (1.0, 0.7, 1.3)), ((1, 1, 1), (1.0, 1.0, 1.0)),
                                 ((2, 5, 1), (2.0, 1.0, 0.5)), ((8, 8, 8), (1.0, 1.0, 1.0))])
def test_blocks_and_vectors_match_oracle(cuda, n, L):
    from hippymfem_b200 import BoxMesh, LatticePattern

    mesh = BoxMesh(n, L)
    mo = q2.Lattice(n, L)
    pat = LatticePattern(mesh, with_transpose=False)
    u, m, p = _point(mesh.ndof, 1)
    vals, vecs, _ = _device_assemble(mesh, pat, u, m, p, f=1.7)
    rvals, rvecs = _oracle(mo, u, m, p, f=1.7)
    for b in BLOCKS:
        assert np.isfinite(vals[b]).all(), b
        assert _rel(vals[b], rvals[b]) <= TOL, (b, _rel(vals[b], rvals[b]))
    for s in range(3):
        assert _rel(vecs[s], rvecs[s]) <= TOL, (s, _rel(vecs[s], rvecs[s]))


def test_elimination_policies_match_oracle(cuda):
    """A: rows and columns of the Dirichlet dofs zeroed, unit diagonal; C and Wum rows
    zeroed; Wmm untouched (hippymfem/fem/bcs.py:13-30); vectors zeroed on request."""
    from hippymfem_b200 import BoxMesh, LatticePattern

    n = (5, 4, 3)
    mesh = BoxMesh(n)
    mo = q2.Lattice(n)
    pat = LatticePattern(mesh, with_transpose=False)
    u, m, p = _point(mesh.ndof, 2)
    ess = mo.boundary_dofs()
    mask = np.zeros(mesh.ndof, bool)
    mask[ess] = True
    vals, vecs, _ = _device_assemble(mesh, pat, u, m, p, ess=ess, zero_ess=True)
    rvals, rvecs = _oracle(mo, u, m, p, ess_mask=mask)
    for b in BLOCKS:
        assert _rel(vals[b], rvals[b]) <= TOL, b
    indptr = pat.indptr.cpu().numpy()
    assert np.all(vals["A"][indptr[ess]] == 1.0)
    for s in (0, 2):
        r = rvecs[s].copy()
        r[ess] = 0.0
        assert _rel(vecs[s], r) <= TOL
        assert np.all(vecs[s][ess] == 0.0)
    assert _rel(vecs[1], rvecs[1]) <= TOL


def test_benchmark_field_16_cubed(cuda):
    """The CPU-runnable configuration: 16^3, the seeded log-conductivity of the
    benchmark, u = 0 on the boundary."""
    from hippymfem_b200 import BoxMesh, LatticePattern
    from hippymfem_b200.synthetic import log_conductivity

    mesh = BoxMesh(16)
    mo = q2.Lattice(16)
    pat = LatticePattern(mesh, with_transpose=False)
    m = log_conductivity(mo.node_coords(), seed=0)
    u, _, p = _point(mesh.ndof, 3)
    ess = mo.boundary_dofs()
    mask = np.zeros(mesh.ndof, bool)
    mask[ess] = True
    vals, vecs, _ = _device_assemble(mesh, pat, u, m, p, ess=ess)
    rvals, rvecs = _oracle(mo, u, m, p, ess_mask=mask)
    for b in BLOCKS:
        assert _rel(vals[b], rvals[b]) <= TOL, b
    for s in range(3):
        assert _rel(vecs[s], rvecs[s]) <= TOL, s


def test_assembly_is_bit_reproducible(cuda):
    from hippymfem_b200 import BoxMesh, LatticePattern

    mesh = BoxMesh((6, 7, 5))
    pat = LatticePattern(mesh, with_transpose=False)
    u, m, p = _point(mesh.ndof, 4)
    a, va, _ = _device_assemble(mesh, pat, u, m, p)
    b, vb, _ = _device_assemble(mesh, pat, u, m, p)
    for k in BLOCKS:
        assert np.array_equal(a[k], b[k])
    for s in range(3):
        assert np.array_equal(va[s], vb[s])


@pytest.mark.parametrize("blocks", [(), ("C",), ("Wum", "Wmm"), BLOCKS])
def test_vectors_alone_and_with_their_blocks_agree(cuda, blocks):
    """A vector assembled with its block (the block's row sums) and alone (its own
    contractions), with the Dirichlet rows zeroed, against each other and the oracle."""
    from hippymfem_b200 import BoxMesh, LatticePattern

    n = (7, 6, 9)
    mesh = BoxMesh(n, (1.0, 0.8, 1.2))
    mo = q2.Lattice(n, (1.0, 0.8, 1.2))
    pat = LatticePattern(mesh, with_transpose=False)
    u, m, p = _point(mesh.ndof, 6)
    ess = mo.boundary_dofs()
    _, alone, _ = _device_assemble(mesh, pat, u, m, p, ess=ess, f=0.6, blocks=(), zero_ess=True)
    vals, mixed, _ = _device_assemble(mesh, pat, u, m, p, ess=ess, f=0.6, blocks=blocks,
                                      zero_ess=True)
    _, rvecs = _oracle(mo, u, m, p, f=0.6)
    for s in range(3):
        r = rvecs[s].copy()
        if s != 1:
            r[ess] = 0.0
        assert _rel(mixed[s], alone[s]) <= 1e-13, (s, _rel(mixed[s], alone[s]))
        assert _rel(mixed[s], r) <= TOL, s
    for b in blocks:
        assert np.isfinite(vals[b]).all(), b


def test_fp32_contractions_error_is_bounded(cuda):
    from hippymfem_b200 import BoxMesh, LatticePattern

    n = (6, 6, 6)
    mesh = BoxMesh(n)
    pat = LatticePattern(mesh, with_transpose=False)
    u, m, p = _point(mesh.ndof, 5)
    v64, w64, _ = _device_assemble(mesh, pat, u, m, p, precision=0)
    v32, w32, _ = _device_assemble(mesh, pat, u, m, p, precision=1)
    for b in BLOCKS:
        assert _rel(v32[b], v64[b]) <= TOL_FP32, (b, _rel(v32[b], v64[b]))
    for s in range(3):
        assert _rel(w32[s], w64[s]) <= TOL_FP32


def test_nonfinite_parameter_is_reported(cuda):
    """A non-finite value in the fields raises RuntimeError (require_finite_arrays)."""
    from hippymfem_b200 import (BoxMesh, DirichletBC, PARAMETER, PDEVariationalProblem,
                                Q2Space)

    mesh = BoxMesh(3)
    V = Q2Space(mesh)
    prob = PDEVariationalProblem([V, V, V], bc=DirichletBC(V))
    m = V.vector()
    m[5] = float("nan")
    with pytest.raises(RuntimeError):
        prob._residual([None, m, None], PARAMETER)


@pytest.mark.parametrize("with_mhat", [False, True])
def test_direct_vectors_match_the_oracle_and_the_tile_path(cuda, with_mhat):
    """hm_lattice_vectors (fields -> element vectors -> node gather, no pointwise data)
    against the oracle's assembled vectors and against the tile kernel's vector phases:
    the point's dR/du, dR/dm, dR/dp with the source, or the directional products C mhat,
    W_um mhat, W_mm mhat along mhat; zeroing on the Dirichlet nodes as asked."""
    from hippymfem_b200 import BoxMesh, DirichletBC, Q2Space
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    n, L = (5, 6, 4), (1.0, 0.9, 0.7)
    mesh = BoxMesh(n, L)
    mo = q2.Lattice(n, L)
    u, m, p = _point(mesh.ndof, 9)
    mh = np.random.default_rng(10).standard_normal(mesh.ndof)
    marker = DirichletBC(Q2Space(mesh)).marker
    U, M, P, MH = (torch.as_tensor(v, device=cuda) for v in (u, m, p, mh))
    f = 0.0 if with_mhat else 1.3
    work = torch.empty(lib.hm_lattice_vectors_workspace_bytes(mesh.handle, 3) // 8,
                       dtype=torch.float64, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    out = [torch.full((mesh.ndof,), float("nan"), dtype=torch.float64, device=cuda)
           for _ in range(3)]
    check(lib.hm_lattice_vectors(mesh.handle, ptr(U), ptr(M), ptr(P), ptr(MH) if with_mhat else None,
                                 f, ptr(marker), ptr(out[0]), ptr(out[1]), ptr(out[2]), 1,
                                 ptr(work), ptr(status), stream_ptr()), "hm_lattice_vectors")
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=cuda)
    if with_mhat:
        check(lib.hm_lattice_quadrature_dir(mesh.handle, ptr(U), ptr(M), ptr(P), ptr(MH),
                                            _lib.HM_FP64, ptr(quad), ptr(status), stream_ptr()))
    else:
        check(lib.hm_lattice_quadrature(mesh.handle, ptr(U), ptr(M), ptr(P), _lib.HM_FP64,
                                        ptr(quad), ptr(status), stream_ptr()))
    tile = [torch.empty(mesh.ndof, dtype=torch.float64, device=cuda) for _ in range(3)]
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, None, ptr(marker), f,
                                  None, None, None, None, ptr(tile[0]), ptr(tile[1]),
                                  ptr(tile[2]), 1, stream_ptr()))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    ess = mo.boundary_dofs()
    E = mo.edofs()
    if with_mhat:
        blk = q2.element_blocks(mo, E, u, m, p)
        pat = q2.build_tables(E, E, mo.ndof, mo.ndof, True)
        ref = {}
        for s, name in ((0, "Wum"), (1, "Wmm"), (2, "C")):
            M_ = q2.csr(pat, q2.scatter(pat[2], blk[name], pat[3]), (mo.ndof, mo.ndof))
            ref[s] = M_ @ mh
    else:
        ev = q2.element_vectors(mo, E, u, m, p, f)
        ref = {s: q2.assemble_vector(E, ev[s], mo.ndof) for s in range(3)}
    for s in range(3):
        r = ref[s].copy()
        if s != 1:
            r[ess] = 0.0
        got = out[s].cpu().numpy()
        assert _rel(got, r) <= TOL, (s, _rel(got, r))
        assert _rel(got, tile[s].cpu().numpy()) <= 1e-13, s
