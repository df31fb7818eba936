"""The device lattice pattern against the reference's arrays (golden) and the host
build; the transpose map.  GPU."""

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import q2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 2, 2), (3, 2, 4), (4, 4, 4)])
def test_lattice_pattern_matches_reference_golden(cuda, n):
    from hippymfem_b200 import BoxMesh, LatticePattern

    z = load_golden("pattern_q2_lattice_%dx%dx%d.npz" % n)
    mesh = BoxMesh(n)
    pat = LatticePattern(mesh, with_slot=True)
    torch.cuda.synchronize()
    assert pat.nnz == int(z["nnz"])
    for t, key in ((pat.indptr, "indptr"), (pat.indices, "indices"), (pat.slot, "slot")):
        a = t.cpu().numpy()
        assert a.dtype == z[key].dtype, key
        assert np.array_equal(a, z[key]), key


@pytest.mark.parametrize("n", [(5, 3, 7), (9, 8, 6)])
def test_lattice_pattern_matches_host_build(cuda, n):
    from hippymfem_b200 import BoxMesh, LatticePattern, build_tables

    mesh = BoxMesh(n)
    pat = LatticePattern(mesh, with_slot=True)
    E = mesh.edofs()
    ref = build_tables(E, E, mesh.ndof, mesh.ndof)
    assert np.array_equal(pat.indptr.cpu().numpy(), ref[0])
    assert np.array_equal(pat.indices.cpu().numpy(), ref[1])
    assert np.array_equal(pat.slot.cpu().numpy(), ref[2])
    assert pat.nnz == ref[3] == mesh.nnz


def test_transpose_map(cuda):
    from hippymfem_b200 import BoxMesh, LatticePattern

    mesh = BoxMesh((4, 5, 3))
    pat = LatticePattern(mesh)
    indptr = pat.indptr.cpu().numpy().astype(np.int64)
    indices = pat.indices.cpu().numpy()
    tpos = pat.tpos.cpu().numpy()
    rows = np.repeat(np.arange(mesh.ndof), np.diff(indptr))
    # entry tpos[s] is (col(s), row(s))
    assert np.array_equal(indices[tpos], rows)
    assert np.array_equal(rows[tpos], indices)
    assert np.array_equal(np.sort(tpos), np.arange(mesh.nnz))


def test_pattern_64_cubed_counts(cuda):
    """The benchmark size: nnz = 513^3, every row's diagonal first."""
    from hippymfem_b200 import BoxMesh, LatticePattern

    mesh = BoxMesh(64)
    pat = LatticePattern(mesh, with_transpose=False)
    assert pat.nnz == 135005697
    ip = pat.indptr
    assert int(ip[-1]) == pat.nnz
    rows = torch.arange(mesh.ndof, device=ip.device, dtype=torch.int64)
    assert torch.equal(pat.indices[ip[:-1].long()].long(), rows)
