"""The device-built pointwise observation operator B and the deterministic CSR
transpose against the oracle's B (pointwiseObservation.py:94-170 restated) and scipy's
transpose.  GPU."""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from oracle import q2

pytestmark = pytest.mark.gpu


def _host_rows(mesh, pts):
    """The same formulas on the host (the basis products in the device's order)."""
    h = np.asarray(mesh.h)
    n = np.asarray(mesh.n)
    s = pts / h
    e = np.clip(np.floor(s), 0, n - 1)
    t = s - e
    b = np.stack([2.0 * (t - 0.5) * (t - 1.0), -4.0 * t * (t - 1.0), 2.0 * t * (t - 0.5)], -1)
    a = np.arange(27)
    a1, a2, a3 = a % 3, (a // 3) % 3, a // 9
    e = e.astype(np.int64)
    Nx, Ny, _ = mesh.N
    cols = (2 * e[:, 0:1] + a1) + Nx * ((2 * e[:, 1:2] + a2) + Ny * (2 * e[:, 2:3] + a3))
    vals = (b[:, 0, :][:, a1] * b[:, 1, :][:, a2]) * b[:, 2, :][:, a3]
    return cols, vals


@pytest.mark.parametrize("n,L", [((4, 3, 5), (1.0, 0.7, 1.3)), ((16, 16, 16), (1.0, 1.0, 1.0))])
def test_rows_match_oracle_and_host_formulas(cuda, n, L):
    from hippymfem_b200 import BoxMesh, device_observation_operator

    mesh = BoxMesh(n, L)
    rng = np.random.default_rng(3)
    pts = rng.random((500, 3)) * np.asarray(L)
    # targets on nodes, faces and the far corner of the box
    pts[:3] = [[0.0, 0.0, 0.0], list(L), [L[0] / 2, 0.0, L[2]]]
    pts[3:6, 0] = np.asarray(mesh.h[0]) * np.array([1, 2, 3])
    B = device_observation_operator(mesh, pts)
    assert B.shape == (500, mesh.ndof)
    indptr = B.indptr.cpu().numpy()
    cols = B.indices.cpu().numpy().reshape(-1, 27)
    vals = B.values.cpu().numpy().reshape(-1, 27)
    assert np.array_equal(indptr, 27 * np.arange(501))
    assert np.all(np.diff(cols, axis=1) > 0)
    hc, hv = _host_rows(mesh, pts)
    assert np.array_equal(cols, hc)
    assert np.array_equal(vals, hv)          # bit for bit: no contraction on the device
    mo = q2.Lattice(n, L)
    ref = q2.observation_matrix(mo, pts).toarray()
    got = B.to_scipy().toarray()
    assert np.abs(got - ref).max() <= 1e-14
    assert np.allclose(got.sum(axis=1), 1.0, atol=1e-13)   # partition of unity


def test_targets_outside_raise(cuda):
    from hippymfem_b200 import BoxMesh, device_observation_operator

    mesh = BoxMesh((3, 3, 3))
    with pytest.raises(ValueError, match="outside the mesh"):
        device_observation_operator(mesh, [[0.5, 0.5, 0.5], [0.5, 1.5, 0.5]])
    with pytest.raises(ValueError, match="outside the mesh"):
        device_observation_operator(mesh, [[np.nan, 0.5, 0.5]])


@pytest.mark.parametrize("shape,density", [((300, 4000), 0.01), ((1, 7), 1.0), ((50, 60), 0.0)])
def test_transpose_matches_scipy_and_is_deterministic(cuda, shape, density):
    from hippymfem_b200 import DeviceCSR

    M = sp.random(*shape, density=density, format="csr", random_state=1)
    M.sort_indices()
    D = DeviceCSR(M, cuda)
    T1, T2 = D.transpose(), D.transpose()
    ref = M.T.tocsr()
    ref.sort_indices()
    assert T1.shape == ref.shape
    for T in (T1, T2):
        assert np.array_equal(T.indptr.cpu().numpy(), ref.indptr)
        assert np.array_equal(T.indices.cpu().numpy(), ref.indices)
        assert np.array_equal(T.values.cpu().numpy(), ref.data)


def test_misfit_gradient_uses_the_transpose(cuda):
    """grad_u of the pointwise misfit = B^T (B u - d) / sigma^2 against the host B."""
    from hippymfem_b200 import BoxMesh, PointwiseStateObservation, Q2Space
    from hippymfem_b200.problem import STATE
    from hippymfem_b200.synthetic import interior_points

    mesh = BoxMesh((8, 7, 6))
    V = Q2Space(mesh)
    pts = interior_points(300, seed=4)
    rng = np.random.default_rng(5)
    d = rng.standard_normal(300)
    mis = PointwiseStateObservation(V, pts, data=d, noise_variance=0.04)
    u = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
    g = V.vector()
    mis.grad(STATE, [u, None, None], g)
    Bh = q2.observation_matrix(q2.Lattice((8, 7, 6)), pts)
    ref = Bh.T @ (Bh @ u.cpu().numpy() - d) / 0.04
    assert np.abs(g.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("missing", ["warn", "ignore"])
def test_targets_outside_are_left_out_on_request(cuda, capsys, missing):
    """missing="warn"/"ignore": B has a row per target inside the box, in target order
    (pointwiseObservation.py:104-112); "warn" prints the reference's message."""
    from hippymfem_b200 import BoxMesh, PointwiseStateObservation, Q2Space, device_observation_operator

    mesh = BoxMesh((4, 3, 5), (1.0, 0.7, 1.3))
    rng = np.random.default_rng(8)
    pts = rng.random((40, 3)) * np.array([1.0, 0.7, 1.3])
    pts[[3, 17, 30]] = [[1.5, 0.1, 0.1], [0.2, -0.1, 0.3], [np.nan, 0.2, 0.2]]
    B = device_observation_operator(mesh, pts, missing=missing)
    keep = np.setdiff1d(np.arange(40), [3, 17, 30])
    assert np.array_equal(B.owned_targets, keep)
    ref = device_observation_operator(mesh, pts[keep])
    assert B.shape == (37, mesh.ndof)
    assert np.array_equal(B.indices.cpu().numpy(), ref.indices.cpu().numpy())
    assert np.array_equal(B.values.cpu().numpy(), ref.values.cpu().numpy())
    out = capsys.readouterr().out
    assert ("3 observation target(s) are outside the mesh" in out) == (missing == "warn")
    mis = PointwiseStateObservation(Q2Space(mesh), pts, data=np.zeros(37), noise_variance=1.0,
                                    missing=missing)
    assert mis.B.shape == (37, mesh.ndof)
    with pytest.raises(ValueError, match="missing must be"):
        device_observation_operator(mesh, pts, missing="drop")
