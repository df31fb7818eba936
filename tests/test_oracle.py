"""The oracle pinned: against the reference's own pattern code (golden fixtures), exact
integrals, AD of the density and finite differences.  CPU only."""

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle import ad, q2


@pytest.mark.parametrize("name", golden_cases())
def test_pattern_matches_reference_golden(name):
    """Same arrays, dtypes and nnz as the reference's numba passes produced
    (test_assembly.py:135 compares the sort-free and sorted routes the same way)."""
    z = load_golden(name)
    got = q2.build_tables(z["tdofs"], z["cdofs"], int(z["nrow"]), int(z["ncol"]),
                          bool(z["diag_first"]))
    for a, key in zip(got[:3], ("indptr", "indices", "slot")):
        assert a.dtype == z[key].dtype, key
        assert np.array_equal(a, z[key]), key
    assert got[3] == int(z["nnz"])


def test_pattern_rows_lead_with_diagonal():
    z = load_golden("pattern_q2_lattice_3x2x4.npz")
    indptr, indices = z["indptr"], z["indices"]
    rows = np.arange(len(indptr) - 1)
    assert np.array_equal(indices[indptr[:-1]], rows)
    for r in rows[:50]:
        rest = indices[indptr[r] + 1:indptr[r + 1]]
        assert np.all(np.diff(rest) > 0)


def _point(mesh, seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    u, m, p = (rng.standard_normal(mesh.ndof) for _ in range(3))
    return u, scale * m, p


def test_blocks_match_ad():
    mesh = q2.Lattice((2, 3, 2), L=(1.0, 0.7, 1.3))
    E = mesh.edofs()
    u, m, p = _point(mesh)
    cf = q2.element_blocks(mesh, E, u, m, p)
    adb = ad.element_blocks(mesh, E, u, m, p)
    for k in cf:
        assert np.abs(cf[k] - adb[k]).max() <= 1e-13 * np.abs(cf[k]).max(), k
    cv = q2.element_vectors(mesh, E, u, m, p)
    av = ad.element_vectors(mesh, E, u, m, p)
    for s in range(3):
        assert np.abs(cv[s] - av[s]).max() <= 1e-13 * np.abs(cv[s]).max()


def test_constant_coefficient_stiffness_is_exact():
    """At m = 0 the 3-point rule integrates Q2 gradients exactly: A is the tensor
    product of the 1D mass and stiffness matrices (test_kernels.py:90-139 pins A
    against MFEM's DiffusionIntegrator the same way)."""
    mesh = q2.Lattice((2, 2, 3), L=(1.0, 2.0, 0.5))
    E = mesh.edofs()
    u, _, p = _point(mesh)
    A = q2.element_blocks(mesh, E, u, np.zeros(mesh.ndof), p, which=("A",))["A"]
    M1 = lambda h: h / 30 * np.array([[4, 2, -1], [2, 16, 2], [-1, 2, 4.0]])
    K1 = lambda h: 1 / (3 * h) * np.array([[7, -8, 1], [-8, 16, -8], [1, -8, 7.0]])
    hx, hy, hz = mesh.h
    Aex = (np.kron(M1(hz), np.kron(M1(hy), K1(hx))) + np.kron(M1(hz), np.kron(K1(hy), M1(hx)))
           + np.kron(K1(hz), np.kron(M1(hy), M1(hx))))
    assert np.abs(A - Aex[None]).max() <= 1e-14 * np.abs(Aex).max()


def test_assembled_properties():
    """Row sums of A vanish before elimination (constants are in its kernel,
    test_modeling.py:1280-1300); A and Wmm are symmetric; the elimination leaves a unit
    diagonal on the boundary rows of A."""
    mesh = q2.Lattice((3, 3, 2))
    E = mesh.edofs()
    u, m, p = _point(mesh)
    pat = q2.build_tables(E, E, mesh.ndof, mesh.ndof, True)
    blk = q2.element_blocks(mesh, E, u, m, p)
    A = q2.csr(pat, q2.scatter(pat[2], blk["A"], pat[3]), (mesh.ndof,) * 2)
    assert np.abs(A @ np.ones(mesh.ndof)).max() <= 1e-13 * abs(A).max()
    assert abs(A - A.T).max() <= 1e-15 * abs(A).max()
    Wmm = q2.csr(pat, q2.scatter(pat[2], blk["Wmm"], pat[3]), (mesh.ndof,) * 2)
    assert abs(Wmm - Wmm.T).max() <= 1e-15 * abs(Wmm).max()
    ess = np.zeros(mesh.ndof, bool)
    ess[mesh.boundary_dofs()] = True
    Ae = q2.csr(pat, q2.assemble_block("A", pat, blk["A"], ess), (mesh.ndof,) * 2)
    d = Ae.diagonal()
    assert np.all(d[ess] == 1.0)
    Ae = Ae.tolil()
    for r in np.flatnonzero(ess)[:20]:
        row = Ae.getrow(r).toarray().ravel()
        assert row[r] == 1.0 and np.count_nonzero(row) == 1


def _assembled_residual(mesh, E, u, m, p, slot):
    v = q2.element_vectors(mesh, E, u, m, p)[slot]
    return q2.assemble_vector(E, v, mesh.ndof)


def test_blocks_by_finite_differences():
    """A = d(residual)/du, C = d(residual)/dm by central differences, h = 1e-6, relative
    tolerance 1e-7 (test_kernels.py:377-451)."""
    mesh = q2.Lattice((2, 2, 2))
    E = mesh.edofs()
    u, m, p = _point(mesh, 1)
    pat = q2.build_tables(E, E, mesh.ndof, mesh.ndof, True)
    blk = q2.element_blocks(mesh, E, u, m, p)
    A = q2.csr(pat, q2.scatter(pat[2], blk["A"], pat[3]), (mesh.ndof,) * 2)
    C = q2.csr(pat, q2.scatter(pat[2], blk["C"], pat[3]), (mesh.ndof,) * 2)
    Wum = q2.csr(pat, q2.scatter(pat[2], blk["Wum"], pat[3]), (mesh.ndof,) * 2)
    Wmm = q2.csr(pat, q2.scatter(pat[2], blk["Wmm"], pat[3]), (mesh.ndof,) * 2)
    rng = np.random.default_rng(5)
    d = rng.standard_normal(mesh.ndof)
    h = 1e-6
    ADJ, PAR, STA = q2.ADJOINT, q2.PARAMETER, q2.STATE
    fd = (_assembled_residual(mesh, E, u + h * d, m, p, ADJ)
          - _assembled_residual(mesh, E, u - h * d, m, p, ADJ)) / (2 * h)
    assert np.linalg.norm(fd - A @ d) <= 1e-7 * np.linalg.norm(A @ d)
    fd = (_assembled_residual(mesh, E, u, m + h * d, p, ADJ)
          - _assembled_residual(mesh, E, u, m - h * d, p, ADJ)) / (2 * h)
    assert np.linalg.norm(fd - C @ d) <= 1e-7 * np.linalg.norm(C @ d)
    fd = (_assembled_residual(mesh, E, u, m + h * d, p, STA)
          - _assembled_residual(mesh, E, u, m - h * d, p, STA)) / (2 * h)
    assert np.linalg.norm(fd - Wum @ d) <= 1e-7 * np.linalg.norm(Wum @ d)
    fd = (_assembled_residual(mesh, E, u, m + h * d, p, PAR)
          - _assembled_residual(mesh, E, u, m - h * d, p, PAR)) / (2 * h)
    assert np.linalg.norm(fd - Wmm @ d) <= 1e-7 * np.linalg.norm(Wmm @ d)


def test_hessian_action_by_finite_differences():
    """The restated TrueHessian against central differences of the reduced gradient
    (FDHessian, reducedHessian.py:133), on a 3^3 mesh with a pointwise misfit."""
    mesh = q2.Lattice((3, 3, 3))
    E = mesh.edofs()
    nd = mesh.ndof
    ess = mesh.boundary_dofs()
    essm = np.zeros(nd, bool)
    essm[ess] = True
    pat = q2.build_tables(E, E, nd, nd, True)
    rng = np.random.default_rng(3)
    B = q2.observation_matrix(mesh, 0.1 + 0.8 * rng.random((40, 3)))
    data = rng.standard_normal(40)
    nv = 0.5
    f = 1.0

    def solve_state(m):
        z = np.zeros(nd)
        blk = q2.element_blocks(mesh, E, z, m, z, which=("A",))
        A = q2.csr(pat, q2.assemble_block("A", pat, blk["A"], essm), (nd, nd))
        r = _assembled_residual(mesh, E, z, m, z, q2.ADJOINT)
        r[ess] = 0.0
        import scipy.sparse.linalg as spl
        return spl.spsolve(A.tocsc(), -r), A

    def gradient(m):
        import scipy.sparse.linalg as spl
        u, A = solve_state(m)
        rhs = -(B.T @ (B @ u - data)) / nv
        rhs[ess] = 0.0
        p = spl.spsolve(A.tocsc(), rhs)
        return _assembled_residual(mesh, E, u, m, p, q2.PARAMETER), u, p

    m0 = 0.2 * rng.standard_normal(nd)
    g0, u0, p0 = gradient(m0)
    blk = q2.element_blocks(mesh, E, u0, m0, p0)
    blocks = {k: q2.csr(pat, q2.assemble_block(k, pat, blk[k], essm), (nd, nd)) for k in blk}
    x = rng.standard_normal(nd)
    Hx, _ = q2.hessian_apply(blocks, x, ess, Wuu=(B.T @ B) / nv, rtol=1e-13)
    h = 1e-5
    fd = (gradient(m0 + h * x)[0] - gradient(m0 - h * x)[0]) / (2 * h)
    assert np.linalg.norm(fd - Hx) <= 1e-6 * np.linalg.norm(Hx)


def test_consistent_blocks_are_exact_on_the_constants():
    """consistent_block (kernel.py:1503-1571) restated: the single-precision element
    matrices err by ~1e-7; corrected, their products with the constants (and, two-sided,
    their transposes') equal the double-precision ones to rounding, A and W_mm are
    symmetric to the last bit, and the entries stay within the single-precision error."""
    mesh = q2.Lattice((3, 4, 2), (1.0, 0.8, 1.1))
    E = mesh.edofs()
    rng = np.random.default_rng(12)
    u, p = rng.standard_normal(mesh.ndof), rng.standard_normal(mesh.ndof)
    m = 0.5 * rng.standard_normal(mesh.ndof)
    K64 = q2.element_blocks(mesh, E, u, m, p)
    K32 = q2.element_blocks_fp32(mesh, E, u, m, p)
    Kc = q2.consistent_blocks(mesh, E, u, m, p)
    one = np.ones(27)
    for name in ("A", "C", "Wum", "Wmm"):
        scale = np.abs(K64[name]).max()
        err32 = np.abs(K32[name] - K64[name]).max() / scale
        assert 1e-9 < err32 < 1e-5, (name, err32)              # single precision
        assert np.abs(Kc[name] - K64[name]).max() / scale < 10 * err32
        d64 = K64[name] @ one
        assert np.abs(Kc[name] @ one - d64).max() <= 1e-13 * scale, name
        if name in q2.SYMMETRIC_BLOCKS:
            assert np.array_equal(Kc[name], Kc[name].transpose(0, 2, 1)), name
        else:
            t64 = K64[name].transpose(0, 2, 1) @ one
            assert np.abs(Kc[name].transpose(0, 2, 1) @ one - t64).max() <= 1e-13 * scale
        # the uncorrected block's row sums carry its single-precision error
        assert np.abs(K32[name] @ one - d64).max() > 1e3 * np.abs(Kc[name] @ one - d64).max()


def test_assembled_rows_equal_the_whole_mesh_assembly():
    """The row-restricted oracle (used to check the 64^3 benchmark assembly on a sample of
    its rows) gives exactly the rows of the whole-mesh scatter, elimination and vector
    assembly."""
    mesh = q2.Lattice((4, 3, 5), (1.0, 0.7, 1.3))
    E = mesh.edofs()
    nd = mesh.ndof
    rng = np.random.default_rng(21)
    u, m, p = rng.standard_normal(nd), 0.3 * rng.standard_normal(nd), rng.standard_normal(nd)
    ess = np.zeros(nd, bool)
    ess[mesh.boundary_dofs()] = True
    pat = q2.build_tables(E, E, nd, nd, True)
    blk = q2.element_blocks(mesh, E, u, m, p)
    ev = q2.element_vectors(mesh, E, u, m, p, 1.3)
    rows = np.unique(np.concatenate([rng.choice(nd, 60, replace=False), mesh.boundary_dofs()[:9]]))
    got_b, got_v = q2.assembled_rows(mesh, u, m, p, rows, ess, 1.3)
    row_of = np.repeat(np.arange(nd), np.diff(pat[0]))
    sel = np.isin(row_of, rows)
    keys = row_of[sel] * nd + pat[1][sel]
    order = np.argsort(keys)
    for name in ("A", "C", "Wum", "Wmm"):
        full = q2.assemble_block(name, pat, blk[name], ess)
        assert np.array_equal(got_b[name][0], keys[order]), name
        assert np.array_equal(got_b[name][1], full[sel][order]), name
    for s in range(3):
        assert np.array_equal(got_v[s], q2.assemble_vector(E, ev[s], nd)[rows]), s


def test_boundary_mass_known_answers():
    """The oracle's boundary mass: symmetric, int 1 ds = |boundary|, int x^2 ds by faces."""
    mo = q2.Lattice((3, 2, 4), (1.0, 0.7, 1.3))
    B = q2.boundary_mass(mo)
    assert abs(B - B.T).max() <= 1e-16
    one = np.ones(mo.ndof)
    area = 2 * (1.0 * 0.7 + 0.7 * 1.3 + 1.0 * 1.3)
    assert abs(one @ (B @ one) - area) <= 1e-13 * area
    x = mo.node_coords()[:, 0]
    want = 0.7 * 1.3 + 2 * 1.3 / 3 + 2 * 0.7 / 3       # x = 1 face, then the y and z faces
    assert abs(x @ (B @ x) - want) <= 1e-13 * want
