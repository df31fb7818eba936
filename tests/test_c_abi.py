"""The C ABI without a GPU: the library loads, exports every declared entry point, and
its host pattern build reproduces the reference's arrays.  CPU only."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_cases, load_golden
from oracle import q2

HEADER = os.path.join(ROOT, "include", "hippymfem_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hm_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from hippymfem_b200 import _lib

    names = declared_symbols()
    assert len(names) >= 18
    for n in names:
        assert hasattr(_lib.lib, n), n
        assert n in _lib.SIGNATURES, "no ctypes signature for %s" % n
    assert _lib.lib.hm_version() >= 100
    assert _lib.lib.hm_error_string(1).decode().startswith("invalid")


@pytest.mark.parametrize("name", golden_cases())
def test_host_pattern_build_matches_reference_golden(name):
    from hippymfem_b200.pattern import build_tables

    z = load_golden(name)
    got = build_tables(z["tdofs"], z["cdofs"], int(z["nrow"]), int(z["ncol"]),
                       bool(z["diag_first"]), nthreads=3)
    for a, key in zip(got[:3], ("indptr", "indices", "slot")):
        assert a.dtype == z[key].dtype, key
        assert np.array_equal(a, z[key]), key
    assert got[3] == int(z["nnz"])


def test_host_pattern_build_large_lattice_matches_oracle():
    from hippymfem_b200.pattern import build_tables

    mesh = q2.Lattice((6, 5, 7))
    E = mesh.edofs()
    rng = np.random.default_rng(1)
    perm = rng.permutation(mesh.ndof)
    E = perm[E]                                  # an arbitrary global numbering
    got = build_tables(E, E, mesh.ndof, mesh.ndof, nthreads=4)
    ref = q2.build_tables(E, E, mesh.ndof, mesh.ndof, True)
    for a, b in zip(got[:3], ref[:3]):
        assert np.array_equal(a, b)
    assert got[3] == ref[3]


def test_host_pattern_build_errors():
    from hippymfem_b200.pattern import build_tables

    t = np.array([[0, 1, 2], [2, 3, 9]])
    with pytest.raises(IndexError):
        build_tables(t, t, 5, 5)
    with pytest.raises(ValueError):
        build_tables(t, t[:1], 5, 5)


def test_lattice_handle_sizes():
    from hippymfem_b200 import _lib

    h = ctypes.c_void_p()
    _lib.check(_lib.lib.hm_lattice_create(64, 64, 64, 1.0, 1.0, 1.0, ctypes.byref(h)))
    ne, nd, nnz, qb = (ctypes.c_int64() for _ in range(4))
    _lib.check(_lib.lib.hm_lattice_sizes(h, _lib.HM_FP64, ctypes.byref(ne), ctypes.byref(nd),
                                         ctypes.byref(nnz), ctypes.byref(qb)))
    assert (ne.value, nd.value, nnz.value) == (262144, 2146689, 135005697)
    assert qb.value == 262144 * 216 * 8
    _lib.lib.hm_lattice_destroy(h)
    with pytest.raises(ValueError):
        _lib.check(_lib.lib.hm_lattice_create(0, 4, 4, 1.0, 1.0, 1.0, ctypes.byref(h)))
    with pytest.raises(NotImplementedError):      # nnz beyond int32 (hypre's HYPRE_Int)
        _lib.check(_lib.lib.hm_lattice_create(256, 256, 256, 1.0, 1.0, 1.0, ctypes.byref(h)))


def test_ops_refuse_host_tensors():
    """No CPU fallback: a host tensor is an error, not a slow path."""
    import torch
    from hippymfem_b200._lib import ptr

    with pytest.raises(ValueError):
        ptr(torch.zeros(4, dtype=torch.float64))


def test_observation_box_test_matches_the_kernel_rule():
    """targets_in_box (host) applies -1e-12 <= x / h <= n + 1e-12 per axis, finite: the
    targets it keeps are the ones hm_lattice_observation accepts."""
    from types import SimpleNamespace

    from hippymfem_b200.modeling import targets_in_box

    mesh = SimpleNamespace(h=(0.25, 0.7 / 3, 1.3 / 5), n=(4, 3, 5))
    pts = np.array([[0.0, 0.0, 0.0], [1.0, 0.7, 1.3], [1.0 + 1e-14, 0.1, 0.1],
                    [1.0 + 1e-9, 0.1, 0.1], [-1e-9, 0.1, 0.1], [0.5, np.nan, 0.5],
                    [0.5, np.inf, 0.5], [0.3, 0.3, 0.3]])
    assert targets_in_box(mesh, pts).tolist() == [True, True, True, False, False, False,
                                                 False, True]


def test_dof_permutation_from_a_caller_table():
    """hm_lattice_dof_permutation (host): the permuted fixture's table (random global
    numbering, random element-local order) gives back its global permutation; a table
    that puts two dofs at one node, or a bad local order, is refused."""
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import hptr

    z = load_golden("pattern_q2_permuted_3x3x2.npz")
    mo = q2.Lattice((3, 3, 2))
    rng = np.random.default_rng(20261203)           # the fixture's generator, in its order
    perm = rng.permutation(mo.ndof)
    local_fix = rng.permutation(27)
    tp = np.ascontiguousarray(z["tdofs"], dtype=np.int64)
    assert np.array_equal(perm[mo.edofs()][:, local_fix], tp)
    h = ctypes.c_void_p()
    _lib.check(_lib.lib.hm_lattice_create(3, 3, 2, 1.0, 1.0, 1.0, ctypes.byref(h)))
    try:
        local = np.ascontiguousarray(np.argsort(local_fix), dtype=np.int32)
        out = np.empty(mo.ndof, dtype=np.int32)
        _lib.check(_lib.lib.hm_lattice_dof_permutation(h, hptr(tp), hptr(local), hptr(out)))
        assert np.array_equal(out, perm)
        bad = tp.copy()
        bad[0, 0], bad[0, 1] = bad[0, 1], bad[0, 0]          # two dofs swapped in one element
        with pytest.raises(ValueError):
            _lib.check(_lib.lib.hm_lattice_dof_permutation(h, hptr(bad), hptr(local), hptr(out)))
        dup = local.copy()
        dup[1] = dup[0]
        with pytest.raises(ValueError):
            _lib.check(_lib.lib.hm_lattice_dof_permutation(h, hptr(tp), hptr(dup), hptr(out)))
        big = tp.copy()
        big[2, 3] = mo.ndof
        with pytest.raises(IndexError):
            _lib.check(_lib.lib.hm_lattice_dof_permutation(h, hptr(big), hptr(local), hptr(out)))
    finally:
        _lib.lib.hm_lattice_destroy(h)


def _mg_levels(n):
    """The multigrid hierarchy's (elements, nodes) per level, restated: the Q2 lattice, Q1
    on the same elements, then Q1 coarsened 2:1 while every axis stays even and >= 4."""
    nx, ny, nz = n
    lv = [(nx * ny * nz, (2 * nx + 1) * (2 * ny + 1) * (2 * nz + 1))]
    if min(n) < 2:
        return lv, 0
    lv.append((nx * ny * nz, (nx + 1) * (ny + 1) * (nz + 1)))
    while len(lv) < 16 and all(a % 2 == 0 and a >= 4 for a in (nx, ny, nz)):
        nx, ny, nz = nx // 2, ny // 2, nz // 2
        lv.append((nx * ny * nz, (nx + 1) * (ny + 1) * (nz + 1)))
    return lv, (nx - 1) * (ny - 1) * (nz - 1)


@pytest.mark.parametrize("n", [(64, 64, 64), (16, 8, 12), (8, 8, 8), (24, 24, 24)])
def test_single_cycle_workspace_matches_the_level_plan(n):
    """hm_mg_single_workspace_bytes: the point's D and the element results (54 floats per
    element), per level the coefficients (Q1 levels), reciprocal diagonal and five vectors,
    the coarse inverse when the coarsest level has at most 64 interior nodes; every piece
    rounded up to 32 floats."""
    from hippymfem_b200 import _lib

    h = ctypes.c_void_p()
    _lib.check(_lib.lib.hm_lattice_create(*n, 1.0, 1.0, 1.0, ctypes.byref(h)))
    levels, interior = _mg_levels(n)
    up = lambda k: (k + 31) // 32 * 32                       # noqa: E731
    floats = up(54 * levels[0][0])
    for l, (ne, nodes) in enumerate(levels):
        floats += (up(ne) if l >= 1 else 0) + 6 * up(nodes)
    if len(levels) > 1 and 1 <= interior <= 64:
        floats += up(64 * 64)
    assert _lib.lib.hm_mg_single_workspace_bytes(h) == 4 * floats
    _lib.lib.hm_lattice_destroy(h)
