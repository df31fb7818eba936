"""Generate the sparsity-pattern golden fixtures from the reference's own code.

Run in a container that holds the hIPPyMFEM source tree (it is not needed anywhere
else; the fixtures it writes are committed):

    python tests/golden/make_golden.py <path of the hIPPyMFEM source tree>

It loads ``hippymfem/fem/_patternkernels.py`` by file path (numba + numpy only; the rest
of the package needs MFEM/JAX/MPI, which are absent) and drives its three table passes
``group_table``, ``order_table`` and ``place_table`` exactly as
``hippymfem/fem/patternbuild.py:209-253`` (``build_tables``) does, then stores the dof
tables and the arrays the reference produced.  The driver below is a restatement of
those few lines (thread count, dtype choices); the passes themselves are the
reference's.
"""

import importlib.util
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_passes(ref_root):
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="numba_golden_"))
    path = os.path.join(ref_root, "hippymfem", "fem", "_patternkernels.py")
    spec = importlib.util.spec_from_file_location("_ref_patternkernels", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_build_tables(pk, tdofs, cdofs, nrow, ncol, diag_first):
    """The reference's ``build_tables`` driver around its compiled passes."""
    tdofs = np.ascontiguousarray(tdofs, dtype=np.int64)
    cdofs = np.ascontiguousarray(cdofs, dtype=np.int64)
    ne, ndt = tdofs.shape
    ndr = int(cdofs.shape[1])
    n = int(ne) * int(ndt) * ndr
    col_t = np.int32 if ncol <= np.iinfo(np.int32).max else np.int64
    rcount, runs_of_row = pk.group_table(tdofs, int(nrow))
    maxlen = int(np.max(np.diff(rcount))) * ndr if nrow else 1
    assert maxlen < (1 << pk.QBITS)
    wide = np.int32 if n <= np.iinfo(np.int32).max else np.int64
    ucount = np.zeros(int(nrow), np.int64)
    slot = np.empty(n, wide)
    pk.order_table(cdofs, int(ndt), rcount, runs_of_row, int(nrow), bool(diag_first),
                   ucount, slot, max(maxlen, 1), 4096)
    indptr = np.zeros(int(nrow) + 1, np.int64)
    np.cumsum(ucount, out=indptr[1:])
    nnz = int(indptr[-1])
    indices = np.empty(nnz, col_t)
    pk.place_table(cdofs, int(ndt), rcount, runs_of_row, indptr, int(nrow), indices, slot)
    idx_t = np.int32 if nnz <= np.iinfo(np.int32).max else np.intp
    if slot.dtype != idx_t:
        slot = slot.astype(idx_t)
    # hypre's HYPRE_Int is 32-bit in the reference's default build
    return indptr.astype(np.int32), indices.astype(np.int32), slot, nnz


def lattice_edofs(n, order=2):
    """Element dof table of a uniform hex lattice, lexicographic numbering, for a
    Lagrange space of ``order`` 1 or 2."""
    nx, ny, nz = n
    k = order
    Nx, Ny = k * nx + 1, k * ny + 1
    nd1 = k + 1
    ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ex, ey, ez = (v.transpose(2, 1, 0).reshape(-1) for v in (ex, ey, ez))
    a = np.arange(nd1 ** 3)
    a1, a2, a3 = a % nd1, (a // nd1) % nd1, a // (nd1 * nd1)
    ix = k * ex[:, None] + a1[None]
    iy = k * ey[:, None] + a2[None]
    iz = k * ez[:, None] + a3[None]
    return (ix + Nx * (iy + Ny * iz)).astype(np.int64), Nx * Ny * (k * nz + 1)


def cases(rng):
    out = {}
    # two 1D quadratic elements side by side: rows 1 and 2 lead with their diagonal
    out["toy_two_elements"] = (np.array([[0, 1, 2], [2, 3, 4]]),
                               np.array([[0, 1, 2], [2, 3, 4]]), 5, 5, True)
    for n in ((1, 1, 1), (2, 2, 2), (3, 2, 4), (4, 4, 4)):
        t, nd = lattice_edofs(n)
        out["q2_lattice_%dx%dx%d" % n] = (t, t, nd, nd, True)
    # arbitrary global numbering and element-local order: the drop-in case (MFEM numbers
    # vertices, edges, faces and interiors in its own order)
    t, nd = lattice_edofs((3, 3, 2))
    perm = rng.permutation(nd)
    local = rng.permutation(27)
    tp = perm[t][:, local]
    out["q2_permuted_3x3x2"] = (tp, tp, nd, nd, True)
    # rectangular: Q2 rows, Q1 columns (no diagonal-first order)
    t2, nd2 = lattice_edofs((2, 3, 2), 2)
    t1, nd1 = lattice_edofs((2, 3, 2), 1)
    out["q2xq1_rect_2x3x2"] = (t2, t1, nd2, nd1, nd2 == nd1)
    out["q1xq2_rect_2x3x2"] = (t1, t2, nd1, nd2, nd2 == nd1)
    return out


def main(ref_root):
    pk = load_passes(ref_root)
    rng = np.random.default_rng(20261203)
    for name, (t, c, nrow, ncol, diag_first) in cases(rng).items():
        indptr, indices, slot, nnz = reference_build_tables(pk, t, c, nrow, ncol, diag_first)
        path = os.path.join(HERE, "pattern_%s.npz" % name)
        np.savez_compressed(path, tdofs=np.asarray(t, np.int64), cdofs=np.asarray(c, np.int64),
                            nrow=nrow, ncol=ncol, diag_first=diag_first,
                            indptr=indptr, indices=indices, slot=slot, nnz=nnz)
        print("%-28s nrow=%6d ncol=%6d nnz=%8d entries=%8d" % (name, nrow, ncol, nnz, slot.size))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the hIPPyMFEM source tree>")
    main(sys.argv[1])
