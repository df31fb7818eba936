"""CPU FP64 restatement of the reference's Q2-hex assembly path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may use this
module, as the checker or as the timed CPU restatement; the product never does.

What each function follows in the reference (paths relative to the hIPPyMFEM tree):

* :func:`gauss3`, :func:`lagrange3`, :func:`basis_tables` — the tables of
  ``hippymfem/fem/elementbatch.py:509-525`` (``_basis_tables``: ``N (nq, nd)``,
  ``G (nq, nd, dim)``) for MFEM's Q2 H1 element (nodes 0, 1/2, 1) and the 3x3x3
  Gauss-Legendre rule in MFEM's tensor order, point ``(i, j, k)`` at ``i + 3 (j + 3 k)``
  (``elementbatch.py:121-146``).
* :class:`Lattice` — a uniform ``nx x ny x nz`` hexahedral mesh of a box with the Q2 dofs
  numbered lexicographically on the ``(2nx+1) x (2ny+1) x (2nz+1)`` node lattice; the
  element dof table plays the role of ``_element_dofs`` (``elementbatch.py:528-565``).
  MFEM's own global numbering cannot be reproduced here (MFEM is absent), so pattern
  parity is defined on a shared dof table.
* :func:`element_fields`, :func:`element_blocks`, :func:`element_vectors` — the
  quadrature route ``hippymfem/fem/kernel.py:1431-1485`` written out in closed form for the
  density ``exp(m) grad u . grad p - f p`` (``benchmarks/bench_newton_device.py:392``),
  fields from ``_eval_field`` (``kernel.py:378-394``), vectors as ``grad_block``
  (``kernel.py:1343-1355``); rows are the test slot and columns the trial slot
  (``kernel.py:1704-1710``).
* :func:`element_blocks_fp32`, :func:`consistent_blocks` — the single-precision element
  matrices of ``PRECISION="mixed"`` (``kernel.py:61-99, 1001-1007``) and
  ``consistent_block`` (``kernel.py:1503-1571``): the single-precision block corrected by
  one rank-one term per side so that its products with the constants are the
  double-precision ones (``symmetric``: symmetrized first, symmetric to the last bit).
* :func:`build_tables` — ``hippymfem/fem/patternbuild.py:209-253`` (the arrays of the
  sort route ``hippymfem/fem/pattern.py:548-663``): CSR over rows, diagonal first on a
  square shape, then ascending columns; ``slot[(e*ndt+a)*ndr+b]`` the CSR position of
  entry ``(e, a, b)``; int32 ``indptr``/``indices``/``slot``.
* :func:`scatter`, :func:`masked_slots`, :func:`assemble_block` — ``pattern.py:749-791``
  (``np.bincount(slot, weights, minlength=nnz)``), ``pattern.py:693-713`` and the folded
  elimination of ``hippymfem/fem/csrassemble.py:164-270`` with the diagonal written as in
  ``hippymfem/fem/elimination.py:53-72``; the per-block policy is the table of
  ``hippymfem/fem/bcs.py:13-30`` and ``modeling/PDEVariationalProblem.py:1454-1457``.
* :func:`assemble_vector` — ``pattern.py:1186-1233`` / ``csrassemble.py:402-424`` plus
  ``zero_essential`` (``hippymfem/fem/bcs.py:80``).
* :func:`pcg`, :func:`hessian_apply` — ``modeling/reducedHessian.py:115-131``
  (``TrueHessian``) and ``modeling/PDEVariationalProblem.py:1583-1609``
  (``solveIncremental``: right-hand side zeroed on the essential dofs), with a
  Jacobi-PCG standing in for hypre BoomerAMG-PCG (unavailable here).
* :func:`boundary_mass` — the boundary integrator the reference's ``BiLaplacianPrior``
  adds with ``robin_bc=True`` (``modeling/prior.py:941-944``: ``MassIntegrator`` over the
  boundary elements), integrated face element by face element with the 3x3 Gauss rule.
* :func:`observation_matrix` — ``modeling/pointwiseObservation.py:36-224`` (rows of basis
  values at the points) and ``modeling/misfit.py:102-110`` (``W_uu = B^T B / sigma^2``).
"""

import numpy as np
import scipy.sparse as sp

STATE, PARAMETER, ADJOINT = 0, 1, 2


# ----------------------------------------------------------------------------- tables
def gauss3():
    """3-point Gauss-Legendre rule on [0, 1], ascending points."""
    s = np.sqrt(0.15)
    return np.array([0.5 - s, 0.5, 0.5 + s]), np.array([5.0, 8.0, 5.0]) / 18.0


def lagrange3(x):
    """Q2 Lagrange basis on nodes (0, 1/2, 1) and its derivative at points ``x``:
    ``(B, dB)`` of shape ``(len(x), 3)``."""
    x = np.asarray(x, dtype=np.float64)
    B = np.stack([2.0 * (x - 0.5) * (x - 1.0), -4.0 * x * (x - 1.0), 2.0 * x * (x - 0.5)], -1)
    dB = np.stack([4.0 * x - 3.0, 4.0 - 8.0 * x, 4.0 * x - 1.0], -1)
    return B, dB


def basis_tables():
    """``(N, G, w)``: ``N[q, a]``, ``G[q, a, k]`` on the reference cube, weights ``w[q]``.

    Quadrature points and dofs are both lexicographic, ``q = q1 + 3 q2 + 9 q3`` and
    ``a = a1 + 3 a2 + 9 a3``."""
    x, w1 = gauss3()
    B, dB = lagrange3(x)
    # x/y/z index the points along each axis, a/b/c the dofs; flattening (z, y, x) and
    # (c, b, a) gives q = q1 + 3 q2 + 9 q3 and a = a1 + 3 a2 + 9 a3
    N = np.einsum("xa,yb,zc->zyxcba", B, B, B).reshape(27, 27)
    Gx = np.einsum("xa,yb,zc->zyxcba", dB, B, B).reshape(27, 27)
    Gy = np.einsum("xa,yb,zc->zyxcba", B, dB, B).reshape(27, 27)
    Gz = np.einsum("xa,yb,zc->zyxcba", B, B, dB).reshape(27, 27)
    G = np.stack([Gx, Gy, Gz], -1)
    w = np.einsum("x,y,z->zyx", w1, w1, w1).reshape(27)
    return N, G, w


# ------------------------------------------------------------------------------- mesh
class Lattice:
    """Uniform hexahedral mesh of ``[0, L]`` with lexicographic Q2 dofs.

    Elements ``e = ex + nx (ey + ny ez)``; nodes ``n = ix + Nx (iy + Ny iz)`` with
    ``N* = 2 n* + 1``; element-local dof ``a = a1 + 3 a2 + 9 a3`` is node
    ``(2 ex + a1, 2 ey + a2, 2 ez + a3)``."""

    def __init__(self, n, L=(1.0, 1.0, 1.0)):
        self.n = tuple(int(v) for v in (n if np.ndim(n) else (n, n, n)))
        self.L = tuple(float(v) for v in L)
        self.N = tuple(2 * v + 1 for v in self.n)
        self.ne = int(np.prod(self.n))
        self.ndof = int(np.prod(self.N))
        self.h = tuple(Lv / nv for Lv, nv in zip(self.L, self.n))

    def edofs(self):
        nx, ny, nz = self.n
        Nx, Ny, _ = self.N
        ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        ex, ey, ez = (v.transpose(2, 1, 0).reshape(-1) for v in (ex, ey, ez))
        a = np.arange(27)
        a1, a2, a3 = a % 3, (a // 3) % 3, a // 9
        ix = 2 * ex[:, None] + a1[None]
        iy = 2 * ey[:, None] + a2[None]
        iz = 2 * ez[:, None] + a3[None]
        return (ix + Nx * (iy + Ny * iz)).astype(np.int64)

    def node_coords(self):
        Nx, Ny, Nz = self.N
        i = np.arange(self.ndof)
        ix, iy, iz = i % Nx, (i // Nx) % Ny, i // (Nx * Ny)
        return np.stack([ix * self.h[0] / 2, iy * self.h[1] / 2, iz * self.h[2] / 2], -1)

    def boundary_dofs(self):
        Nx, Ny, Nz = self.N
        i = np.arange(self.ndof)
        ix, iy, iz = i % Nx, (i // Nx) % Ny, i // (Nx * Ny)
        b = (ix == 0) | (ix == Nx - 1) | (iy == 0) | (iy == Ny - 1) | (iz == 0) | (iz == Nz - 1)
        return np.flatnonzero(b).astype(np.int64)

    def wdet(self):
        _, _, w = basis_tables()
        return w * (self.h[0] * self.h[1] * self.h[2])


# ----------------------------------------------------------------- element kernels
def element_fields(mesh, edofs, vals):
    """Values ``(ne, 27)`` and physical gradients ``(ne, 27, 3)`` of a Q2 field at the
    quadrature points (``kernel.py:378-394`` with ``Jinv = diag(1/h)``)."""
    N, G, _ = basis_tables()
    V = np.asarray(vals, dtype=np.float64)[edofs]
    val = V @ N.T
    grad = np.einsum("qak,ea->eqk", G, V) / np.asarray(mesh.h)[None, None, :]
    return val, grad


def _weights(mesh, edofs, u, m, p):
    mq, _ = element_fields(mesh, edofs, m)
    _, gu = element_fields(mesh, edofs, u)
    _, gp = element_fields(mesh, edofs, p)
    D = mesh.wdet()[None, :] * np.exp(mq)
    return D, gu, gp


def element_blocks(mesh, edofs, u, m, p, which=("A", "C", "Wum", "Wmm")):
    """Element matrices ``(ne, 27, 27)`` of the second-derivative blocks at ``(u, m, p)``.

    ``A``   = d2R/dp du: ``sum_q w|J| e^m grad phi_i . grad phi_j``    (ADJOINT, STATE)
    ``C``   = d2R/dp dm: ``sum_q w|J| e^m psi_k grad u . grad phi_i``  (ADJOINT, PARAMETER)
    ``Wum`` = d2R/du dm: ``sum_q w|J| e^m psi_k grad p . grad phi_j``  (STATE, PARAMETER)
    ``Wmm`` = d2R/dm dm: ``sum_q w|J| e^m psi_k psi_l grad u . grad p`` (PARAMETER, PARAMETER)
    """
    N, G, _ = basis_tables()
    Gp = G / np.asarray(mesh.h)[None, None, :]
    D, gu, gp = _weights(mesh, edofs, u, m, p)
    out = {}
    if "A" in which:
        A = 0.0
        for k in range(3):
            X = D[:, :, None] * Gp[None, :, :, k]                   # (ne, q, a)
            A = A + np.matmul(X.transpose(0, 2, 1), Gp[None, :, :, k])
        out["A"] = A
    for name, g in (("C", gu), ("Wum", gp)):
        if name in which:
            # rows: test dof i (grad phi_i . grad field), columns: parameter dof k (psi_k)
            R = np.einsum("eq,eqk,qak->eqa", D, g, Gp)              # (ne, q, i)
            out[name] = np.matmul(R.transpose(0, 2, 1), N[None])   # (ne, i, k)
    if "Wmm" in which:
        s = D * np.einsum("eqk,eqk->eq", gu, gp)
        X = s[:, :, None] * N[None]
        out["Wmm"] = np.matmul(X.transpose(0, 2, 1), N[None])
    return out


def element_blocks_fp32(mesh, edofs, u, m, p, which=("A", "C", "Wum", "Wmm")):
    """The element matrices of :func:`element_blocks` with the element contractions in
    single precision (weights, field gradients and tables rounded to float32, products
    and sums in float32), returned in float64."""
    N, G, _ = basis_tables()
    f32 = np.float32
    N32 = N.astype(f32)
    Gp = (G / np.asarray(mesh.h)[None, None, :]).astype(f32)
    D, gu, gp = _weights(mesh, edofs, u, m, p)
    D, gu, gp = D.astype(f32), gu.astype(f32), gp.astype(f32)
    out = {}
    if "A" in which:
        A = np.zeros((D.shape[0], 27, 27), dtype=f32)
        for k in range(3):
            X = D[:, :, None] * Gp[None, :, :, k]
            A = A + np.matmul(X.transpose(0, 2, 1), Gp[None, :, :, k])
        out["A"] = A
    for name, g in (("C", gu), ("Wum", gp)):
        if name in which:
            R = np.einsum("eq,eqk,qak->eqa", D, g, Gp)
            out[name] = np.matmul(R.transpose(0, 2, 1), N32[None])
    if "Wmm" in which:
        s = D * np.einsum("eqk,eqk->eq", gu, gp)
        X = s[:, :, None] * N32[None]
        out["Wmm"] = np.matmul(X.transpose(0, 2, 1), N32[None])
    return {k: v.astype(np.float64) for k, v in out.items()}


SYMMETRIC_BLOCKS = ("A", "Wmm")


def consistent_blocks(mesh, edofs, u, m, p, which=("A", "C", "Wum", "Wmm")):
    """``consistent_block`` (``kernel.py:1503-1571``) for the lattice's Q2 blocks: the
    single-precision element matrix ``K`` corrected with ``V = 1 / sqrt(27)`` (the
    normalized constants of a scalar Q2 element, ``_low_modes``) and the
    double-precision products ``R_j = K64 V^T`` (one tangent) so that ``K' V^T = R_j``
    and, two-sided, ``K'^T V^T = R_i``.  The symmetric blocks (A, W_mm) are symmetrized
    first and returned symmetric to the last bit (both triangles from the upper one)."""
    K32 = element_blocks_fp32(mesh, edofs, u, m, p, which)
    K64 = element_blocks(mesh, edofs, u, m, p, which)
    V = np.full((1, 27), 1.0 / np.sqrt(27.0))
    iu = np.triu_indices(27)
    out = {}
    for name in which:
        K = K32[name]
        Rj = K64[name] @ V.T                                         # (ne, 27, 1)
        if name in SYMMETRIC_BLOCKS:
            K = 0.5 * (K + K.transpose(0, 2, 1))
            Dj = Rj - K @ V.T
            U = Dj @ V
            S = V @ Dj                                               # (ne, 1, 1)
            W = V.T @ (0.5 * (S + S.transpose(0, 2, 1))) @ V
            M = K + (U + U.transpose(0, 2, 1)) - 0.5 * (W + W.transpose(0, 2, 1))
            up = M[:, iu[0], iu[1]]
            M = np.zeros_like(M)
            M[:, iu[0], iu[1]] = up
            M[:, iu[1], iu[0]] = up
            out[name] = M
        else:
            Ri = K64[name].transpose(0, 2, 1) @ V.T
            Dj = Rj - K @ V.T
            Di = Ri - K.transpose(0, 2, 1) @ V.T
            out[name] = (K + Dj @ V + V.T @ Di.transpose(0, 2, 1)
                         - V.T @ (V @ Dj) @ V)
    return out


def element_vectors(mesh, edofs, u, m, p, f=1.0):
    """Element vectors ``(ne, 27)``: ``dR/dp`` (residual), ``dR/dm`` and ``dR/du``."""
    N, G, w = basis_tables()
    Gp = G / np.asarray(mesh.h)[None, None, :]
    D, gu, gp = _weights(mesh, edofs, u, m, p)
    wdet = mesh.wdet()
    r_adj = np.einsum("eq,eqk,qak->ea", D, gu, Gp) - f * (wdet @ N)[None, :]
    r_par = np.einsum("eq,eq,qa->ea", D, np.einsum("eqk,eqk->eq", gu, gp), N)
    r_sta = np.einsum("eq,eqk,qak->ea", D, gp, Gp)
    return {ADJOINT: r_adj, PARAMETER: r_par, STATE: r_sta}


# ------------------------------------------------------------------------ pattern
def build_tables(tdofs, cdofs, nrow, ncol, diag_first):
    """``(indptr, indices, slot, nnz)`` as ``patternbuild.build_tables`` returns them.

    Entry ``k = (e * ndt + a) * ndr + b`` is row ``tdofs[e, a]``, column ``cdofs[e, b]``.
    Rows hold their distinct columns in ascending order, except that with
    ``diag_first`` the diagonal leads (``_patternkernels.py:56-88``: code 0 for the
    diagonal, ``col + 1`` otherwise).  ``slot[k]`` is the CSR position of entry ``k``."""
    tdofs = np.asarray(tdofs, dtype=np.int64)
    cdofs = np.asarray(cdofs, dtype=np.int64)
    ne, ndt = tdofs.shape
    ndr = cdofs.shape[1]
    rows = np.repeat(tdofs.reshape(-1), ndr)
    cols = np.broadcast_to(cdofs[:, None, :], (ne, ndt, ndr)).reshape(-1)
    code = cols + 1
    if diag_first:
        code = np.where(cols == rows, 0, code)
    key = (rows << 32) | code
    uniq, inv = np.unique(key, return_inverse=True)
    urow = uniq >> 32
    ucode = uniq & ((1 << 32) - 1)
    ucol = np.where(ucode == 0, urow, ucode - 1)
    indptr = np.zeros(nrow + 1, dtype=np.int64)
    np.cumsum(np.bincount(urow, minlength=nrow), out=indptr[1:])
    nnz = int(indptr[-1])
    idx_t = np.int32 if nnz <= np.iinfo(np.int32).max else np.intp
    return (indptr.astype(np.int32), ucol.astype(np.int32), inv.reshape(-1).astype(idx_t), nnz)


def scatter(slot, flat, nnz):
    """``np.bincount(slot, weights=flat, minlength=nnz)`` (``pattern.py:788``)."""
    return np.bincount(slot, weights=np.asarray(flat, dtype=np.float64).reshape(-1),
                       minlength=nnz)


def masked_slots(indptr, indices, row_mask, col_mask):
    """Slots of the masked rows and columns (``pattern.py:693-713``)."""
    nnz = int(indptr[-1])
    hit = (np.repeat(row_mask, np.diff(indptr.astype(np.int64))) if row_mask is not None
           else np.zeros(nnz, dtype=bool))
    if col_mask is not None:
        hit |= col_mask[indices]
    return np.flatnonzero(hit)


#: per block: (eliminate rows, eliminate columns, diagonal value or None)
ELIMINATION = {"A": (True, True, 1.0), "C": (True, False, None),
               "Wum": (True, False, None), "Wmm": (False, False, None)}


def assemble_block(name, pattern, element_matrices, ess_mask):
    """CSR ``data`` of one block with the folded elimination of its policy."""
    indptr, indices, slot, nnz = pattern
    data = scatter(slot, element_matrices, nnz)
    rows, cols, diag = ELIMINATION[name]
    if ess_mask is not None and (rows or cols):
        kill = masked_slots(indptr, indices, ess_mask if rows else None,
                            ess_mask if cols else None)
        data[kill] = 0.0
        if diag is not None:
            ess = np.flatnonzero(ess_mask)
            data[indptr[ess]] = diag          # diagonal first in every square row
    return data


def assemble_vector(edofs, element_vectors, ndof, ess=None):
    out = np.bincount(np.asarray(edofs).reshape(-1),
                      weights=np.asarray(element_vectors).reshape(-1), minlength=ndof)
    if ess is not None and len(ess):
        out[np.asarray(ess)] = 0.0
    return out


def csr(pattern, data, shape):
    """scipy CSR of a block; the pattern arrays are copied (scipy sorts the indices of a
    matrix in place, which would scramble the diagonal-first rows shared by blocks)."""
    indptr, indices, _, _ = pattern
    return sp.csr_matrix((np.array(data), indices.copy(), indptr.copy()), shape=shape)


def elements_of_nodes(mesh, nodes):
    """The elements holding any of the lattice ``nodes`` (ascending element ids): the
    only elements whose element matrices reach those rows."""
    Nx, Ny, _ = mesh.N
    nodes = np.asarray(nodes, dtype=np.int64)
    idx = (nodes % Nx, (nodes // Nx) % Ny, nodes // (Nx * Ny))
    out = set()
    for i, j, k in zip(*idx):
        per_axis = []
        for c, n in zip((i, j, k), mesh.n):
            cand = (c // 2,) if c % 2 else (c // 2 - 1, c // 2)
            per_axis.append([e for e in cand if 0 <= e < n])
        for ez in per_axis[2]:
            for ey in per_axis[1]:
                for ex in per_axis[0]:
                    out.add(ex + mesh.n[0] * (ey + mesh.n[1] * ez))
    return np.array(sorted(out), dtype=np.int64)


def assembled_rows(mesh, u, m, p, rows, ess_mask=None, f=1.0, which=("A", "C", "Wum", "Wmm")):
    """Selected rows of the assembled blocks and vectors, from the elements around them
    only: the same scatter (``pattern.py:749-791``), folded elimination
    (``csrassemble.py:164-270``, ``bcs.py:13-30``) and vector assembly
    (``pattern.py:1186-1233``) as the whole-mesh functions, restricted to ``rows`` so
    that a large lattice can be checked in seconds.

    Returns ``(blocks, vectors)``: ``blocks[name] = (keys, values)`` with
    ``keys = row * ndof + col`` ascending; ``vectors[slot]`` the vector at ``rows``
    (not zeroed on the essential dofs)."""
    rows = np.unique(np.asarray(rows, dtype=np.int64))
    elems = elements_of_nodes(mesh, rows)
    E = mesh.edofs()[elems]
    nd = mesh.ndof
    want = np.isin(E, rows)                                      # (ne_sub, 27) test dofs kept
    er, ea = np.nonzero(want)
    r = E[er, ea]                                                # row of each kept (e, a)
    blocks = {}
    for name in which:
        K = element_blocks(mesh, E, u, m, p, (name,))[name]      # (ne_sub, 27, 27)
        keys = (r[:, None] * nd + E[er]).reshape(-1)
        vals = K[er, ea, :].reshape(-1)
        uk, inv = np.unique(keys, return_inverse=True)
        acc = np.bincount(inv.reshape(-1), weights=vals, minlength=len(uk))
        rr, cc = uk // nd, uk % nd
        pol_rows, pol_cols, diag = ELIMINATION[name]
        if ess_mask is not None:
            kill = np.zeros(len(uk), dtype=bool)
            if pol_rows:
                kill |= ess_mask[rr]
            if pol_cols:
                kill |= ess_mask[cc]
            acc[kill] = 0.0
            if diag is not None:
                acc[kill & (rr == cc) & ess_mask[rr]] = diag
        blocks[name] = (uk, acc)
    ev = element_vectors(mesh, E, u, m, p, f)
    pos = np.searchsorted(rows, r)
    vectors = {s: np.bincount(pos, weights=ev[s][er, ea], minlength=len(rows)) for s in ev}
    return blocks, vectors


# ------------------------------------------------------------------- observations
def boundary_mass(mesh):
    """``int_{boundary} phi_n phi_c ds`` over the six faces of the box (scipy CSR,
    ``ndof x ndof``): each face is a grid of Q2 quadrilaterals, each integrated with the
    3x3 Gauss rule (exact for the products) and scattered by its 9 nodes."""
    x, w = gauss3()
    B, _ = lagrange3(x)                        # B[q, a]
    N = mesh.N
    rows, cols, vals = [], [], []
    for d in range(3):
        a, b = (d + 1) % 3, (d + 2) % 3
        na, nb = mesh.n[a], mesh.n[b]
        jac = mesh.h[a] * mesh.h[b]
        # face-element mass [i1 + 3 i2, j1 + 3 j2] on the reference square
        Wq = w[:, None] * w[None, :]           # [qa, qb]
        M = np.einsum("xy,xi,yj,xk,yl->ijkl", Wq, B, B, B, B) * jac   # (ia, ib, ja, jb)
        M = M.transpose(1, 0, 3, 2).reshape(9, 9)   # [ia + 3 ib, ja + 3 jb]
        ea, eb = np.meshgrid(np.arange(na), np.arange(nb), indexing="ij")
        ea, eb = ea.reshape(-1), eb.reshape(-1)
        loc = np.arange(9)
        ia = 2 * ea[:, None] + (loc % 3)[None]
        ib = 2 * eb[:, None] + (loc // 3)[None]
        for side in (0, N[d] - 1):
            idx = [None, None, None]
            idx[d] = np.full_like(ia, side)
            idx[a], idx[b] = ia, ib
            nodes = idx[0] + N[0] * (idx[1] + N[1] * idx[2])      # (nface, 9)
            rows.append(np.repeat(nodes, 9, axis=1).reshape(-1))
            cols.append(np.tile(nodes, (1, 9)).reshape(-1))
            vals.append(np.broadcast_to(M.reshape(1, 81), (nodes.shape[0], 81)).reshape(-1))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(mesh.ndof, mesh.ndof))


def observation_matrix(mesh, points):
    """Pointwise observation operator ``B``: row ``o`` holds the Q2 basis values at
    ``points[o]`` (``pointwiseObservation.py:36-224``)."""
    pts = np.asarray(points, dtype=np.float64)
    h = np.asarray(mesh.h)
    n = np.asarray(mesh.n)
    e = np.clip(np.floor(pts / h).astype(np.int64), 0, n - 1)
    xi = pts / h - e
    vals = []
    for d in range(3):
        B, _ = lagrange3(xi[:, d])
        vals.append(B)
    Nx, Ny, _ = mesh.N
    rows, cols, data = [], [], []
    for a in range(27):
        a1, a2, a3 = a % 3, (a // 3) % 3, a // 9
        node = (2 * e[:, 0] + a1) + Nx * ((2 * e[:, 1] + a2) + Ny * (2 * e[:, 2] + a3))
        rows.append(np.arange(len(pts)))
        cols.append(node)
        data.append(vals[0][:, a1] * vals[1][:, a2] * vals[2][:, a3])
    return sp.csr_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(len(pts), mesh.ndof))


# ------------------------------------------------------------------------- solves
def pcg(A, b, rtol=1e-12, maxiter=20000, x0=None):
    """Jacobi-preconditioned CG, stopped at ``||r||_2 <= rtol ||b||_2``.
    Returns ``(x, iterations)``."""
    dinv = 1.0 / A.diagonal()
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - A @ x
    bn = np.linalg.norm(b)
    if bn == 0.0:
        return np.zeros_like(b), 0
    z = dinv * r
    pdir = z.copy()
    rz = r @ z
    for it in range(1, maxiter + 1):
        q = A @ pdir
        alpha = rz / (pdir @ q)
        x += alpha * pdir
        r -= alpha * q
        if np.linalg.norm(r) <= rtol * bn:
            return x, it
        z = dinv * r
        rz_new = r @ z
        pdir = z + (rz_new / rz) * pdir
        rz = rz_new
    return x, maxiter


def solve_incremental(A, rhs, ess, rtol):
    r = rhs.copy()
    r[ess] = 0.0
    return pcg(A, r, rtol)


def hessian_apply(blocks, x, ess, Wuu=None, rtol=1e-12):
    """``ReducedHessian.TrueHessian`` (``reducedHessian.py:115-131``), misfit only:
    ``y = Wmm x + C^T phat - Wmu uhat`` with ``uhat = A^{-1} C x`` and
    ``phat = A^{-T} (Wuu uhat - Wum x)``.  Returns ``(y, iterations)``."""
    A, C, Wum, Wmm = blocks["A"], blocks["C"], blocks["Wum"], blocks["Wmm"]
    uhat, k1 = solve_incremental(A, C @ x, ess, rtol)
    rhs = (Wuu @ uhat if Wuu is not None else np.zeros_like(uhat)) - Wum @ x
    phat, k2 = solve_incremental(A.T.tocsr(), rhs, ess, rtol)
    y = Wmm @ x + C.T @ phat - Wum.T @ uhat
    return y, (k1, k2)
