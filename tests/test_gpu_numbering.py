"""The C ABI on a caller's own dof numbering, the element-matrix export and the C-ABI
Hessian action.  GPU.

* ``pattern_q2_permuted_3x3x2.npz`` holds the reference's pattern arrays for a dof table
  with a random global numbering and a random element-local order (the drop-in case:
  MFEM numbers its dofs in its own order).  The lattice path, mapped into that numbering
  (``hm_lattice_dof_permutation`` + ``hm_lattice_caller_map`` + ``hm_gather_f64``),
  reproduces those arrays and the oracle's values on that numbering (1e-12).
* ``hm_lattice_element_blocks`` against the oracle's element matrices, in a permuted
  element-local order.
* ``hm_hessian_apply`` against the Python ``ReducedHessian`` on the same blocks and
  against the oracle's ``TrueHessian`` restatement.
"""

import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import q2

pytestmark = pytest.mark.gpu

TOL = 1e-12
BLOCKS = ("A", "C", "Wum", "Wmm")


def _fixture_numbering():
    """The global and element-local permutations behind the permuted fixture (its
    generator draws them first from seed 20261203), checked against its table."""
    z = load_golden("pattern_q2_permuted_3x3x2.npz")
    mo = q2.Lattice((3, 3, 2))
    t = mo.edofs()
    rng = np.random.default_rng(20261203)
    perm = rng.permutation(mo.ndof)
    local_fix = rng.permutation(27)
    assert np.array_equal(perm[t][:, local_fix], z["tdofs"])
    return z, mo, perm, local_fix


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_lattice_path_on_the_permuted_reference_numbering(cuda):
    from hippymfem_b200 import BoxMesh, LatticePattern
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.numbering import CallerNumbering

    z, mo, perm, local_fix = _fixture_numbering()
    tp = z["tdofs"]
    local = np.argsort(local_fix)            # caller slot of each lattice-local dof
    mesh = BoxMesh((3, 3, 2))
    num = CallerNumbering(mesh, tp, local)
    assert np.array_equal(num.perm_host, perm)
    # the caller's pattern: the reference's arrays, array for array
    for key, got in (("indptr", num.indptr.cpu().numpy()), ("indices", num.indices.cpu().numpy()),
                     ("slot", num.slot_host)):
        assert got.dtype == z[key].dtype and np.array_equal(got, z[key]), key
    # a point given in the caller's numbering
    nd = mesh.ndof
    rng = np.random.default_rng(5)
    uc, mc, pc = rng.standard_normal(nd), 0.3 * rng.standard_normal(nd), rng.standard_normal(nd)
    U, M, P = (num.to_lattice(torch.as_tensor(v, device=cuda)) for v in (uc, mc, pc))
    pat = LatticePattern(mesh, with_transpose=False)
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(U), ptr(M), ptr(P), _lib.HM_FP64, ptr(quad),
                                    ptr(status), stream_ptr()))
    vals = {b: pat.new_values() for b in BLOCKS}
    vecs = [torch.empty(nd, dtype=torch.float64, device=cuda) for _ in range(3)]
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr), None,
                                  1.4, *(ptr(vals[b]) for b in BLOCKS), *(ptr(v) for v in vecs),
                                  0, stream_ptr()))
    got = {b: num.values_to_caller(vals[b]).cpu().numpy() for b in BLOCKS}
    gotv = [num.to_caller(v).cpu().numpy() for v in vecs]
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    # the oracle on the caller's numbering: its table in lattice-local order
    Ec = tp[:, local]
    blk = q2.element_blocks(mo, Ec, uc, mc, pc)
    cpat = (z["indptr"], z["indices"], q2.build_tables(Ec, Ec, nd, nd, True)[2], int(z["nnz"]))
    for b in BLOCKS:
        ref = q2.scatter(cpat[2], blk[b], cpat[3])
        assert _rel(got[b], ref) <= TOL, (b, _rel(got[b], ref))
    ev = q2.element_vectors(mo, Ec, uc, mc, pc, 1.4)
    for s in range(3):
        ref = q2.assemble_vector(Ec, ev[s], nd)
        assert _rel(gotv[s], ref) <= TOL, s


def test_caller_map_rejects_a_foreign_pattern(cuda):
    from hippymfem_b200 import BoxMesh
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.numbering import CallerNumbering

    mesh = BoxMesh((3, 2, 2))
    E = mesh.edofs()
    num = CallerNumbering(mesh, E)                        # the lattice's own numbering
    assert torch.equal(num.perm.cpu(), torch.arange(mesh.ndof, dtype=torch.int32))
    bad = num.indices.clone()
    bad[5] = (bad[5] + 1) % mesh.ndof                    # one wrong column
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    check(lib.hm_lattice_caller_map(mesh.handle, ptr(num.perm), ptr(num.indptr), ptr(bad),
                                    ptr(num.src_pos), ptr(status), stream_ptr()))
    torch.cuda.synchronize()
    assert int(status.item()) != 0


def test_assembly_rejects_a_foreign_row_pointer_array(cuda):
    """hm_lattice_assemble compares the indptr it is given with the lattice pattern's:
    another one sets HM_STATUS_RANGE in the library's status word."""
    from hippymfem_b200 import BoxMesh, LatticePattern
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    mesh = BoxMesh((4, 3, 3))
    pat = LatticePattern(mesh, with_transpose=False)
    quad = torch.zeros(mesh.quad_bytes() // 8, dtype=torch.float64, device=cuda)
    vals = pat.new_values()
    st = np.zeros(1, dtype=np.uint32)
    check(lib.hm_device_status(st.ctypes.data, 1))
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr), None,
                                  1.0, ptr(vals), None, None, None, None, None, None, 0,
                                  stream_ptr()))
    check(lib.hm_device_status(st.ctypes.data, 1))
    assert st[0] == 0
    wrong = pat.indptr.clone()
    wrong[1:] += 1
    vals.fill_(float("nan"))
    vec = torch.full((mesh.ndof,), float("nan"), dtype=torch.float64, device=cuda)
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(wrong), None, 1.0,
                                  ptr(vals), None, None, None, ptr(vec), None, None, 0,
                                  stream_ptr()))
    check(lib.hm_device_status(st.ctypes.data, 1))
    assert st[0] & _lib.HM_STATUS_RANGE
    # every tile sees a row pointer that is not the lattice's: nothing is written
    assert bool(torch.isnan(vals).all()) and bool(torch.isnan(vec).all())


def test_element_matrices_match_the_oracle(cuda):
    from hippymfem_b200 import BoxMesh
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.numbering import element_matrices

    n, L = (3, 4, 2), (1.0, 0.8, 1.1)
    mesh = BoxMesh(n, L)
    mo = q2.Lattice(n, L)
    rng = np.random.default_rng(8)
    u, m, p = rng.standard_normal(mesh.ndof), 0.4 * rng.standard_normal(mesh.ndof), \
        rng.standard_normal(mesh.ndof)
    U, M, P = (torch.as_tensor(v, device=cuda) for v in (u, m, p))
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(U), ptr(M), ptr(P), _lib.HM_FP64, ptr(quad),
                                    ptr(status), stream_ptr()))
    local = rng.permutation(27)
    e0, count = 3, mesh.ne - 5
    got = element_matrices(mesh, quad, e0=e0, count=count, local=local)
    ref = q2.element_blocks(mo, mo.edofs(), u, m, p)
    for b in BLOCKS:
        want = np.empty((count, 27, 27))
        want[:, local[:, None], local[None, :]] = ref[b][e0:e0 + count]
        assert _rel(got[b].cpu().numpy(), want) <= 1e-13, b


def test_c_abi_hessian_action(cuda):
    """hm_hessian_apply at the solved point: the Python ReducedHessian's action on the
    same assembled blocks (both FP64 Jacobi-PCG to 1e-12), and the oracle's."""
    from hippymfem_b200 import (BoxMesh, DirichletBC, LatticePattern, Model,
                                PDEVariationalProblem, PointwiseStateObservation, Q2Space,
                                ReducedHessian)
    from hippymfem_b200.numbering import AssembledHessian
    from hippymfem_b200.sparse import SolvePlan
    from hippymfem_b200.synthetic import interior_points, log_conductivity

    n = (6, 5, 7)
    mesh = BoxMesh(n)
    V = Q2Space(mesh)
    bc = DirichletBC(V)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=bc, solver_tolerance=1e-12)
    misfit = PointwiseStateObservation(V, interior_points(48, seed=4),
                                       data=np.random.default_rng(1).standard_normal(48) * 1e-3,
                                       noise_variance=1e-4)
    model = Model(prob, None, misfit)
    m = V.project(lambda x: log_conductivity(x, seed=0))
    u, p = V.vector(), V.vector()
    x = [u, m, p]
    model.solveFwd(u, x)
    model.solveAdj(p, x)
    model.setPointForHessianEvaluations(x)
    v = torch.as_tensor(np.random.default_rng(9).standard_normal(mesh.ndof), device=cuda)
    y_py = V.vector()
    ReducedHessian(model, misfit_only=True).mult(v, y_py)
    pat = LatticePattern(mesh, with_transpose=True)
    prob._pattern = pat
    quad = prob._quadrature(prob._lin_point, "hess_c_abi")
    blocks, _ = prob._assemble(quad, blocks=("C", "Wum", "Wmm"))
    plan = SolvePlan(mesh, bc.marker, precision="fp64", rel_tolerance=1e-12)
    plan.set_point(quad)
    H = AssembledHessian(mesh, pat, blocks["C"].values, blocks["Wum"].values,
                         blocks["Wmm"].values, misfit, bc.marker, plan)
    y = V.vector()
    H.mult(v, y, rel_tolerance=1e-12)
    torch.cuda.synchronize()
    assert all(k > 0 for k in H.iterations)
    yn, yp = y.cpu().numpy(), y_py.cpu().numpy()
    assert np.linalg.norm(yn - yp) <= 1e-9 * np.linalg.norm(yp)
    # the oracle's TrueHessian on the same point
    mo = q2.Lattice(n)
    E = mo.edofs()
    nd = mo.ndof
    ess = mo.boundary_dofs()
    mask = np.zeros(nd, bool)
    mask[ess] = True
    pt = q2.build_tables(E, E, nd, nd, True)
    blk = q2.element_blocks(mo, E, u.cpu().numpy(), m.cpu().numpy(), p.cpu().numpy())
    bl = {k: q2.csr(pt, q2.assemble_block(k, pt, blk[k], mask), (nd, nd)) for k in blk}
    Bh = misfit.Bh
    yref, _ = q2.hessian_apply(bl, v.cpu().numpy(), ess, Wuu=(Bh.T @ Bh) / 1e-4, rtol=1e-12)
    assert np.linalg.norm(yn - yref) <= 1e-8 * np.linalg.norm(yref)
    # Gauss-Newton: y = C^T phat with phat from W_uu uhat only
    G = AssembledHessian(mesh, pat, blocks["C"].values, None, None, misfit, bc.marker, plan)
    yg = V.vector()
    G.mult(v, yg)
    model.setPointForHessianEvaluations(x, gauss_newton_approx=True)
    yg_py = V.vector()
    ReducedHessian(model, misfit_only=True).mult(v, yg_py)
    assert torch.linalg.norm(yg - yg_py) <= 1e-9 * torch.linalg.norm(yg_py)
