"""Products, solves and the Hessian action on the device against the oracle.  GPU."""

import numpy as np
import pytest
import scipy.sparse.linalg as spl
import torch

from oracle import q2

pytestmark = pytest.mark.gpu


def _setup(n, seed=0, obs=64, matrix_free=False, tol=1e-12):
    from hippymfem_b200 import (BoxMesh, DirichletBC, Model, PDEVariationalProblem,
                                PointwiseStateObservation, Q2Space)
    from hippymfem_b200.synthetic import interior_points, log_conductivity

    mesh = BoxMesh(n)
    V = Q2Space(mesh)
    bc = DirichletBC(V)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=bc, solver_tolerance=tol,
                                 matrix_free_solves=matrix_free)
    pts = interior_points(obs, seed=seed + 10)
    misfit = PointwiseStateObservation(V, pts, data=np.random.default_rng(seed).standard_normal(obs)
                                       * 1e-3, noise_variance=1e-4)
    model = Model(prob, None, misfit)
    m = V.project(lambda x: log_conductivity(x, seed=seed))
    return mesh, V, prob, model, m


def test_spmv_and_transpose(cuda):
    from hippymfem_b200 import BoxMesh, CSRBlock, LatticePattern

    mesh = BoxMesh((5, 4, 6))
    pat = LatticePattern(mesh)
    rng = np.random.default_rng(0)
    vals = torch.as_tensor(rng.standard_normal(mesh.nnz), device=cuda)
    M = CSRBlock(pat, vals)
    S = M.to_scipy()
    x = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
    y = torch.empty_like(x)
    M.mult(x, y)
    ref = S @ x.cpu().numpy()
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    M.mult_transpose(x, y)
    ref = S.T @ x.cpu().numpy()
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    y0 = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
    y = y0.clone()
    M.mult(x, y, alpha=2.0, beta=-0.5)
    ref = 2.0 * (S @ x.cpu().numpy()) - 0.5 * y0.cpu().numpy()
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


def test_matrix_free_jacobian_matches_assembled(cuda):
    mesh, V, prob, model, m = _setup((6, 5, 7))
    A, _ = prob._jacobian([None, m, None])
    quad = prob._quadrature([None, m, None], "mf")
    from hippymfem_b200 import MatrixFreeJacobian

    mf = MatrixFreeJacobian(mesh, quad, prob.bc0.marker)
    x = torch.as_tensor(np.random.default_rng(1).standard_normal(mesh.ndof), device=cuda)
    y1, y2 = torch.empty_like(x), torch.empty_like(x)
    A.mult(x, y1)
    mf.mult(x, y2)
    assert (y1 - y2).abs().max().item() <= 1e-12 * y1.abs().max().item()
    d1, d2 = A.diagonal(), mf.diagonal()
    assert (d1 - d2).abs().max().item() <= 1e-12 * d1.abs().max().item()


@pytest.mark.parametrize("matrix_free", [False, True])
def test_forward_solve_matches_oracle(cuda, matrix_free):
    n = (8, 8, 8)
    mesh, V, prob, model, m = _setup(n, matrix_free=matrix_free)
    u = V.vector()
    prob.solveFwd(u, [u, m, None])
    assert prob.last_solve.converged
    mo = q2.Lattice(n)
    E = mo.edofs()
    mn = m.cpu().numpy()
    z = np.zeros(mo.ndof)
    ess = mo.boundary_dofs()
    mask = np.zeros(mo.ndof, bool)
    mask[ess] = True
    pat = q2.build_tables(E, E, mo.ndof, mo.ndof, True)
    A = q2.csr(pat, q2.assemble_block("A", pat, q2.element_blocks(mo, E, z, mn, z, ("A",))["A"],
                                      mask), (mo.ndof,) * 2)
    r = q2.assemble_vector(E, q2.element_vectors(mo, E, z, mn, z)[q2.ADJOINT], mo.ndof, ess)
    uref = spl.spsolve(A.tocsc(), -r)
    un = u.cpu().numpy()
    assert np.abs(un - uref).max() <= 1e-9 * np.abs(uref).max()


def test_pcg_is_deterministic_and_check_interval_independent(cuda):
    mesh, V, prob, model, m = _setup((6, 6, 6))
    A, _ = prob._jacobian([None, m, None])
    from hippymfem_b200 import PCGSolver

    b = torch.as_tensor(np.random.default_rng(2).standard_normal(mesh.ndof), device=cuda)
    prob.bc0.zero(b)
    out = []
    for every in (1, 7, 64):
        s = PCGSolver(A, rel_tolerance=1e-10, check_every=every)
        x = V.vector()
        s.solve(x, b)
        out.append((x.cpu().numpy(), s.last.iterations))
    assert out[0][1] == out[1][1] == out[2][1]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][0], out[2][0])


@pytest.mark.parametrize("matrix_free", [False, True])
def test_hessian_action_matches_oracle(cuda, matrix_free):
    """TrueHessian (reducedHessian.py:115-131) at the solved linearization point, against
    the oracle's restatement with the same Jacobi-PCG tolerance; parity is stated at
    the solve tolerance (1e-12 each solve -> 1e-9 on the action)."""
    from hippymfem_b200 import ReducedHessian, STATE, PARAMETER, ADJOINT

    n = (8, 6, 7)
    mesh, V, prob, model, m = _setup(n, matrix_free=matrix_free)
    u, p = V.vector(), V.vector()
    x = [u, m, p]
    model.solveFwd(u, x)
    model.solveAdj(p, x)
    model.setPointForHessianEvaluations(x)
    H = ReducedHessian(model)
    v = torch.as_tensor(np.random.default_rng(7).standard_normal(mesh.ndof), device=cuda)
    y = V.vector()
    H.mult(v, y)
    # oracle
    mo = q2.Lattice(n)
    E = mo.edofs()
    nd = mo.ndof
    ess = mo.boundary_dofs()
    mask = np.zeros(nd, bool)
    mask[ess] = True
    pat = q2.build_tables(E, E, nd, nd, True)
    un, mn, pn = u.cpu().numpy(), m.cpu().numpy(), p.cpu().numpy()
    blk = q2.element_blocks(mo, E, un, mn, pn)
    blocks = {k: q2.csr(pat, q2.assemble_block(k, pat, blk[k], mask), (nd, nd)) for k in blk}
    Bh = model.misfit.Bh
    Wuu = (Bh.T @ Bh) / model.misfit.noise_variance
    yref, _ = q2.hessian_apply(blocks, v.cpu().numpy(), ess, Wuu=Wuu, rtol=1e-12)
    yn = y.cpu().numpy()
    assert np.linalg.norm(yn - yref) <= 1e-8 * np.linalg.norm(yref)
    assert H.iterations and all(k > 0 for k in H.iterations)


def test_gradient_matches_adjoint_identity(cuda):
    """dR/dm at (u, m, p) equals C^T p (evalGradientParameter's docstring)."""
    from hippymfem_b200 import PARAMETER, ADJOINT

    mesh, V, prob, model, m = _setup((5, 5, 5))
    rng = np.random.default_rng(9)
    u = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
    p = torch.as_tensor(rng.standard_normal(mesh.ndof), device=cuda)
    prob.bc0.zero(p)
    x = [u, m, p]
    g = V.vector()
    prob.evalGradientParameter(x, g)
    prob.setLinearizationPoint(x)
    # C has its essential rows zeroed; p is zero there, so C^T p is unaffected
    ctp = V.vector()
    prob.apply_ij(PARAMETER, ADJOINT, p, ctp)
    # dR/dm_k = sum_i C_ik p_i only holds for the unconstrained C: compare on the values
    assert (g - ctp).abs().max().item() <= 1e-12 * g.abs().max().item()


@pytest.mark.parametrize("n", [(2, 2, 2), (4, 3, 5)])
def test_small_assembled_solves(cuda, n):
    """Systems smaller than the fixed reduction grid (here 125 and 693 dofs): the CSR
    PCG's partial sums must not reach its scalars."""
    from hippymfem_b200.sparse import PCGSolver

    mesh, V, prob, model, m = _setup(n)
    A, _ = prob._jacobian([None, m, None])
    b = torch.as_tensor(np.random.default_rng(1).standard_normal(mesh.ndof), device=cuda)
    prob.bc0.zero(b)
    x = V.vector()
    s = PCGSolver(A, rel_tolerance=1e-12)
    s.solve(x, b)
    assert s.last.converged and s.last.iterations > 0
    r = V.vector()
    A.mult(x, r)
    assert float((r - b).norm()) <= 1e-10 * float(b.norm())


def test_vectors_at_the_point_decided_on_the_device(cuda):
    """Without finiteness checks the residual and gradient at the linearization point
    come from hm_lattice_vectors_at, which compares the point on the device: the point's
    own vectors (its fused pass) where x is the point, the vectors from the fields as
    soon as one entry differs -- each bit for bit as the synchronous route gives them."""
    from hippymfem_b200 import (ADJOINT, PARAMETER, STATE, BoxMesh, DirichletBC,
                                PDEVariationalProblem, Q2Space)

    mesh = BoxMesh((5, 4, 6))
    V = Q2Space(mesh)
    bc = DirichletBC(V)
    sync = PDEVariationalProblem([V, V, V], f=1.0, bc=bc, check_finite=True)
    fast = PDEVariationalProblem([V, V, V], f=1.0, bc=bc, check_finite=False)
    rng = np.random.default_rng(21)
    u, m, p = (torch.as_tensor(rng.standard_normal(mesh.ndof) * s, device=cuda)
               for s in (1.0, 0.3, 1.0))
    x = [u, m, p]
    for prob in (sync, fast):
        prob.setLinearizationPoint(x)
    for var in (STATE, PARAMETER, ADJOINT):
        a, b = sync._residual(x, var), fast._residual(x, var)
        assert torch.equal(a, b)
        assert torch.equal(b, fast._lin_vectors[var])        # the point's own vector
    # one entry moved: every vector from the fields, as the synchronous route computes it
    x2 = [u.clone(), m.clone(), p]
    x2[PARAMETER][mesh.ndof // 2] += 1e-3
    for var in (STATE, PARAMETER, ADJOINT):
        a, b = sync._residual(x2, var), fast._residual(x2, var)
        assert torch.equal(a, b)
        assert not torch.equal(b, fast._lin_vectors[var])
    # and back at the point
    g1, g2 = V.vector(), V.vector()
    sync.evalGradientParameter(x, g1)
    fast.evalGradientParameter(x, g2)
    assert torch.equal(g1, g2)
