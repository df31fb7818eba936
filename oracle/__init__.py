"""CPU FP64 oracle for the Q2 log-conductivity diffusion path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``hippymfem_b200``) imports,
links or executes anything under ``oracle/``; only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm use it,
and there only as the checker or as the timed CPU restatement of the reference.

Parity status (see each module's header):

* sparsity pattern (``indptr``, ``indices``, ``slot``, ``nnz``, dtypes) — PINNED:
  :mod:`oracle.q2` restates ``hippymfem/fem/patternbuild.py:209-253`` and is checked
  array-for-array against fixtures produced by the reference's own numba passes
  (``hippymfem/fem/_patternkernels.py``), see ``tests/golden/make_golden.py``;
* element blocks and vectors — pinned to known answers only (the reference's JAX
  blocks cannot be produced here: JAX/MFEM are absent): exact tensor-product integrals
  at constant coefficient, forward-over-reverse AD of the same density by
  ``torch.func`` (:mod:`oracle.ad`, the stand-in for ``hippymfem/fem/kernel.py:1392-1405``)
  and central finite differences;
* solves / Hessian action — restated (``hippymfem/modeling/reducedHessian.py:115-131``)
  with a Jacobi-PCG in place of hypre BoomerAMG-PCG; parity is stated at the solve
  tolerance.
"""
