"""Element blocks by automatic differentiation of the density — TEST INFRASTRUCTURE ONLY.

The reference derives every element block from the pointwise density by JAX:
forward-over-reverse, ``jax.jacfwd`` of ``jax.grad`` over one column slot at a time,
vmapped over elements (``hippymfem/fem/kernel.py:1392-1405``, ``_hess_slot_element_fn``)
and run over element windows of ``HOST_BATCH`` on the host (``kernel.py:659-748``).
JAX is absent here; ``torch.func`` computes the same derivatives of the same density
(``exp(m) grad u . grad p - f p``, ``benchmarks/bench_newton_device.py:392``) in FP64 on
the CPU.  Used as the AD cross-check of :mod:`oracle.q2` and as the timed CPU
restatement of the reference's host algorithm (``bench.py --impl reference``).
"""

import numpy as np
import torch
from torch.func import grad, jacfwd, vmap

from . import q2

STATE, PARAMETER, ADJOINT = q2.STATE, q2.PARAMETER, q2.ADJOINT

#: element window of the reference's host route (kernel.py HOST_BATCH)
HOST_BATCH = 2048


class ADKernel:
    def __init__(self, mesh, f=1.0):
        N, G, w = q2.basis_tables()
        h = np.asarray(mesh.h)
        self.N = torch.as_tensor(N)
        self.Gp = torch.as_tensor(G / h[None, None, :])
        self.wdet = torch.as_tensor(mesh.wdet())
        self.f = float(f)

    def density_sum(self, u, m, p):
        """``R_e = sum_q w|J| (e^m grad u . grad p - f p)`` of one element."""
        mq = self.N @ m
        pq = self.N @ p
        gu = torch.einsum("qak,a->qk", self.Gp, u)
        gp = torch.einsum("qak,a->qk", self.Gp, p)
        return torch.sum(self.wdet * (torch.exp(mq) * (gu * gp).sum(-1) - self.f * pq))

    def hess_slot(self, j):
        """``(ne, 27)^3 -> tuple over row slots i of (ne, 27, 27)`` by forward tangents
        over slot ``j`` (the reference's one differentiation primitive)."""
        def per_element(u, m, p):
            z = [u, m, p]

            def g(zj):
                zz = [zj if s == j else z[s] for s in range(3)]
                return grad(lambda a, b, c: self.density_sum(a, b, c), argnums=(0, 1, 2))(*zz)
            return jacfwd(g)(z[j])
        return vmap(per_element)

    def vectors(self):
        return vmap(grad(lambda a, b, c: self.density_sum(a, b, c), argnums=(0, 1, 2)))


def element_blocks(mesh, edofs, u, m, p, f=1.0, batch=HOST_BATCH):
    """``A, C, Wum, Wmm`` element matrices (numpy) by AD, in element windows."""
    K = ADKernel(mesh, f)
    U = torch.as_tensor(np.asarray(u)[edofs])
    M = torch.as_tensor(np.asarray(m)[edofs])
    P = torch.as_tensor(np.asarray(p)[edofs])
    slot_u, slot_m = K.hess_slot(STATE), K.hess_slot(PARAMETER)
    out = {"A": [], "C": [], "Wum": [], "Wmm": []}
    with torch.no_grad():
        for a in range(0, edofs.shape[0], batch):
            b = min(a + batch, edofs.shape[0])
            hu = slot_u(U[a:b], M[a:b], P[a:b])
            hm = slot_m(U[a:b], M[a:b], P[a:b])
            out["A"].append(hu[ADJOINT])
            out["C"].append(hm[ADJOINT])
            out["Wum"].append(hm[STATE])
            out["Wmm"].append(hm[PARAMETER])
    return {k: torch.cat(v).numpy() for k, v in out.items()}


def element_vectors(mesh, edofs, u, m, p, f=1.0, batch=HOST_BATCH):
    K = ADKernel(mesh, f)
    fn = K.vectors()
    U = torch.as_tensor(np.asarray(u)[edofs])
    M = torch.as_tensor(np.asarray(m)[edofs])
    P = torch.as_tensor(np.asarray(p)[edofs])
    outs = [[], [], []]
    with torch.no_grad():
        for a in range(0, edofs.shape[0], batch):
            b = min(a + batch, edofs.shape[0])
            g = fn(U[a:b], M[a:b], P[a:b])
            for s in range(3):
                outs[s].append(g[s])
    return {s: torch.cat(outs[s]).numpy() for s in range(3)}
