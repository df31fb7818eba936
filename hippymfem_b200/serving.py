"""A request loop for forward solves and Hessian-vector applies on meshes of several
sizes -- the MCMC / forward-UQ pattern in which the reference's ``Model`` is called
once per sample (modeling/model.py:139-261, modeling/reducedHessian.py:87-131).

Continuous batching over CUDA streams.  ``Server`` owns ``slots`` worker threads, each
with its own stream.  Requests wait in arrival order; a free slot takes the oldest one
as soon as its working set fits the device-memory budget (``memory_budget`` bytes):
workspaces stay resident per slot and mesh size between requests, and the least
recently used idle ones are released when a new size needs room.  Requests on different
slots run at the same time on the device (the library's calls release the GIL and
synchronise only their own stream), so requests that arrive while others run are
admitted as slots and memory free up.

Per mesh size the server keeps, once for all slots: the lattice, its Dirichlet markers,
the node coordinates and a misfit (pointwise observations).  Per slot and size: the
quadrature buffers and a ``SolvePlan`` (operator storage, Jacobi diagonal, PCG workspace;
its iteration batches replay a captured CUDA graph).  The batch length of the graph is
picked per mesh size by ``autotune`` (timed solves over a few candidates; the result of
a solve does not depend on it).

Work of a request (FP64 outer loops; FP32 operator and recurrence with FP64 reliable
updates when ``precision="mixed"``; with ``multigrid=True``, FP64 solves preconditioned
by the lattice multigrid V-cycle):

* ``forward``: ``m`` from the request's seed (the benchmark's cosine field, computed on
  the device), its quadrature data, the residual at ``u = 0`` (Dirichlet data 0), one
  Jacobi-PCG solve to ``rel_tolerance`` -> ``u``;
* ``hessian``: the forward solve, the adjoint solve of the misfit, then the true
  (misfit-only) Hessian action on ``v`` from the seed: ``C v``, ``W_um v``, ``W_mm v``
  from one directional quadrature pass, the two incremental solves, ``C^T p^`` and
  ``W_mu u^`` from the vector kernels -> ``H v`` (as ``ReducedHessian.TrueHessian``).

Every kernel is deterministic, so a request's result does not depend on what else runs.
"""

import math
import threading
import time

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr, stream_ptr
from .mesh import BoxMesh, DirichletBC, Q2Space
from .modeling import DiscreteStateObservation, PointwiseStateObservation
from .problem import STATE
from .sparse import Multigrid, SolveGroup, SolvePlan
from .synthetic import field_params, interior_points


class Request:
    """One request: ``kind`` "forward" or "hessian", mesh ``n`` (n^3 elements), the
    ``seed`` of its parameter field (and of ``v``), arrival time in seconds."""

    __slots__ = ("kind", "n", "seed", "arrival", "t_admit", "t_done", "result", "iterations",
                 "slot")

    def __init__(self, kind, n, seed, arrival=0.0):
        if kind not in ("forward", "hessian"):
            raise ValueError("kind must be 'forward' or 'hessian'")
        self.kind, self.n, self.seed, self.arrival = kind, int(n), int(seed), float(arrival)
        self.t_admit = self.t_done = None
        self.result = None
        self.iterations = []
        self.slot = None

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival


class _MeshState:
    """Read-only state of one mesh size, shared by the slots."""

    def __init__(self, n, device, nobs=256, sigma=0.1):
        self.n = n
        self.mesh = BoxMesh(n, device=device)
        self.V = Q2Space(self.mesh)
        self.bc = DirichletBC(self.V)
        self.coords = torch.as_tensor(self.mesh.node_coords(), device=device)
        pts = interior_points(nobs, seed=7)
        self.misfit = PointwiseStateObservation(self.V, pts, data=np.zeros(nobs),
                                                noise_variance=1e-4)
        self.sigma = sigma

    def field(self, seed):
        a, w, phi = field_params(seed, self.sigma)
        a = torch.as_tensor(a, device=self.coords.device)
        w = torch.as_tensor(w.astype(np.float64), device=self.coords.device)
        phi = torch.as_tensor(phi, device=self.coords.device)
        return torch.cos(2.0 * math.pi * (self.coords @ w.T) + phi) @ a

    def direction(self, seed):
        g = torch.Generator(device="cpu").manual_seed(int(seed) + 7919)
        return torch.randn(self.mesh.ndof, dtype=torch.float64, generator=g).to(self.coords.device)

    def footprint(self, precision, multigrid=False):
        """Bytes of one slot's workspace for this size."""
        nd, q = self.mesh.ndof, self.mesh.quad_bytes(_lib.HM_FP64)
        mg = Multigrid.workspace_bytes(self.mesh) if multigrid else 0
        jac = lib.hm_lattice_jacobian_bytes(self.mesh.handle, _lib.HM_FP64)
        if precision == "mixed":
            jac += lib.hm_lattice_jacobian_bytes(self.mesh.handle, _lib.HM_FP32)
            work = lib.hm_pcg_mixed_workspace_bytes(nd)
        else:
            work = lib.hm_pcg_workspace_bytes(nd)
        return int(2 * q + jac + work + mg + 14 * 8 * nd)


class _Workspace:
    """One slot's resident buffers for one mesh size."""

    def __init__(self, ms, precision, rtol, check_every, multigrid=False):
        self.ms = ms
        mesh, dev = ms.mesh, ms.mesh.device
        nq = (mesh.quad_bytes(_lib.HM_FP64) + 7) // 8
        self.quad = torch.empty(nq, dtype=torch.float64, device=dev)
        self.quad2 = torch.empty(nq, dtype=torch.float64, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.plan = SolvePlan(mesh, ms.bc.marker, precision, rel_tolerance=rtol,
                              check_every=check_every, multigrid=multigrid)
        nd = mesh.ndof
        self.vec = {k: torch.zeros(nd, dtype=torch.float64, device=dev)
                    for k in ("u", "p", "uh", "ph", "zero", "r1", "r2", "r3", "y")}
        # the misfit keeps scratch of its own: one per workspace (slots run concurrently)
        mis = ms.misfit
        self.misfit = DiscreteStateObservation(mis.B, mis.d, mis.noise_variance, device=dev)
        self.nbytes = ms.footprint(precision, multigrid)
        self.in_use = False
        self.last_used = 0.0

    # -- kernels of the path -------------------------------------------------------
    def _quad(self, buf, u, m, p, mhat=None):
        h = self.ms.mesh.handle
        if mhat is None:
            check(lib.hm_lattice_quadrature(h, ptr(u), ptr(m), ptr(p), _lib.HM_FP64, ptr(buf),
                                            ptr(self.status), stream_ptr()), "hm_lattice_quadrature")
        else:
            check(lib.hm_lattice_quadrature_dir(h, ptr(u), ptr(m), ptr(p), ptr(mhat), _lib.HM_FP64,
                                                ptr(buf), ptr(self.status), stream_ptr()),
                  "hm_lattice_quadrature_dir")

    def _vectors(self, buf, f, state=None, param=None, adj=None, zero_ess=False):
        check(lib.hm_lattice_assemble(self.ms.mesh.handle, ptr(buf), _lib.HM_FP64, None,
                                      ptr(self.ms.bc.marker), float(f), None, None, None, None,
                                      ptr(state), ptr(param), ptr(adj), int(bool(zero_ess)),
                                      stream_ptr()), "hm_lattice_assemble")

    # A request's work as a generator: it yields each solve it needs as (out, rhs) and
    # is resumed once out holds A^{-1} rhs, so that the solves of several same-size
    # requests can run as one group (SolveGroup); its return value is the result.
    def forward_steps(self, m, req):
        v = self.vec
        z = v["zero"]
        self._quad(self.quad, z, m, z)
        self.plan.set_point(self.quad)
        self._vectors(self.quad, 1.0, adj=self.plan.b, zero_ess=True)
        self.plan.b.neg_()
        yield v["u"], self.plan.b
        return v["u"]

    def hessian_steps(self, m, x, req):
        v, mask, mis = self.vec, self.ms.bc.mask, self.misfit
        u = yield from self.forward_steps(m, req)
        # adjoint: A^T p = -B^T (B u - d) / sigma^2
        mis.grad(STATE, [u, m, None], v["r1"])
        v["r1"].neg_().masked_fill_(mask, 0.0)
        yield v["p"], v["r1"]
        p = v["p"]
        # C x, W_um x, W_mm x from one directional pass (f = 0)
        self._quad(self.quad2, u, m, p, mhat=x)
        self._vectors(self.quad2, 0.0, state=v["r2"], param=v["y"], adj=v["r1"])
        v["r1"].masked_fill_(mask, 0.0)                       # C x, rows eliminated
        v["r2"].masked_fill_(mask, 0.0)                       # W_um x
        yield v["uh"], v["r1"]                                # A u^ = C x
        mis.apply_ij(STATE, STATE, v["uh"], v["r3"])          # W_uu u^
        v["r3"].sub_(v["r2"]).masked_fill_(mask, 0.0)
        yield v["ph"], v["r3"]                                # A^T p^ = W_uu u^ - W_um x
        # y = W_mm x + C^T p^ - W_mu u^
        self._quad(self.quad2, u, m, v["ph"].masked_fill_(mask, 0.0))
        self._vectors(self.quad2, 0.0, param=v["r3"])
        v["y"].add_(v["r3"])
        self._quad(self.quad2, v["uh"].masked_fill_(mask, 0.0), m, p)
        self._vectors(self.quad2, 0.0, param=v["r3"])
        v["y"].sub_(v["r3"])
        return v["y"]

    def steps(self, req):
        ms = self.ms
        m = ms.field(req.seed)
        if req.kind == "forward":
            return self.forward_steps(m, req)
        return self.hessian_steps(m, ms.direction(req.seed), req)

    def _drive(self, gen, req):
        try:
            out, rhs = next(gen)
            while True:
                self.plan.solve(out, rhs)
                req.iterations.append(self.plan.last.iterations)
                out, rhs = gen.send(None)
        except StopIteration as stop:
            return stop.value

    def forward(self, m, req):
        return self._drive(self.forward_steps(m, req), req)

    def hessian(self, m, x, req):
        return self._drive(self.hessian_steps(m, x, req), req)

    def close(self):
        self.plan.close()


class Server:
    """``Server(slots=4, precision="mixed", rel_tolerance=1e-8, memory_budget=None)``.

    ``run(requests)`` feeds the requests at their arrival times (seconds from the call)
    and returns when all are done; each request gets ``result`` (a host FP64 array),
    ``t_admit``, ``t_done`` (seconds from the call), ``iterations`` and ``slot``.
    ``memory_budget``: bytes the slots' workspaces may hold (default: half of the free
    device memory)."""

    def __init__(self, slots=4, precision="mixed", rel_tolerance=1e-8, memory_budget=None,
                 device=None, check_every=None, keep_results=True, multigrid=False,
                 group_size=1):
        if multigrid and precision != "fp64":
            raise ValueError("the multigrid solves are FP64")
        self.multigrid = bool(multigrid)
        self.device = torch.device(device if device is not None else "cuda")
        self.slots = int(slots)
        self.precision = precision
        self.rtol = float(rel_tolerance)
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget = free // 2
        self.budget = int(memory_budget)
        self.fixed_check_every = check_every
        self.keep_results = keep_results
        self.meshes = {}
        self.tuned = {}
        # same-size batching (FP64 solves only): a slot takes up to group_size waiting
        # requests of one size and kind and runs their solves as one group
        self.group_size = max(1, int(group_size))
        self.group_by_n = {}
        self._groups = {}
        self._busy = 0           # slots serving a request now
        self._ws = {}            # (slot, n) -> _Workspace
        self._resident = 0
        self.peak_resident = 0
        self._lock = threading.Condition()
        self._streams = [torch.cuda.Stream(device=self.device) for _ in range(self.slots)]

    # -- per-size state ------------------------------------------------------------
    def mesh_state(self, n):
        with self._lock:
            ms = self.meshes.get(n)
        if ms is None:
            ms = _MeshState(n, self.device)
            with self._lock:
                ms = self.meshes.setdefault(n, ms)
        return ms

    def check_every(self, n):
        if self.fixed_check_every is not None:
            return int(self.fixed_check_every)
        return self.tuned.get(n, 16)

    def group_size_for(self, n):
        if self.precision != "fp64":
            return 1
        return int(self.group_by_n.get(n, self.group_size))

    def autotune(self, sizes, candidates=(4, 8, 16, 32), reps=3, group_candidates=()):
        """Pick the graph batch length per mesh size: the fastest forward solve (CUDA
        events, in a side stream, after one warm-up that captures the graph).  With
        ``group_candidates`` (FP64 servers) also the group size: the one whose grouped
        forward requests take the least time per request, a larger group only where it
        saves at least ``GROUP_GAIN`` of that time."""
        stream = torch.cuda.Stream(device=self.device)
        for n in sizes:
            ms = self.mesh_state(n)
            best = None
            for ce in candidates:
                ws = _Workspace(ms, self.precision, self.rtol, ce, self.multigrid)
                req = Request("forward", n, 0)
                with torch.cuda.stream(stream):
                    m = ms.field(0)
                    ws.forward(m, req)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    for _ in range(reps):
                        ws.forward(m, req)
                    e1.record(stream)
                stream.synchronize()
                t = e0.elapsed_time(e1) / reps
                ws.close()
                del ws
                if best is None or t < best[0]:
                    best = (t, ce)
            self.tuned[n] = best[1]
            if group_candidates and self.precision == "fp64":
                self.group_by_n[n] = self._tune_group(ms, best[1], group_candidates, reps,
                                                      stream)
        return dict(self.tuned)

    # a larger group must cut the time per request by this fraction against the best
    # smaller one: a group holds one slot for all its members, so a group that saves
    # little lengthens every member's latency and takes concurrency from the other slots
    GROUP_GAIN = 0.2

    def _tune_group(self, ms, ce, group_candidates, reps, stream):
        best = None
        for k in sorted(int(c) for c in group_candidates):
            wss = [_Workspace(ms, self.precision, self.rtol, ce, self.multigrid)
                   for _ in range(int(k))]
            reqs = [Request("forward", ms.n, j) for j in range(int(k))]
            grp = SolveGroup([w.plan for w in wss]) if k > 1 else None
            with torch.cuda.stream(stream):
                self._run_group_with(wss, reqs, grp)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    self._run_group_with(wss, reqs, grp)
                e1.record(stream)
            stream.synchronize()
            t = e0.elapsed_time(e1) / (reps * int(k))
            if grp is not None:
                grp.close()
            for w in wss:
                w.close()
            if best is None or t < (1.0 - self.GROUP_GAIN) * best[0]:
                best = (t, int(k))
        return best[1]

    def _run_group_with(self, wss, reqs, grp):
        """The requests' work on their workspaces (one each): alone through the
        workspace's own solves, or with every solve of the group as one SolveGroup."""
        gens = [w.steps(r) for w, r in zip(wss, reqs)]
        if grp is None:
            return [wss[0]._drive(gens[0], reqs[0])]
        cur = [next(g) for g in gens]
        results = [None] * len(gens)
        while True:
            res = grp.solve([c[0] for c in cur], [c[1] for c in cur])
            for r, pr in zip(reqs, res):
                r.iterations.append(pr.iterations)
            nxt = []
            for j, g in enumerate(gens):
                try:
                    nxt.append(g.send(None))
                except StopIteration as stop:
                    results[j] = stop.value
                    nxt.append(None)
            if all(x is None for x in nxt):
                return results
            if any(x is None for x in nxt):
                raise RuntimeError("the requests of a group took different numbers of solves")
            cur = nxt

    def _group(self, wss):
        key = tuple(id(w) for w in wss)
        grp = self._groups.get(key)
        if grp is None:
            grp = self._groups[key] = SolveGroup([w.plan for w in wss])
        return grp

    def _drop_groups(self, ws):
        for key in [k for k in self._groups if id(ws) in k]:
            self._groups.pop(key).close()

    # -- admission -------------------------------------------------------------------
    def _acquire(self, slot, n, j=0, block=True):
        """The slot's j-th workspace for size n, ``(ws, None, True)``; when missing,
        room is made for it (idle workspaces released, least recently used first) and
        ``(None, bytes reserved, True)`` returned.  Without room it waits for some
        (``block``) or returns ``(None, None, False)``.  Under the lock."""
        ws = self._ws.get((slot, n, j))
        if ws is not None:
            ws.in_use = True
            return ws, None, True
        need = self.mesh_state_locked(n).footprint(self.precision, self.multigrid)
        while self._resident + need > self.budget:
            idle = [(w.last_used, k) for k, w in self._ws.items() if not w.in_use]
            if idle:
                _, k = min(idle)
                w = self._ws.pop(k)
                self._resident -= w.nbytes
                self._drop_groups(w)
                w.close()
                continue
            if not block:
                return None, None, False
            if self._resident == 0:
                raise MemoryError("a workspace for n=%d needs %d bytes, more than the budget"
                                  % (n, need))
            self._lock.wait()
        self._resident += need
        self.peak_resident = max(self.peak_resident, self._resident)
        return None, need, True

    def mesh_state_locked(self, n):
        ms = self.meshes.get(n)
        if ms is None:
            self._lock.release()
            try:
                ms = self.mesh_state(n)
            finally:
                self._lock.acquire()
        return ms

    def _worker(self, slot, pending, t0, done):
        stream = self._streams[slot]
        while True:
            with self._lock:
                while not pending and not done["fed"]:
                    self._lock.wait()
                if not pending:
                    return
                req = pending.popleft()
                # the oldest request, and (FP64) up to group_size - 1 more of its size and
                # kind that are waiting, taken in arrival order -- only from a backlog:
                # while another slot is idle, a waiting request is served there, in
                # parallel, rather than in this slot's group
                group = [req]
                kmax = self.group_size_for(req.n)
                idle_others = self.slots - 1 - self._busy
                if kmax > 1 and len(pending) > idle_others:
                    for other in pending:
                        if len(group) >= kmax:
                            break
                        if other.n == req.n and other.kind == req.kind:
                            group.append(other)
                    for other in group[1:]:
                        pending.remove(other)
                got = []
                for j, r in enumerate(group):
                    ws, reserved, ok = self._acquire(slot, r.n, j, block=j == 0)
                    if not ok:                    # no room for more: the rest waits
                        for r2 in reversed(group[j:]):
                            pending.appendleft(r2)
                        group = group[:j]
                        break
                    got.append((ws, reserved))
                self._busy += 1
            wss = []
            for j, (ws, reserved) in enumerate(got):
                if ws is None:
                    ms = self.mesh_state(req.n)
                    with torch.cuda.stream(stream):
                        ws = _Workspace(ms, self.precision, self.rtol, self.check_every(req.n),
                                        self.multigrid)
                    ws.nbytes = reserved
                    ws.in_use = True
                    with self._lock:
                        self._ws[(slot, req.n, j)] = ws
                wss.append(ws)
            t_admit = time.perf_counter() - t0
            for r in group:
                r.t_admit, r.slot = t_admit, slot
            with torch.cuda.stream(stream):
                grp = self._group(wss) if len(wss) > 1 else None
                outs = self._run_group_with(wss, group, grp)
                res = [o.to("cpu", non_blocking=False) if self.keep_results else None
                       for o in outs]
                stream.synchronize()
            t_done = time.perf_counter() - t0
            for r, x in zip(group, res):
                r.result = x.numpy() if x is not None else None
                r.t_done = t_done
            with self._lock:
                for ws in wss:
                    ws.in_use = False
                    ws.last_used = t_done
                self._busy -= 1
                self._lock.notify_all()

    def run(self, requests):
        """Serve ``requests`` (arrival times in seconds from now); returns them."""
        import collections

        reqs = sorted(requests, key=lambda r: r.arrival)
        for n in sorted({r.n for r in reqs}):
            self.mesh_state(n)
        pending = collections.deque()
        done = {"fed": False}
        t0 = time.perf_counter()
        errors = []

        def guarded(slot):
            try:
                self._worker(slot, pending, t0, done)
            except BaseException as e:                    # noqa: BLE001
                errors.append(e)
                with self._lock:
                    done["fed"] = True
                    pending.clear()
                    self._lock.notify_all()

        threads = [threading.Thread(target=guarded, args=(k,), daemon=True)
                   for k in range(self.slots)]
        for t in threads:
            t.start()
        for r in reqs:
            delay = r.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            with self._lock:
                if errors:
                    break
                pending.append(r)
                self._lock.notify_all()
        with self._lock:
            done["fed"] = True
            self._lock.notify_all()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        return reqs

    def close(self):
        with self._lock:
            for g in self._groups.values():
                g.close()
            self._groups.clear()
            for w in self._ws.values():
                w.close()
            self._ws.clear()
            self._resident = 0


def latency_stats(requests):
    lat = np.array([r.latency for r in requests if r.latency is not None])
    span = max(r.t_done for r in requests) - min(r.arrival for r in requests)
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "requests_per_s": len(lat) / span,
            "n": int(len(lat))}


def poisson_trace(nreq, rate, sizes=(8, 12, 16, 24, 32, 48), p_forward=0.7, seed=0):
    """``nreq`` requests with Poisson arrivals at ``rate`` per second, sizes uniform over
    ``sizes``, 70% forward solves / 30% Hessian actions, one parameter seed each."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, nreq))
    n = rng.choice(sizes, nreq)
    kind = np.where(rng.random(nreq) < p_forward, "forward", "hessian")
    return [Request(k, int(nn), 1000 + i, float(ti)) for i, (k, nn, ti) in enumerate(zip(kind, n, t))]


def plain_fp64(req, device=None, rel_tolerance=1e-8, cache=None):
    """The same request through the library's plain per-request path: a fresh
    ``PDEVariationalProblem`` / ``Model`` / ``ReducedHessian`` in FP64 on the default
    stream (no resident workspace, no graphs).  The reference for the server's results
    and the baseline of the serving benchmark."""
    from .modeling import Model, ReducedHessian
    from .problem import PDEVariationalProblem

    cache = {} if cache is None else cache
    ms = cache.get(req.n)
    if ms is None:
        ms = cache[req.n] = _MeshState(req.n, device or "cuda")
    prob = PDEVariationalProblem([ms.V, ms.V, ms.V], f=1.0, bc=ms.bc, solver_tolerance=rel_tolerance,
                                 matrix_free_solves=True, check_finite=False)
    m = ms.field(req.seed)
    u = ms.V.vector()
    if req.kind == "forward":
        prob.solveFwd(u, [u, m, None])
        return u
    model = Model(prob, None, ms.misfit)
    p = ms.V.vector()
    x = [u, m, p]
    model.solveFwd(u, x)
    model.solveAdj(p, x)
    prob.setLinearizationPoint(x, matrix_free=True)
    H = ReducedHessian(model)
    y = ms.V.vector()
    H.mult(ms.direction(req.seed), y)
    return y
