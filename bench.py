#!/usr/bin/env python
"""Benchmark of the Q2 log-conductivity assembly + Hessian-action path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 64]
                    [--config main|precision|differentiation|solve] [--shard]

Workload (one step): the linearization point of the 64^3 Q2 configuration in FP64 --
pointwise data of (u, m, p) and one fused assembly of the full block set (A = K, its
adjoint A^T = A, C = dr/dm, W_um, W_mm) with the assembled vectors (residual, dR/dm,
dR/du) into the diagonal-first CSR pattern, eliminated on the boundary.  ``value`` is
Q2 elements assembled per second (whole job), device-timed with inputs resident.
After the timed steps, Hessian actions (misfit 4096 pointwise observations, two
matrix-free solves at rtol 1e-12 each: multigrid-PCG as the headline, Jacobi-PCG and
mixed-precision Jacobi-PCG beside it) are timed for H-applies/s and their p50/p99
latency.  ``e2e`` repeats the step through the public API with the fields copied
from pinned host memory and the gradient dR/dm copied back, inside the timed region.

Under torchrun (N > 1) every rank runs an independent replica of the workload (the
path does not shard: one GPU per request stream); value = all ranks' elements / the
slowest rank's time (every timing is the maximum over the ranks).  ``--impl reference`` times the reference's algorithm on the host
cores instead (element blocks by forward-over-reverse AD in 2048-element windows and a
bincount scatter, restated in oracle/; rank 0 only).
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Q2 elems/s, H-applies/s at 64^3 vs plain FP64; p50/p99 batched-solve latency"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes per algorithmic byte of k_tile_assemble<double>, from one ncu capture of the
# kernel at 48^3 (dram__bytes_read.sum + dram__bytes_write.sum over the bytes it must move)
TRAFFIC_PER_ALG_BYTE = 2030.9 / 2043.7


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--happly", type=int, default=5, help="timed Hessian actions")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving", type=int, default=2000,
                    help="requests of the serving trace (0: skip)")
    ap.add_argument("--shard", action="store_true",
                    help="the Hessian action sharded over z-slabs of the 64^3 lattice across "
                         "the ranks (one per GPU; halo exchange by point-to-point messages, "
                         "plane-ordered dot products; Jacobi-PCG), H-applies/s, strong scaling")
    ap.add_argument("--mg-precision", choices=("fp64", "fp32"), default="fp64",
                    help="the V-cycle's precision in --config solve (the CG stays FP64)")
    ap.add_argument("--config", choices=("main", "precision", "differentiation", "solve"),
                    default="main",
                    help="precision: 128^3, FP32 contractions and mixed-precision Hessian "
                         "actions against FP64; differentiation: 32^3 finite-difference "
                         "checks of the autograd wrappers; solve: one incremental solve "
                         "(FP64 multigrid-PCG, rtol 1e-12) at --n, repeated")
    return ap.parse_args()


# ------------------------------------------------------------------------ ranks
def max_over_ranks(values, world, dev=None):
    """Each value's maximum over the ranks (every rank calls this with the same number
    of values, at the same point); the values themselves on one rank."""
    vals = [float(v) for v in values]
    if world == 1:
        return vals
    import torch
    import torch.distributed as dist

    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def whole_job_rate(units_per_rank, ms, world):
    """Units per second of the whole job: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / (ms / 1000.0)


# ------------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi samples during the timed region (read-only queries)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # wait (at most 5 s) for the first sample, so the timed region is covered
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, smax, power, reasons = [], None, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                power.append(float(r[3]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def peaks():
    try:
        with open(PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU baselines
def cpu_port_baseline(budget_s=12.0, n_sample=32):
    """The oracle's closed-form assembly of every block (oracle/q2.py) on a 32^3 sample
    of the per-element work (a working set well beyond the host caches, as the 64^3 one
    is), bincount scatter and elimination included."""
    from oracle import q2

    try:
        from threadpoolctl import threadpool_info
        cores = max([i.get("num_threads", 1) for i in threadpool_info()] + [1])
    except Exception:                                     # noqa: BLE001
        cores = os.cpu_count() or 1
    mesh = q2.Lattice(n_sample)
    E = mesh.edofs()
    rng = np.random.default_rng(0)
    u, m, p = (rng.standard_normal(mesh.ndof) for _ in range(3))
    ess = np.zeros(mesh.ndof, bool)
    ess[mesh.boundary_dofs()] = True
    pat = q2.build_tables(E, E, mesh.ndof, mesh.ndof, True)
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s or done == 0:
        blk = q2.element_blocks(mesh, E, u, 0.1 * m, p)
        for k in blk:
            q2.assemble_block(k, pat, blk[k], ess)
        q2.element_vectors(mesh, E, u, 0.1 * m, p)
        done += mesh.ne
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "elements/s", "cores": int(cores), "kind": "port",
            "sample": "oracle closed-form assembly of A, C, Wum, Wmm + vectors on %d^3 "
                      "(%d elements) repeated for %.1f s" % (n_sample, mesh.ne, dt)}


def reference_step_fn(n_sample=32):
    """One step of the reference's host algorithm on a 32^3 sample of the 64^3 workload
    (32,768 elements, 16.97 M entries per block: a working set beyond the host caches,
    as the full size is): blocks by AD in 2048-element windows (oracle/ad.py) + bincount
    scatter + folded elimination."""
    from oracle import ad, q2

    mesh = q2.Lattice(n_sample)
    E = mesh.edofs()
    rng = np.random.default_rng(0)
    u, m, p = (rng.standard_normal(mesh.ndof) for _ in range(3))
    ess = np.zeros(mesh.ndof, bool)
    ess[mesh.boundary_dofs()] = True
    pat = q2.build_tables(E, E, mesh.ndof, mesh.ndof, True)

    def step():
        blk = ad.element_blocks(mesh, E, u, 0.1 * m, p)
        for k in blk:
            q2.assemble_block(k, pat, blk[k], ess)
        ad.element_vectors(mesh, E, u, 0.1 * m, p)
        return mesh.ne
    return step


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    torch.set_num_threads(os.cpu_count() or 1)
    step = reference_step_fn()
    for _ in range(a.warmup):
        step()
    t0 = time.perf_counter()
    done = 0
    for _ in range(a.steps):
        done += step()
    dt = time.perf_counter() - t0
    v = done / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "elements/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000.0 * dt / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "Q2 hex linearization-point assembly (A, C, Wum, Wmm + "
                                   "vectors), reference algorithm on the host",
                       "mesh": "32^3 sample of the 64^3 per-element work", "precision": "fp64"},
            "cpu_baseline": {"value": v, "unit": "elements/s", "cores": torch.get_num_threads(),
                             "kind": "port",
                             "sample": "32^3 (32768 elements) per step: torch.func "
                                       "forward-over-reverse AD in 2048-element windows "
                                       "+ bincount scatter + elimination"},
            "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------- ours
def _capacity(srv, sizes, poisson_trace, n=240):
    """Requests/s of a burst from the serving mix, all arriving at once, after a first
    burst has created every slot's workspaces and captured its graphs."""
    from hippymfem_b200.serving import latency_stats

    for seed in (10, 11):
        burst = poisson_trace(n, 1e9, sizes, seed=seed)
        for r in burst:
            r.arrival = 0.0
        srv.run(burst)
    return latency_stats(burst)["requests_per_s"]


def run_serving(nreq, dev, sizes=(8, 12, 16, 24, 32, 48), slots=4, plain_sample=200):
    """The serving configuration: requests on n^3 meshes, n uniform over ``sizes``, 70%
    forward solves / 30% Hessian actions (solves to rtol 1e-8), Poisson arrivals at 80% of
    the measured capacity, through the request loop: 4 slots, FP64 solves preconditioned by
    the lattice multigrid V-cycle, one request per slot, graph-replayed iteration batches
    (batch length per size from the autotuner); the same trace through the server that
    batches same-size requests into solve groups from a backlog (one CUDA graph per
    iteration batch for the whole group).  Beside it the same mix with the FP32-recurrence solves
    (FP64 reliable updates; not groupable) and the plain FP64 per-request path on a
    sample of the same trace, one request at a time."""
    import torch

    from hippymfem_b200.serving import Server, latency_stats, plain_fp64, poisson_trace

    def serve(srv, what, capacity=None):
        if capacity is None:
            capacity = _capacity(srv, sizes, poisson_trace)
        trace = poisson_trace(nreq, 0.8 * capacity, sizes, seed=12)
        srv.run(trace)
        st = latency_stats(trace)
        st.update({"capacity_requests_per_s": capacity, "arrival_rate": 0.8 * capacity,
                   "slots": slots, "peak_workspace_bytes": srv.peak_resident, "what": what,
                   "solves_per_s": sum(len(r.iterations) for r in trace) / (
                       max(r.t_done for r in trace) - min(r.arrival for r in trace))})
        return st, trace

    # the load: 80 % of the capacity of the FP64 multigrid server serving one request per
    # slot (a burst); the headline is that server.  The same trace through the server that
    # also batches same-size requests into solve groups from a backlog is reported beside
    # it with its own burst capacity (groups full): in this mix a group's members finish
    # together, later than alone, and the groups' capacity is barely above the other's
    srv = Server(slots=slots, precision="fp64", multigrid=True, rel_tolerance=1e-8, device=dev,
                 keep_results=False)
    tuned = srv.autotune(sizes, candidates=(4, 8, 16), reps=2)
    st, trace = serve(srv, "FP64 solves with the lattice multigrid V-cycle, one request per "
                           "slot, graph-replayed iteration batches")
    st["graph_batch_by_n"] = {str(k): v for k, v in tuned.items()}
    cap = st["capacity_requests_per_s"]
    srv.close()
    srv = Server(slots=slots, precision="fp64", multigrid=True, rel_tolerance=1e-8, device=dev,
                 keep_results=False)
    tuned_g = srv.autotune(sizes, candidates=(4, 8, 16), reps=2, group_candidates=(1, 2, 4))
    cap_groups = _capacity(srv, sizes, poisson_trace)
    st_g, _ = serve(srv, "the same trace through the same server with same-size requests "
                         "batched into solve groups from a backlog", capacity=cap)
    st["solve_groups"] = {k: st_g[k] for k in ("p50_ms", "p99_ms", "mean_ms", "requests_per_s",
                                                "arrival_rate", "what")}
    st["solve_groups"]["capacity_with_groups_requests_per_s"] = cap_groups
    st["solve_groups"]["group_size_by_n"] = {str(k): v for k, v in srv.group_by_n.items()}
    st["solve_groups"]["graph_batch_by_n"] = {str(k): v for k, v in tuned_g.items()}
    srv.close()
    srv = Server(slots=slots, precision="mixed", rel_tolerance=1e-8, device=dev,
                 keep_results=False)
    tuned_mx = srv.autotune(sizes, candidates=(8, 16, 32), reps=2)
    st_mx, _ = serve(srv, "the same request mix (same sizes, seeds) at 80% of this server's "
                          "capacity: Jacobi-PCG with the FP32 recurrence and FP64 reliable "
                          "updates, one request per slot")
    st_mx["graph_batch_by_n"] = {str(k): v for k, v in tuned_mx.items()}
    st["mixed_fp32"] = st_mx
    srv.close()
    # the plain FP64 path, request by request (no overlap, no resident workspace)
    cache = {}
    sample = trace[:plain_sample]
    for r in sample[:6]:
        plain_fp64(r, dev, cache=cache)
    lat = []
    for r in sample:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        plain_fp64(r, dev, cache=cache)
        e1.record()
        torch.cuda.synchronize()
        lat.append(e0.elapsed_time(e1))
    st["plain_fp64"] = {"p50_ms": float(np.percentile(lat, 50)),
                        "p99_ms": float(np.percentile(lat, 99)),
                        "requests_per_s": 1000.0 * len(lat) / float(np.sum(lat)),
                        "sample": len(lat),
                        "what": "service time of each request alone (no queueing), FP64, "
                                "fresh problem objects, default stream"}
    st["trace"] = ("%d-request Poisson trace at 80%% of the server's capacity (a burst), n in %s, "
                   "70%% forward / 30%% Hessian actions, rtol 1e-8; latency = completion - "
                   "arrival" % (nreq, list(sizes)))
    return st


def run_ours(a):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import hippymfem_b200 as hm
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr
    from hippymfem_b200.sparse import default_smoothing_degree
    from hippymfem_b200.synthetic import interior_points, log_conductivity, normal_vector

    dev = torch.device("cuda", local)
    n = a.n
    mesh = hm.BoxMesh(n, device=dev)
    V = hm.Q2Space(mesh)
    bc = hm.DirichletBC(V)
    pat = hm.LatticePattern(mesh)
    ne, nd, nnz = mesh.ne, mesh.ndof, mesh.nnz
    coords = mesh.node_coords()
    m_h = log_conductivity(coords, seed=0)
    rng = np.random.default_rng(11)
    u_h, p_h = rng.standard_normal(nd), rng.standard_normal(nd)
    u, m, p = (torch.as_tensor(x, device=dev) for x in (u_h, m_h, p_h))
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    vals = [torch.empty(nnz, dtype=torch.float64, device=dev) for _ in range(4)]
    vecs = [torch.empty(nd, dtype=torch.float64, device=dev) for _ in range(3)]
    marker = bc.marker
    stream = torch.cuda.current_stream()
    sp = stream_ptr(stream)
    ev_k0 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ev_k1 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]

    def step(i=None):
        check(lib.hm_lattice_quadrature(mesh.handle, ptr(u), ptr(m), ptr(p), _lib.HM_FP64,
                                        ptr(quad), ptr(status), sp))
        if i is not None:
            ev_k0[i].record(stream)
        check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, ptr(pat.indptr),
                                      ptr(marker), 1.0, *(ptr(v) for v in vals),
                                      *(ptr(v) for v in vecs), 0, sp))
        if i is not None:
            ev_k1[i].record(stream)

    launches_per_step = 2
    clocks = Clocks(local)
    clocks.start()
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for i in range(a.steps):
        step(i)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    k_ms = statistics.mean(ev_k0[i].elapsed_time(ev_k1[i]) for i in range(a.steps))
    ms, k_ms = max_over_ranks([ms, k_ms], world, dev)
    assert int(status.item()) == 0, "non-finite values in the benchmark fields"
    value = whole_job_rate(ne * a.steps, ms, world)

    # roofline of the fused assembly kernel: bytes it must move per launch
    alg_bytes = 8 * nnz * 4 + 8 * nd * 3 + 8 * 216 * ne + 4 * (nd + 1) + nd
    peak, peak_kind = peaks()
    achieved = alg_bytes / (k_ms / 1000.0) / 1e9
    step_bytes = 8 * nnz * 4 + 8 * nd * 5            # 4 blocks, 3 fields in, 2 vectors out

    # ------------------------------------------------------------ e2e (public API)
    # Every step copies its fields from pinned host memory, sets the linearization point
    # (all blocks and the vectors of the point in the fused pass) and the gradient dR/dm
    # through the public API, and copies the gradient back.  The copies run on two copy
    # streams (host to device, device to host: the two directions of the link) with two
    # buffer sets, so that step i + 1's inputs and step i - 1's result move while step i
    # computes; every copy of a timed step is inside the timed region.
    pin = [torch.empty(nd, dtype=torch.float64).pin_memory() for _ in range(3)]
    for h, src in zip(pin, (u_h, m_h, p_h)):
        h.copy_(torch.as_tensor(src))
    gpin = [torch.empty(nd, dtype=torch.float64).pin_memory() for _ in range(2)]
    prob = hm.PDEVariationalProblem([V, V, V], f=1.0, bc=bc, check_finite=False)
    prob._pattern = pat
    ins = [[torch.empty(nd, dtype=torch.float64, device=dev) for _ in range(3)] for _ in range(2)]
    gs = [torch.empty(nd, dtype=torch.float64, device=dev) for _ in range(2)]
    cstream = torch.cuda.Stream(device=dev)            # host -> device
    dstream = torch.cuda.Stream(device=dev)            # device -> host
    ready = [torch.cuda.Event() for _ in range(2)]     # buffer set b: inputs landed
    done = [torch.cuda.Event() for _ in range(2)]      # buffer set b: its step computed
    taken = [torch.cuda.Event() for _ in range(2)]     # buffer set b: its gradient copied out

    def h2d(b, after=None):
        with torch.cuda.stream(cstream):
            if after is not None:                      # the step that read this set is done
                cstream.wait_event(after)
            for dst, src in zip(ins[b], pin):
                dst.copy_(src, non_blocking=True)
            ready[b].record(cstream)

    def e2e_run(nsteps, start=None):
        for cs in (cstream, dstream):
            if start is not None:
                cs.wait_event(start)
        for b in range(min(2, nsteps)):
            h2d(b)
        for i in range(nsteps):
            b = i % 2
            stream.wait_event(ready[b])
            if i >= 2:                                 # gs[b] copied out two steps ago
                stream.wait_event(taken[b])
            prob._jac_cache = None                     # a new point: the Jacobian too
            prob.setLinearizationPoint(ins[b])
            prob.evalGradientParameter(ins[b], gs[b])
            done[b].record(stream)
            with torch.cuda.stream(dstream):
                dstream.wait_event(done[b])
                gpin[b].copy_(gs[b], non_blocking=True)
                taken[b].record(dstream)
            if i + 2 < nsteps:
                h2d(b, after=done[b])
        stream.wait_stream(cstream)
        stream.wait_stream(dstream)

    e2e_run(3)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_steps = max(3, a.steps // 2)
    e0.record(stream)
    e2e_run(e_steps, start=e0)
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = e0.elapsed_time(e1)
    (e_ms,) = max_over_ranks([e_ms], world, dev)
    e2e_value = whole_job_rate(ne * e_steps, e_ms, world)
    del prob
    torch.cuda.empty_cache()

    # ------------------------------------------------------ Hessian actions
    prob = hm.PDEVariationalProblem([V, V, V], f=1.0, bc=bc, matrix_free_solves=True,
                                    check_finite=False, solver_tolerance=1e-12)
    prob._pattern = pat
    pts = interior_points(4096, seed=2)
    misfit = hm.PointwiseStateObservation(V, pts, data=np.zeros(4096), noise_variance=1.0)
    model = hm.Model(prob, None, misfit)
    mt = torch.as_tensor(log_conductivity(coords, seed=1), device=dev)
    ut = V.vector()
    model.solveFwd(ut, [ut, mt, None])
    Bu = misfit.Bh @ ut.cpu().numpy()
    noise = 0.01 * float(ut.abs().max())
    misfit.d.copy_(torch.as_tensor(Bu + noise * np.random.default_rng(5).standard_normal(4096)))
    misfit.noise_variance = noise ** 2
    uu, pp = V.vector(), V.vector()
    x = [uu, m, pp]
    model.solveFwd(uu, x)
    model.solveAdj(pp, x)
    model.setPointForHessianEvaluations(x)
    H = hm.ReducedHessian(model)
    v = torch.as_tensor(normal_vector(nd, seed=4), device=dev)
    y = V.vector()
    H.mult(v, y)
    torch.cuda.synchronize()
    lat = []
    H.iterations.clear()
    for _ in range(a.happly):
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        H.mult(v, y)
        h1.record(stream)
        torch.cuda.synchronize()
        lat.append(h0.elapsed_time(h1))
    iters = list(H.iterations)
    y64 = y.clone()

    # the same actions with mixed-precision solves (FP32 recurrence, FP64 reliable updates)
    del H, model, prob
    torch.cuda.empty_cache()
    prob = hm.PDEVariationalProblem([V, V, V], f=1.0, bc=bc, solver_precision="mixed",
                                    check_finite=False, solver_tolerance=1e-12)
    prob._pattern = pat
    model = hm.Model(prob, None, misfit)
    model.setPointForHessianEvaluations(x)
    H = hm.ReducedHessian(model)
    H.mult(v, y)
    torch.cuda.synchronize()
    lat32 = []
    H.iterations.clear()
    for _ in range(a.happly):
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        H.mult(v, y)
        h1.record(stream)
        torch.cuda.synchronize()
        lat32.append(h0.elapsed_time(h1))
    mixed_err = float((y - y64).norm() / y64.norm())
    iters32 = list(H.iterations)
    del H, model, prob
    torch.cuda.empty_cache()

    # the same actions with the lattice multigrid preconditioner, in a stream of their
    # own, where the solver replays its iteration batches as CUDA graphs: the FP64 CG with
    # the V-cycle in FP64 ("fp64") and in FP32 ("mixed")
    hs = torch.cuda.Stream(device=dev)

    def mg_actions(solver_precision):
        torch.cuda.synchronize()
        with torch.cuda.stream(hs):
            prob = hm.PDEVariationalProblem([V, V, V], f=1.0, bc=bc, preconditioner="mg",
                                            check_finite=False, solver_tolerance=1e-12,
                                            solver_precision=solver_precision)
            prob._pattern = pat
            model = hm.Model(prob, None, misfit)
            model.setPointForHessianEvaluations(x)
            H = hm.ReducedHessian(model)
            H.mult(v, y)
            hs.synchronize()
            lats = []
            H.iterations.clear()
            for _ in range(a.happly):
                h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                h0.record(hs)
                H.mult(v, y)
                h1.record(hs)
                hs.synchronize()
                lats.append(h0.elapsed_time(h1))
        torch.cuda.synchronize()
        its = list(H.iterations)
        del H, model, prob
        torch.cuda.empty_cache()
        return lats, y.clone(), its

    lat_mg, y_mg, iters_mg = mg_actions("fp64")
    mg_err = float((y_mg - y64).norm() / y64.norm())
    lat_mg32, y_mg32, iters_mg32 = mg_actions("mixed")
    mg32_err = float((y_mg32 - y64).norm() / y64.norm())
    mg32_vs_mg = float((y_mg32 - y_mg).norm() / y_mg.norm())
    ck = clocks.stop()

    # the latency figures of the three solvers: each the maximum over the ranks
    def lat_stats(ls):
        return [statistics.mean(ls), float(np.percentile(ls, 50)), float(np.percentile(ls, 99))]

    hs_mg, hs_j, hs_32, hs_mg32 = (max_over_ranks(lat_stats(ls), world, dev)
                                   for ls in (lat_mg, lat, lat32, lat_mg32))
    mg_degree = default_smoothing_degree(mesh)

    serving = None
    if a.serving > 0 and world == 1:
        serving = run_serving(a.serving, dev)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_port_baseline()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "elements/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "Q2 hex %d^3 linearization-point assembly: A(=K=A^T), C, "
                                   "Wum, Wmm + residual, dR/dm, dR/du, FP64, boundary "
                                   "eliminated" % n,
                       "elements": ne, "dofs": nd, "nnz_per_block": nnz,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs and outputs larger than L2 (4.3 GB written per step)"},
            "dofs_per_s": whole_job_rate(nd * a.steps, ms, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": alg_bytes * TRAFFIC_PER_ALG_BYTE,
                         "traffic_source": "ncu dram__bytes_read+write of one 48^3 launch "
                                           "(2030.9 MB for 2043.7 algorithmic MB), scaled "
                                           "by the algorithmic bytes",
                         "kernel": "k_tile_assemble<double>", "kernel_ms": k_ms,
                         "alg_bytes_per_launch": alg_bytes,
                         "step_alg_bytes": step_bytes,
                         "step_frac": step_bytes / (ms / a.steps / 1000.0) / 1e9 / peak},
            "h_applies_per_s": whole_job_rate(1, hs_mg[0], world),
            "latency_ms": {"p50": hs_mg[1], "p99": hs_mg[2],
                           "what": "one Hessian action (2 matrix-free FP64 solves, PCG with the "
                                   "lattice multigrid V-cycle, rtol 1e-12)"},
            "pcg_iterations": iters_mg,
            "jacobi_fp64": {"h_applies_per_s": whole_job_rate(1, hs_j[0], world),
                            "latency_ms": {"p50": hs_j[1], "p99": hs_j[2]},
                            "pcg_iterations": iters,
                            "what": "the same action with Jacobi-PCG (FP64, rtol 1e-12)"},
            "mixed": {"h_applies_per_s": whole_job_rate(1, hs_32[0], world),
                      "latency_ms": {"p50": hs_32[1], "p99": hs_32[2]},
                      "rel_err_vs_fp64": mixed_err,
                      "speedup_vs_fp64_jacobi": hs_j[0] / hs_32[0],
                      "pcg_iterations": iters32,
                      "what": "Jacobi-PCG with the recurrence in FP32, reliable updates to the "
                              "FP64 true residual (delta 0.1), rtol 1e-12"},
            "multigrid": {"h_applies_per_s": whole_job_rate(1, hs_mg[0], world),
                          "latency_ms": {"p50": hs_mg[1], "p99": hs_mg[2]},
                          "rel_err_vs_jacobi": mg_err,
                          "speedup_vs_fp64_jacobi": hs_j[0] / hs_mg[0],
                          "pcg_iterations": iters_mg,
                          "what": "FP64 PCG preconditioned by the lattice multigrid V-cycle "
                                  "(Q2 -> Q1 -> coarser Q1, Chebyshev-Jacobi degree %d, the coarsest "
                                  "level solved exactly when it has at most 64 interior "
                                  "nodes), rtol 1e-12" % mg_degree},
            "multigrid_fp32_cycle": {
                "h_applies_per_s": whole_job_rate(1, hs_mg32[0], world),
                "latency_ms": {"p50": hs_mg32[1], "p99": hs_mg32[2]},
                "rel_err_vs_jacobi": mg32_err, "rel_err_vs_fp64_cycle": mg32_vs_mg,
                "speedup_vs_fp64_cycle": hs_mg[0] / hs_mg32[0],
                "speedup_vs_fp64_jacobi": hs_j[0] / hs_mg32[0],
                "pcg_iterations": iters_mg32,
                "what": "the same FP64 PCG (recurrence, inner products and stopping test in "
                        "FP64, rtol 1e-12) with the V-cycle run in FP32 on single-precision "
                        "copies of the level data"},
            "e2e": {"value": e2e_value, "unit": "elements/s",
                    "h2d_bytes_per_step": 3 * 8 * nd, "d2h_bytes_per_step": 8 * nd,
                    "steps": e_steps,
                    "what": "setLinearizationPoint + evalGradientParameter per step, fields "
                            "from pinned host memory and the gradient back; the copies on "
                            "two copy streams (one per direction) with two buffer sets "
                            "(step i+1's inputs and step i-1's result move during step i)"},
            "clocks": ck,
            "serving": serving,
            "gpu_launches": launches_per_step * a.steps,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _problem_at(n, sigma, dev, precision="fp64", preconditioner="jacobi", lines=False):
    """Mesh, space, problem, misfit (data from m_true, 1 % noise) and m of a config."""
    import torch

    import hippymfem_b200 as hm
    from hippymfem_b200.synthetic import interior_points, log_conductivity, vertical_lines

    mesh = hm.BoxMesh(n, device=dev)
    V = hm.Q2Space(mesh)
    bc = hm.DirichletBC(V)
    prob = hm.PDEVariationalProblem([V, V, V], f=1.0, bc=bc, check_finite=False,
                                    solver_tolerance=1e-12, matrix_free_solves=True,
                                    solver_precision=precision, preconditioner=preconditioner)
    coords = mesh.node_coords()
    m = torch.as_tensor(log_conductivity(coords, seed=0, sigma=sigma), device=dev)
    mt = torch.as_tensor(log_conductivity(coords, seed=1, sigma=sigma), device=dev)
    pts = vertical_lines(60, 64, seed=3) if lines else interior_points(4096, seed=2)
    ut = V.vector()
    prob.solveFwd(ut, [ut, mt, None])
    d = hm.observation_operator(mesh, pts) @ ut.cpu().numpy()
    noise = 0.01 * float(np.abs(d).max())
    d = d + noise * np.random.default_rng(5).standard_normal(d.shape)
    misfit = hm.PointwiseStateObservation(V, pts, data=d, noise_variance=noise ** 2)
    return mesh, V, bc, prob, misfit, m


def run_precision(a, n=128, nactions=20):
    """The precision configuration: 128^3, m of amplitude sigma = 1.  Every block and
    vector assembled with FP32 element contractions (FP64 CSR values) against the FP64
    kernels, and nactions Hessian actions whose solves run the FP32 recurrence with FP64
    reliable updates against FP64 solves; relative errors per block and per action."""
    import torch

    import hippymfem_b200 as hm
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    dev = torch.device("cuda", 0)
    mesh, V, bc, prob, misfit, m = _problem_at(n, 1.0, dev, preconditioner="mg")
    model = hm.Model(prob, None, misfit)
    u, p = V.vector(), V.vector()
    x = [u, m, p]
    model.solveFwd(u, x)
    model.solveAdj(p, x)
    pat = hm.LatticePattern(mesh)
    prob._pattern = pat
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    sp = stream_ptr()
    blocks = {}
    cwork = torch.empty(lib.hm_lattice_consistent_workspace_bytes(mesh.handle) // 8 + 1,
                        dtype=torch.float64, device=dev)
    for name in ("A", "C", "Wum", "Wmm"):
        vals, ms = {}, {}
        for prec in (_lib.HM_FP64, _lib.HM_FP32):
            quad = torch.empty(mesh.quad_bytes(prec) // 8 + 1, dtype=torch.float64, device=dev)
            v = pat.new_values()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            check(lib.hm_lattice_quadrature(mesh.handle, ptr(u), ptr(m), ptr(p), prec, ptr(quad),
                                            ptr(status), sp))
            check(lib.hm_lattice_assemble(
                mesh.handle, ptr(quad), prec, ptr(pat.indptr), ptr(bc.marker), 1.0,
                *(ptr(v) if name == b else None for b in ("A", "C", "Wum", "Wmm")),
                None, None, None, 0, sp))
            e1.record()
            torch.cuda.synchronize()
            vals[prec], ms[prec] = v, e0.elapsed_time(e1)
            if prec == _lib.HM_FP64:
                # the constant-exact single-precision block (consistent_block) from the
                # same FP64 pointwise data
                c = pat.new_values()
                e0.record()
                check(lib.hm_lattice_assemble_consistent(
                    mesh.handle, ptr(quad), ptr(bc.marker),
                    *(ptr(c) if name == b else None for b in ("A", "C", "Wum", "Wmm")),
                    ptr(cwork), sp), "hm_lattice_assemble_consistent")
                e1.record()
                torch.cuda.synchronize()
                vals["consistent"], ms["consistent"] = c, e0.elapsed_time(e1)
            del quad
        ref = vals[_lib.HM_FP64]
        # products with the constants (row sums): what the consistent correction fixes
        ones = torch.ones(mesh.ndof, dtype=torch.float64, device=dev)
        rows = {}
        for key in (_lib.HM_FP64, _lib.HM_FP32, "consistent"):
            rows[key] = V.vector()
            hm.CSRBlock(pat, vals[key]).mult(ones, rows[key])
        scale = float(ref.abs().max())
        row_defect_fp32 = float((rows[_lib.HM_FP32] - rows[_lib.HM_FP64]).abs().max()) / scale
        row_defect_cons = float((rows["consistent"] - rows[_lib.HM_FP64]).abs().max()) / scale
        del rows, ones
        d = vals[_lib.HM_FP32] - ref
        dc = vals["consistent"] - ref
        blocks[name] = {"rel_err_max": float(d.abs().max() / ref.abs().max()),
                        "rel_err_fro": float(d.norm() / ref.norm()),
                        "consistent_rel_err_max": float(dc.abs().max() / ref.abs().max()),
                        "consistent_rel_err_fro": float(dc.norm() / ref.norm()),
                        "row_sum_defect_fp32": row_defect_fp32,
                        "row_sum_defect_consistent": row_defect_cons,
                        "ms_fp64": ms[_lib.HM_FP64], "ms_fp32": ms[_lib.HM_FP32],
                        "ms_consistent": ms["consistent"]}
        del vals, d, dc, ref
        torch.cuda.empty_cache()
    del cwork
    torch.cuda.empty_cache()
    # Hessian actions: FP64 (multigrid) against mixed-precision solves
    model.setPointForHessianEvaluations(x)
    H64 = hm.ReducedHessian(model)
    prob32 = hm.PDEVariationalProblem([V, V, V], f=1.0, bc=bc, check_finite=False,
                                      solver_tolerance=1e-12, solver_precision="mixed")
    prob32._pattern = pat
    model32 = hm.Model(prob32, None, misfit)
    model32.setPointForHessianEvaluations(x)
    H32 = hm.ReducedHessian(model32)
    rng = np.random.default_rng(21)
    errs, t64, t32 = [], [], []
    y64, y32 = V.vector(), V.vector()
    for i in range(nactions):
        v = torch.as_tensor(rng.standard_normal(mesh.ndof), device=dev)
        for H, y, t in ((H64, y64, t64), (H32, y32, t32)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            H.mult(v, y)
            e1.record()
            torch.cuda.synchronize()
            t.append(e0.elapsed_time(e1))
        errs.append(float((y32 - y64).norm() / y64.norm()))
    line = {"config": {"workload": "precision: Q2 hex %d^3, sigma = 1" % n, "dofs": mesh.ndof,
                       "nnz_per_block": mesh.nnz},
            "blocks_fp32_vs_fp64": blocks,
            "hessian_actions": {"n": nactions, "rel_err_mixed_vs_fp64": errs,
                                "rel_err_max": max(errs),
                                "ms_fp64_multigrid": float(np.mean(t64)),
                                "ms_mixed_jacobi": float(np.mean(t32)),
                                "pcg_iterations_mixed": H32.iterations[:4],
                                "pcg_iterations_fp64": H64.iterations[:4]},
            "data": "synthetic"}
    print(json.dumps(line), flush=True)


def run_differentiation(a, n=32, ndir=16, h=1e-6):
    """The differentiation configuration: 32^3, 60 vertical lines x 64 depths, 1 % noise;
    the gradient of the misfit by the autograd wrappers against central differences
    along ndir seeded directions, and the Hessian action (the gradient's
    vector-Jacobian product) against differences of the gradient."""
    import torch

    import hippymfem_b200 as hm
    from hippymfem_b200.autograd import ReducedGradient, reduced_misfit

    dev = torch.device("cuda", 0)
    mesh, V, bc, prob, misfit, m = _problem_at(n, 0.1, dev, preconditioner="mg", lines=True)
    model = hm.Model(prob, None, misfit)
    mm = m.clone().requires_grad_(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    J = reduced_misfit(mm, prob, misfit)
    (g,) = torch.autograd.grad(J, mm)
    e1.record()
    torch.cuda.synchronize()
    t_grad = e0.elapsed_time(e1)
    rng = np.random.default_rng(6)
    rel = []
    for _ in range(ndir):
        d = torch.as_tensor(rng.standard_normal(mesh.ndof), device=dev)
        with torch.no_grad():
            fd = float((reduced_misfit(m + h * d, prob, misfit) - reduced_misfit(m - h * d, prob, misfit))
                       / (2 * h))
        an = float(torch.dot(g, d))
        rel.append(abs(fd - an) / abs(an))
    mh = m.clone().requires_grad_(True)
    gg = ReducedGradient.apply(mh, model)
    hrel = []
    t_hv = []
    for _ in range(4):
        v = torch.as_tensor(rng.standard_normal(mesh.ndof), device=dev)
        e0.record()
        (hv,) = torch.autograd.grad(gg, mh, v, retain_graph=True)
        e1.record()
        torch.cuda.synchronize()
        t_hv.append(e0.elapsed_time(e1))
        with torch.no_grad():
            fd = (ReducedGradient.apply(m + h * v, model) - ReducedGradient.apply(m - h * v, model)) / (2 * h)
        hrel.append(float((fd - hv).norm() / hv.norm()))
    line = {"config": {"workload": "differentiation: Q2 hex %d^3, 60 lines x 64 depths" % n,
                       "dofs": mesh.ndof},
            "gradient_fd": {"directions": ndir, "h": h, "rel_err_max": max(rel),
                            "rel_err": rel, "ms_gradient": t_grad},
            "hessian_fd": {"directions": 4, "rel_err_max": max(hrel), "rel_err": hrel,
                           "ms_hessian_vector": float(np.mean(t_hv))},
            "data": "synthetic"}
    print(json.dumps(line), flush=True)


def run_solve(a):
    """One incremental solve A x = b at n^3 (the matrix-free FP64 Jacobian at the
    benchmark field, multigrid-PCG to rtol 1e-12, graph-replayed in a side stream, the
    V-cycle in --mg-precision), warm-up then --steps timed solves with CUDA events."""
    import torch

    from hippymfem_b200 import BoxMesh, DirichletBC, PDEVariationalProblem, Q2Space
    from hippymfem_b200.sparse import MGPCGSolver
    from hippymfem_b200.synthetic import log_conductivity

    mesh = BoxMesh(a.n)
    V = Q2Space(mesh)
    prob = PDEVariationalProblem([V, V, V], f=1.0, bc=DirichletBC(V), solver_tolerance=1e-12,
                                 matrix_free_solves=True)
    m = V.project(lambda x: log_conductivity(x, seed=0, sigma=0.1))
    A, _ = prob._jacobian([None, m, None])
    b = torch.as_tensor(np.random.default_rng(1).standard_normal(mesh.ndof),
                        device=mesh.device).masked_fill_(prob.bc0.mask, 0.0)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        solver = MGPCGSolver(A, rel_tolerance=1e-12, mg_precision=a.mg_precision)
        x = V.vector()
        for _ in range(max(a.warmup, 1)):
            solver.solve(x, b)
        s.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(a.steps):
            solver.solve(x, b)
        e1.record(s)
        s.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    line = {"metric": "incremental solves/s (FP64 multigrid-PCG, rtol 1e-12)",
            "value": 1e3 / ms, "unit": "solves/s", "ms_per_solve": ms,
            "iterations": solver.last.iterations, "relres": solver.last.relres,
            "mg_precision": solver.mg.precision, "fallbacks": solver.fallbacks,
            "steps": a.steps, "warmup": a.warmup,
            "config": {"workload": "Q2 hex %d^3 Jacobian solve at the benchmark field" % a.n,
                       "dofs": mesh.ndof},
            "data": "synthetic"}
    print(json.dumps(line), flush=True)


def run_shard(a):
    """The sharded Hessian action (``shard.ShardedHessian`` with the CUDA slab operators)
    at the benchmark's m on the 64^3 lattice, seeded u and p, 4096 observations, split
    into z-slabs, one per rank; every
    operator of the action is an assembly on the rank's slab after one halo exchange of
    its input, every inner product a plane-ordered sum of all ranks' plane partials, so
    the action is bit for bit the same on any number of ranks.  Timed like the main line
    (CUDA events, barrier on both sides, maximum over the ranks)."""
    import datetime

    import torch
    import torch.distributed as dist

    from hippymfem_b200 import synthetic
    from hippymfem_b200.shard import DeviceSlabOps, ShardedHessian, SlabPartition

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    n = (a.n, a.n, a.n)
    L = (1.0, 1.0, 1.0)
    part = SlabPartition(n, L, world)
    N = part.N
    nd = N[0] * N[1] * N[2]
    x = np.stack(np.meshgrid(*(np.linspace(0.0, Lv, Nv) for Lv, Nv in zip(L, N)),
                             indexing="ij"), -1).transpose(2, 1, 0, 3).reshape(-1, 3)
    m = synthetic.log_conductivity(x, seed=0)
    rng = np.random.default_rng(0)
    u, p, d = rng.standard_normal(nd), rng.standard_normal(nd), rng.standard_normal(nd)
    i = np.arange(nd)
    ix, iy, iz = i % N[0], (i // N[0]) % N[1], i // (N[0] * N[1])
    ess = ((ix == 0) | (ix == N[0] - 1) | (iy == 0) | (iy == N[1] - 1) | (iz == 0) |
           (iz == N[2] - 1)).astype(np.int32)
    k0, k1 = part.owned_planes(rank)
    own = [torch.as_tensor(v.reshape(N[2], -1)[k0:k1].copy(), device=dev)
           for v in (u, m, p, ess, d)]
    pts = synthetic.interior_points(4096, seed=2)
    ops = DeviceSlabOps(part, rank, pts, 1e-4, dev)
    H = ShardedHessian(part, rank, ops, *own[:4], rtol=1e-12)
    for _ in range(max(1, min(a.warmup, 2))):
        H.mult(own[4])
    k = max(1, min(a.steps, 3))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(k):
        H.mult(own[4])
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    (ms,) = max_over_ranks([e0.elapsed_time(e1)], world, dev)
    if rank == 0:
        print(json.dumps({
            "metric": "sharded Hessian action at %d^3 (z-slabs, Jacobi-PCG rtol 1e-12)" % a.n,
            "value": k / (ms / 1000.0), "unit": "H-applies/s", "n_gpus": world, "steps": k,
            "warmup": max(1, min(a.warmup, 2)), "ms_per_step": ms / k,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "pcg_iterations": H.iterations[-2:],
            "config": {"workload": "TrueHessian action, 4096 pointwise observations, %d^3 Q2 "
                                   "split into %d z-slabs" % (a.n, world),
                       "parallelism": "z-slabs x%d" % world}}), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.shard and a.impl != "reference":
        run_shard(a)
        return
    if a.impl == "reference":
        run_reference(a)
    elif a.config == "precision":
        run_precision(a)
    elif a.config == "differentiation":
        run_differentiation(a)
    elif a.config == "solve":
        run_solve(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
