"""The request loop: each result is the same alone and in the mix; results agree with
the plain per-request FP64 path within the solve tolerance; admission keeps the
workspaces within the memory budget while requests overlap on the device.  GPU."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_SAME = 1e-14      # alone vs in the mix: deterministic kernels, same arithmetic
TOL_FWD = 1e-6        # served (mixed precision, rtol 1e-8) vs plain FP64 (rtol 1e-8)
TOL_HESS = 1e-5


def _trace():
    from hippymfem_b200.serving import Request

    kinds = ["forward", "hessian", "forward", "forward", "hessian", "forward"] * 3
    sizes = [8, 12, 16, 12, 8, 16, 16, 8, 12] * 2
    return [Request(k, n, 100 + i, 0.002 * i) for i, (k, n) in enumerate(zip(kinds, sizes))]


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_results_are_the_same_alone_and_in_the_mix(cuda):
    from hippymfem_b200.serving import Request, Server

    mixed = Server(slots=4, precision="mixed", check_every=16)
    reqs = mixed.run(_trace())
    # the requests did overlap on the device
    spans = sorted((r.t_admit, r.t_done) for r in reqs)
    assert any(b[0] < a[1] for a, b in zip(spans, spans[1:]))
    assert len({r.slot for r in reqs}) > 1
    alone = Server(slots=1, precision="mixed", check_every=16)
    for r in reqs:
        (a,) = alone.run([Request(r.kind, r.n, r.seed, 0.0)])
        assert _rel(r.result, a.result) <= TOL_SAME, (r.kind, r.n, _rel(r.result, a.result))
        assert r.iterations == a.iterations
    mixed.close()
    alone.close()


def test_served_results_match_the_plain_fp64_path(cuda):
    from hippymfem_b200.serving import Request, Server, plain_fp64

    reqs = [Request("forward", 12, 5), Request("hessian", 12, 6), Request("forward", 16, 7),
            Request("hessian", 8, 8)]
    srv = Server(slots=2, precision="mixed")
    srv.autotune([8, 12, 16], candidates=(8, 16), reps=1)
    srv.run(reqs)
    cache = {}
    for r in reqs:
        ref = plain_fp64(r, cache=cache).cpu().numpy()
        tol = TOL_FWD if r.kind == "forward" else TOL_HESS
        assert _rel(r.result, ref) <= tol, (r.kind, r.n, _rel(r.result, ref))
    srv.close()


def test_admission_keeps_workspaces_within_the_budget(cuda):
    from hippymfem_b200.serving import Request, Server

    probe = Server(slots=1, precision="fp64")
    need16 = probe.mesh_state(16).footprint("fp64")
    need12 = probe.mesh_state(12).footprint("fp64")
    budget = need16 + need12 + need12 // 2
    srv = Server(slots=3, precision="fp64", memory_budget=budget)
    reqs = [Request("forward" if i % 3 else "hessian", 16 if i % 2 else 12, 200 + i, 0.0)
            for i in range(12)]
    srv.run(reqs)
    assert all(r.result is not None for r in reqs)
    assert srv.peak_resident <= budget
    srv.close()


@pytest.mark.parametrize("multigrid", [True, False])
def test_grouped_solves_equal_each_request_alone(cuda, multigrid):
    """Same-size requests whose solves run as one group (SolveGroup: one CUDA graph per
    batch of iterations, a branch per request) give each request's result and iteration
    counts bit for bit as its solves alone; so does the server with groups."""
    import torch

    from hippymfem_b200.serving import Request, Server, _Workspace
    from hippymfem_b200.sparse import SolveGroup

    srv = Server(slots=1, precision="fp64", multigrid=multigrid, check_every=4, group_size=4)
    ms = srv.mesh_state(12)
    stream = torch.cuda.Stream()
    for kind in ("forward", "hessian"):
        wss = [_Workspace(ms, "fp64", 1e-8, 4, multigrid) for _ in range(3)]
        reqs = [Request(kind, 12, 700 + j) for j in range(3)]
        grp = SolveGroup([w.plan for w in wss])
        with torch.cuda.stream(stream):
            outs = [o.clone() for o in srv._run_group_with(wss, reqs, grp)]
            again = [o.clone() for o in srv._run_group_with(wss, reqs, grp)]   # graph replayed
        stream.synchronize()
        solo = _Workspace(ms, "fp64", 1e-8, 4, multigrid)
        for r, o, o2 in zip(reqs, outs, again):
            ra = Request(kind, 12, r.seed)
            with torch.cuda.stream(stream):
                a = srv._run_group_with([solo], [ra], None)[0].clone()
            stream.synchronize()
            assert torch.equal(o, a) and torch.equal(o2, a), (kind, r.seed)
            assert r.iterations[:len(ra.iterations)] == ra.iterations
        grp.close()
        for w in wss + [solo]:
            w.close()
    reqs = [Request("forward", 12, 800 + i, 0.0) for i in range(5)] + \
        [Request("hessian", 8, 900 + i, 0.0) for i in range(3)]
    srv.run(reqs)
    alone = Server(slots=1, precision="fp64", multigrid=multigrid, check_every=4)
    for r in reqs:
        (a,) = alone.run([Request(r.kind, r.n, r.seed, 0.0)])
        assert np.array_equal(r.result, a.result) and r.iterations == a.iterations
    srv.close()
    alone.close()
