"""The serving loop's host logic without a GPU: admission of a slot's workspace under the
memory budget, least-recently-used eviction of idle workspaces, waiting while every
resident workspace is busy, the error for a workspace larger than the budget, and the
trace / latency helpers.  The workspaces here are stand-ins with a size.  CPU only."""

import threading
import time

import numpy as np
import pytest


class _FakeMesh:
    def __init__(self, nbytes):
        self.nbytes = nbytes

    def footprint(self, precision, multigrid=False):
        return self.nbytes


class _FakeWorkspace:
    def __init__(self, nbytes, last_used=0.0):
        self.nbytes = nbytes
        self.in_use = False
        self.last_used = last_used
        self.closed = False

    def close(self):
        self.closed = True


def _server(budget, sizes):
    """A Server with only its admission state (no device, no streams)."""
    from hippymfem_b200.serving import Server

    s = Server.__new__(Server)
    s.budget = budget
    s.precision = "mixed"
    s.multigrid = False
    s.meshes = {n: _FakeMesh(b) for n, b in sizes.items()}
    s._ws = {}
    s._groups = {}
    s._resident = 0
    s.peak_resident = 0
    s._lock = threading.Condition()
    return s


def _admit(s, slot, n, j=0, block=True):
    """As the worker does: reserve, then register a new workspace of the reserved size
    (the slot's j-th for size n: the members of a same-size group)."""
    with s._lock:
        ws, reserved, ok = s._acquire(slot, n, j, block=block)
        if not ok:
            return None, None
        if ws is None:
            ws = _FakeWorkspace(reserved)
            ws.in_use = True
            s._ws[(slot, n, j)] = ws
    return ws, reserved


def _release(s, ws, t):
    with s._lock:
        ws.in_use = False
        ws.last_used = t
        s._lock.notify_all()


def test_reuse_and_reservation():
    s = _server(100, {8: 30, 16: 50})
    a, r = _admit(s, 0, 8)
    assert r == 30 and s._resident == 30
    _release(s, a, 1.0)
    b, r = _admit(s, 0, 8)                     # the same slot and size: the resident one
    assert b is a and r is None and a.in_use and s._resident == 30
    _admit(s, 1, 16)
    assert s._resident == 80 and s.peak_resident == 80


def test_idle_workspaces_are_evicted_least_recently_used_first():
    s = _server(100, {8: 30, 12: 30, 16: 30, 24: 60})
    w8, _ = _admit(s, 0, 8)
    w12, _ = _admit(s, 1, 12)
    w16, _ = _admit(s, 2, 16)
    _release(s, w12, 1.0)                      # idle longest
    _release(s, w8, 2.0)
    _release(s, w16, 3.0)                      # most recent
    _admit(s, 3, 24)                           # needs 60 of 100 with 90 resident: two go
    assert w12.closed and w8.closed and not w16.closed
    assert set(s._ws) == {(2, 16, 0), (3, 24, 0)}
    assert s._resident == 90


def test_admission_waits_for_a_busy_workspace():
    s = _server(60, {8: 40, 16: 40})
    w8, _ = _admit(s, 0, 8)                    # in use: nothing can be evicted
    got = {}

    def second():
        got["ws"] = _admit(s, 1, 16)

    t = threading.Thread(target=second, daemon=True)
    t.start()
    time.sleep(0.2)
    assert t.is_alive() and "ws" not in got    # blocked on the budget
    _release(s, w8, 5.0)                       # idle now: the waiter evicts it
    t.join(timeout=10)
    assert not t.is_alive()
    assert w8.closed and got["ws"][1] == 40 and s._resident == 40


def test_a_workspace_beyond_the_budget_raises():
    s = _server(10, {48: 11})
    with pytest.raises(MemoryError, match="more than the budget"):
        _admit(s, 0, 48)


def test_poisson_trace_and_latency_stats():
    from hippymfem_b200.serving import Request, latency_stats, poisson_trace

    tr = poisson_trace(2000, rate=100.0, seed=3)
    t = np.array([r.arrival for r in tr])
    assert len(tr) == 2000 and np.all(np.diff(t) > 0)
    assert 15.0 < t[-1] < 25.0                 # 2000 arrivals at 100/s
    frac = np.mean([r.kind == "forward" for r in tr])
    assert 0.66 < frac < 0.74
    assert {r.n for r in tr} == {8, 12, 16, 24, 32, 48}
    assert [r.arrival for r in poisson_trace(50, 10.0, seed=3)] == \
        [r.arrival for r in poisson_trace(50, 10.0, seed=3)]
    reqs = []
    for i in range(100):
        r = Request("forward", 8, i, arrival=0.01 * i)
        r.t_admit = r.arrival
        r.t_done = r.arrival + 0.001 * (i + 1)
        reqs.append(r)
    st = latency_stats(reqs)
    assert st["n"] == 100
    assert st["p50_ms"] == pytest.approx(50.5, rel=1e-9)
    assert st["requests_per_s"] == pytest.approx(100 / (0.99 + 0.1))


def test_group_members_take_room_only_when_there_is_some():
    """A group's further workspaces never wait for room: without it the member request
    goes back to the queue; with it, each member has its own workspace."""
    s = _server(100, {8: 40})
    a, _ = _admit(s, 0, 8, 0)
    b, _ = _admit(s, 0, 8, 1, block=False)
    assert b is not None and b is not a and s._resident == 80
    c, _ = _admit(s, 0, 8, 2, block=False)       # 120 > 100, nothing idle
    assert c is None and s._resident == 80
    _release(s, b, 1.0)
    c, _ = _admit(s, 0, 8, 2, block=False)       # the idle member makes room
    assert c is not None and b.closed and s._resident == 80
