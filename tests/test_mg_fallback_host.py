"""``MGPCGSolver.solve``'s choice between the FP32 and the FP64 V-cycle, with the device
calls replaced by stand-ins: a stalled FP32-cycle solve, or one whose true residual ends
above ten times the tolerance, is solved again with the FP64 cycle, which the solver
keeps; a carried solve is kept as it is; FP64 solves are never checked.  CPU."""

import pytest
import torch

from hippymfem_b200 import _lib
from hippymfem_b200.sparse import MGPCGSolver, PCGResult


class _FakeMG:
    def __init__(self, precision):
        self.precision = precision
        self.work32 = object()

    def set_precision(self, precision, stream=None):
        self.precision = precision
        return self


def _solver(precision, outcomes, carried, raise_on_fail=True):
    """A solver whose plan solves return ``outcomes`` in turn (the FP32-cycle ones while
    the cycle is FP32) and whose true-residual check returns ``carried``."""
    s = object.__new__(MGPCGSolver)
    s.parameters = {"rel_tolerance": 1e-12, "max_iter": 100, "check_every": 4}
    s.raise_on_fail = raise_on_fail
    s.mg = _FakeMG(precision)
    s.b = torch.zeros(5, dtype=torch.float64)
    s.x = torch.zeros(5, dtype=torch.float64)
    s._plan = None
    s._y = None
    s.fallbacks = 0
    s.last = None
    log = {"runs": [], "plans": 0, "checks": 0}

    def run(stream):
        rc, value = outcomes.pop(0)
        log["runs"].append(s.mg.precision)
        s.x.fill_(value)
        s.last = PCGResult(7, 1e-13, rc == _lib.HM_OK)
        return rc

    def make_plan():
        log["plans"] += 1

    def check_carried(stream):
        log["checks"] += 1
        return carried

    s._run, s._make_plan, s._carried = run, make_plan, check_carried
    return s, log


def test_carried_fp32_cycle_solve_is_kept():
    s, log = _solver("fp32", [(_lib.HM_OK, 1.0)], carried=True)
    x = torch.zeros(5, dtype=torch.float64)
    s.solve(x, torch.ones(5, dtype=torch.float64))
    assert log == {"runs": ["fp32"], "plans": 0, "checks": 1}
    assert s.fallbacks == 0 and s.mg.precision == "fp32" and float(x[0]) == 1.0


def test_stalled_fp32_cycle_solve_is_solved_again_in_fp64():
    outcomes = [(_lib.HM_ERR_NOCONV, 1.0), (_lib.HM_OK, 2.0)]
    s, log = _solver("fp32", outcomes, carried=True)
    x = torch.zeros(5, dtype=torch.float64)
    s.solve(x, torch.ones(5, dtype=torch.float64))
    assert log == {"runs": ["fp32", "fp64"], "plans": 1, "checks": 0}
    assert s.fallbacks == 1 and s.mg.precision == "fp64" and s.mg.work32 is None
    assert float(x[0]) == 2.0
    # the solver keeps the FP64 cycle: the next solve is neither checked nor redone
    outcomes.append((_lib.HM_OK, 3.0))
    s.solve(x, torch.ones(5, dtype=torch.float64))
    assert log == {"runs": ["fp32", "fp64", "fp64"], "plans": 1, "checks": 0}
    assert s.fallbacks == 1 and float(x[0]) == 3.0


def test_drifted_fp32_cycle_solve_is_solved_again_in_fp64():
    s, log = _solver("fp32", [(_lib.HM_OK, 1.0), (_lib.HM_OK, 2.0)], carried=False)
    x = torch.zeros(5, dtype=torch.float64)
    s.solve(x, torch.ones(5, dtype=torch.float64))
    assert log == {"runs": ["fp32", "fp64"], "plans": 1, "checks": 1}
    assert s.fallbacks == 1 and float(x[0]) == 2.0


def test_fp64_cycle_solves_are_not_checked():
    s, log = _solver("fp64", [(_lib.HM_OK, 4.0)], carried=False)
    x = torch.zeros(5, dtype=torch.float64)
    s.solve(x, torch.ones(5, dtype=torch.float64))
    assert log == {"runs": ["fp64"], "plans": 0, "checks": 0} and s.fallbacks == 0


def test_fallback_that_does_not_converge_raises_or_returns_its_iterate():
    s, log = _solver("fp32", [(_lib.HM_ERR_NOCONV, 1.0), (_lib.HM_ERR_NOCONV, 5.0)], carried=True)
    with pytest.raises(_lib.NotConvergedError):
        s.solve(torch.zeros(5, dtype=torch.float64), torch.ones(5, dtype=torch.float64))
    s, log = _solver("fp32", [(_lib.HM_ERR_NOCONV, 1.0), (_lib.HM_ERR_NOCONV, 5.0)], carried=True,
                     raise_on_fail=False)
    x = torch.zeros(5, dtype=torch.float64)
    s.solve(x, torch.ones(5, dtype=torch.float64))
    assert float(x[0]) == 5.0 and not s.last.converged and s.fallbacks == 1
