"""bench.py's step accounting on the host, with a fake case in place of the
library: every outer iteration that fails the reference's divergence test
(simpleSolver.cpp:360-364: non-finite continuity, pressure step or fields,
carried by SimpleResult.diverged) or whose continuity error has grown 100x
past the first warm-up step's is counted, so a blown-up trajectory cannot be
reported as throughput; and the per-field errors the JSON line carries."""
import importlib.util
import math
import os
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture()
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.Steps.ref = None
    yield mod
    mod.Steps.ref = None


class FakeCase:
    """Hands out one result per solve from a list of (continuity, diverged)."""

    def __init__(self, trajectory, ms=2.0, launches=5):
        self.trajectory = list(trajectory)
        self.ms, self.launches = ms, launches

    def solve(self, ctl):
        c, div = self.trajectory.pop(0)
        return SimpleNamespace(final_continuity_error=c, diverged=div, u_inner_iterations=30, p_inner_iterations=10)

    def last_timing(self):
        # slot 7 is the whole outer iteration's device time
        return [0.0] * 7 + [self.ms], self.launches


def test_bounded_trajectory_counts_no_divergence(bench):
    case = FakeCase([(0.06, False), (0.034, False), (0.033, False), (0.032, False)])
    warm = bench.Steps().run(case, None, 1)
    timed = bench.Steps().run(case, None, 3)
    assert bench.Steps.ref == 0.06
    assert warm.diverged == 0 and timed.diverged == 0
    assert timed.ms == pytest.approx(6.0) and timed.launches == 15
    assert timed.u == 90 and timed.p == 30
    assert timed.cont == [0.034, 0.033, 0.032]


def test_reference_flag_non_finite_and_growth_each_count(bench):
    case = FakeCase([(0.05, False),     # warm-up: the growth test's reference
                     (0.04, True),      # the reference's own divergence flag
                     (math.nan, False),  # non-finite continuity
                     (math.inf, False),
                     (5.1, False),      # 102x the reference: a blow-up still finite
                     (4.9, False)])     # 98x: not yet
    bench.Steps().run(case, None, 1)
    timed = bench.Steps().run(case, None, 5)
    assert timed.diverged == 4


def test_growth_reference_is_the_first_finite_step(bench):
    # a non-finite first warm-up step is itself diverged and does not become
    # the growth test's reference
    case = FakeCase([(math.nan, False), (1e-3, False), (0.2, False)])
    s = bench.Steps().run(case, None, 3)
    assert bench.Steps.ref == 1e-3
    assert s.diverged == 2


def test_field_errors_and_mean_free_pressure(bench):
    rng = np.random.default_rng(3)
    U0, p0, phi0 = rng.normal(size=(50, 3)), rng.normal(size=50), rng.normal(size=140)
    e = bench.field_errors(U0 * (1 + 1e-9), p0 + 7.0, phi0, U0, p0, phi0, mean_free=True)
    assert e["U"] == pytest.approx(1e-9, rel=1e-3)
    assert e["p"] < 1e-14  # a constant shift is no error when no cell pins p
    assert e["phi"] == 0.0
    e = bench.field_errors(U0, p0 + 7.0, phi0, U0, p0, phi0)
    assert e["p"] > 1.0
    assert bench.rel_l2(np.ones(3), np.zeros(3)) == pytest.approx(math.sqrt(3))
