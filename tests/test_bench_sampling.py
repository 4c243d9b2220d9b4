"""The CPU baseline's sampling rule (bench.py): when the time budget ends
before K steps, the untimed steps are charged from timed steps after the
dam break's start-up transient, never from its capped solves, so the
sampled value errs on the CPU's side.  Plain arithmetic on made-up timings;
no oracle run."""
import numpy as np

import bench

CAP = 101
# the 1M dam break's reference iteration counts over its first steps
ITERS = [101, 101, 101, 101, 101, 92, 2, 2, 2, 6, 4, 2, 2, 2, 2]


def _times(iters, base=0.3, per_iter=0.03):
    return [base + per_iter * it for it in iters]


def test_settled_steps_counts_after_the_last_capped_solve():
    assert bench.settled_steps([], CAP) == 0
    assert bench.settled_steps([101, 101], CAP) == 0
    assert bench.settled_steps(ITERS, CAP) == len(ITERS) - 5
    assert bench.settled_steps([2, 3, 4], CAP) == 3


def test_charge_never_comes_from_capped_solves():
    iters = ITERS[:13]
    times = _times(iters)
    value, tail = bench.sampled_value(times, iters, 500, CAP)
    settled = times[5:]
    assert tail == settled                   # the 92-iteration step and after, no capped one
    assert max(tail) < min(times[:5])
    charge = float(np.median(settled))       # the median skips the 92-iteration step
    assert charge == _times([2])[0]
    assert np.isclose(value, 500 / (sum(times) + 487 * charge))


def test_all_steps_timed():
    times = _times(ITERS)
    value, _ = bench.sampled_value(times, ITERS, len(ITERS), CAP)
    assert np.isclose(value, len(ITERS) / sum(times))


def test_no_settled_step_charges_the_cheapest():
    iters = [101, 101, 101]
    times = _times(iters)
    value, tail = bench.sampled_value(times, iters, 10, CAP)
    assert tail == [min(times)]
    assert np.isclose(value, 10 / (sum(times) + 7 * min(times)))


def test_timing_goes_past_the_budget_until_five_settled_steps():
    budget = 10.0
    iters, times = [], []
    for it in ITERS:
        if not bench.keep_timing(times, iters, 500, budget, CAP):
            break
        iters.append(it)
        times.append(_times([it])[0])
    # the five capped solves alone spend the budget; timing stops once five
    # steps after them are in
    assert sum(times[:5]) > budget
    assert bench.settled_steps(iters, CAP) == 5
    assert len(iters) == 10


def test_timing_stops_at_three_budgets():
    budget = 1.0
    iters, times = [], []
    while bench.keep_timing(times, iters, 500, budget, CAP):
        iters.append(101)
        times.append(0.7)
    assert sum(times) >= 3 * budget
    assert sum(times) - 0.7 < 3 * budget


def test_timing_stops_at_k():
    iters, times = [], []
    while bench.keep_timing(times, iters, 4, 1e9, CAP):
        iters.append(2)
        times.append(0.1)
    assert len(times) == 4
