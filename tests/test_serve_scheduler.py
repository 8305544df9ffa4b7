"""The serving loop's scheduler on a simulated device (no GPU): first-come-first-served
admission under the HBM budget, continuous batching of arrivals into the next launch,
the in-flight limit, and the latency summary; plus the host-only workspace query that
the admission estimate uses."""
import math

import numpy as np
import pytest

from particleclem_b200 import abi, hydro
from particleclem_b200.serve import BudgetError, Request, Scheduler, poisson_arrivals, summarize


class SimExecutor:
    """A device that runs one batch at a time: overhead + cost per cell."""

    def __init__(self, overhead=1e-4, per_cell=1e-9):
        self.t = 0.0
        self.overhead, self.per_cell = overhead, per_cell
        self.busy_until = 0.0
        self.finishes = []
        self.batches = []
        self.evicted = []

    def evict(self, pid):
        self.evicted.append(pid)

    def now(self):
        return self.t

    def launch(self, batch, slot=0):
        start = max(self.t, self.busy_until)
        fin = start + self.overhead + self.per_cell * sum(r.cells for r in batch)
        self.busy_until = fin
        self.finishes.append(fin)
        self.batches.append([r.rid for r in batch])
        return fin

    def done(self, h):
        return self.t >= h

    def finish_time(self, h):
        return h

    def idle(self, next_arrival, busy):
        cands = [f for f in self.finishes if f > self.t]
        if next_arrival is not None and next_arrival > self.t:
            cands.append(next_arrival)
        self.t = min(cands) if cands else self.t + 1e-9


def _requests(n, seed, rate, max_bytes=100):
    rng = np.random.default_rng(seed)
    arr = poisson_arrivals(n, rate, seed)
    return [Request(k, k, float(a), int(rng.integers(1000, 300000)), int(rng.integers(1, max_bytes)))
            for k, a in enumerate(arr)]


@pytest.mark.parametrize("rate", [100.0, 2000.0, math.inf])
def test_budget_fifo_and_completion(rate):
    reqs = _requests(200, 1, rate)
    budget = 400
    ex = SimExecutor()
    sch = Scheduler(ex, budget, max_inflight=2)
    sch.run(reqs)
    assert sch.peak_bytes <= budget
    for r in reqs:
        assert r.arrival <= r.start <= r.finish
    # first come first served: batches never reorder arrivals
    order = sorted(reqs, key=lambda r: (r.arrival, r.rid))
    assert [r.batch for r in order] == sorted(r.batch for r in order)
    # a batch never launches before the one two places ahead of it has completed
    fin = {r.batch: r.finish for r in reqs}
    for r in reqs:
        if r.batch >= 2:
            assert r.start >= fin[r.batch - 2]


def test_arrivals_during_a_batch_join_the_next_one():
    # batches take ~10 ms, requests arrive every 1 ms: each launch after the first two
    # carries the arrivals of the previous batch's run time
    reqs = [Request(k, k, 1e-3 * k, cells=10_000_000, nbytes=1) for k in range(60)]
    ex = SimExecutor(overhead=0.0, per_cell=1e-9)
    sch = Scheduler(ex, budget_bytes=10**9, max_inflight=1)
    sch.run(reqs)
    sizes = [len(b) for b in ex.batches]
    assert sizes[0] == 1 and max(sizes) > 5 and sch.nbatches < len(reqs) // 3
    assert sum(sizes) == len(reqs)


def test_inflight_limit_and_max_batch():
    reqs = [Request(k, k, 0.0, cells=1000, nbytes=1) for k in range(10)]
    ex = SimExecutor()
    sch = Scheduler(ex, budget_bytes=100, max_inflight=2, max_batch=3)
    sch.run(reqs)
    assert [len(b) for b in ex.batches] == [3, 3, 3, 1]


def test_saturated_run_is_one_batch_under_a_large_budget():
    reqs = [Request(k, k, 0.0, cells=1000, nbytes=10) for k in range(50)]
    sch = Scheduler(SimExecutor(), budget_bytes=10**6)
    sch.run(reqs)
    assert sch.nbatches == 1


def test_request_larger_than_budget_is_refused():
    with pytest.raises(BudgetError):
        Scheduler(SimExecutor(), budget_bytes=10).run([Request(0, 0, 0.0, cells=1, nbytes=11)])


def test_summary_percentiles():
    reqs = [Request(k, k, 0.0, cells=100, nbytes=1, finish=(k + 1) * 1e-3, batch=k) for k in range(100)]
    s = summarize(reqs)
    assert s["p50_ms"] == pytest.approx(50.5) and s["p99_ms"] == pytest.approx(99.01)
    assert s["cell_updates_per_s"] == pytest.approx(100 * 100 / 0.1)


def test_workspace_query_is_host_only_and_additive():
    """The query answers without a device, and the bytes of two boxes together are the
    sum of their bytes alone up to the size classes the allocation is rounded to (from
    1 MiB on at most 25 % above the exact size)."""
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        prm = abi.make_params((1, 1, 1), 0.0, 9, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0), precision_mode=prec)
        a = hydro.workspace_bytes(prm, [((0, 0, 0), (31, 31, 31))])
        b = hydro.workspace_bytes(prm, [((0, 0, 0), (15, 23, 7))])
        ab = hydro.workspace_bytes(prm, [((0, 0, 0), (31, 31, 31)), ((0, 0, 0), (15, 23, 7))])
        assert 0 < b < a and 0.8 * (a + b) <= ab <= 1.25 * (a + b)
        # at least the traced states: 2 x 3 directions x (6+NS) values per cell of grow(box,1)
        assert a >= 6 * 15 * 34 ** 3 * (4 if prec == abi.PREC_MIXED else 8)
    m = hydro.workspace_bytes(abi.make_params((1, 1, 1), 0.0, 9, (0,) * 3, (0,) * 3, (0,) * 3, (0,) * 3,
                                              precision_mode=abi.PREC_MIXED), [((0, 0, 0), (31, 31, 31))])
    d = hydro.workspace_bytes(abi.make_params((1, 1, 1), 0.0, 9, (0,) * 3, (0,) * 3, (0,) * 3, (0,) * 3,
                                              precision_mode=abi.PREC_FP64), [((0, 0, 0), (31, 31, 31))])
    assert m < d


def test_steps_of_one_patch_stay_in_order():
    """Two requests for the same patch never share a batch and the second starts after
    the first has finished (each step reads the state the previous one wrote)."""
    reqs = [Request(0, 7, 0.0, cells=1000, nbytes=1), Request(1, 3, 0.0, cells=1000, nbytes=1),
            Request(2, 7, 0.0, cells=1000, nbytes=1)]
    sch = Scheduler(SimExecutor(), budget_bytes=100, max_inflight=2)
    sch.run(reqs)
    assert reqs[0].batch != reqs[2].batch
    assert reqs[2].start >= reqs[0].finish


def test_resident_states_are_evicted_least_recently_used_within_the_budget():
    """Four patches whose states take 40 bytes each (workspace 10) under a budget of 100:
    at most two states fit beside a step's workspace, so idle states are evicted, least
    recently used first, and the budget holds throughout."""
    ex = SimExecutor()
    pids = [0, 1, 2, 3, 0, 1, 2, 3]
    reqs = [Request(k, p, 1e-3 * k, cells=1000, nbytes=10, state_bytes=40) for k, p in enumerate(pids)]
    sch = Scheduler(ex, budget_bytes=100, max_inflight=1)
    sch.run(reqs)
    assert sch.peak_bytes <= 100
    assert ex.evicted[:2] == [0, 1]  # patch 2 evicts 0, patch 3 evicts 1
    assert sch.evictions == len(ex.evicted) and sch.uploads == 4 + sch.evictions - (4 - len(sch.resident))


def test_max_batch_cells():
    reqs = [Request(k, k, 0.0, cells=1000, nbytes=1) for k in range(10)]
    ex = SimExecutor()
    Scheduler(ex, budget_bytes=100, max_inflight=2, max_batch_cells=2500).run(reqs)
    assert [len(b) for b in ex.batches] == [2, 2, 2, 2, 2]
