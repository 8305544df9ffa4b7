"""Continuous-batching serving loop for patch advances.

A request asks for the hydro source of one resident patch over one step, i.e. one box
iteration of PeleC::construct_hydro_source (Source/Hydro.cpp:70-288) with the patch's
own CFL timestep. Requests arrive over time (an ensemble of runs submitting boxes); the
scheduler admits them first come first served while the device bytes they hold stay
within an HBM budget, and every round launches all admitted requests that are not yet
running as ONE batched call (pcg_hydro_boxes: one launch per stage over uneven boxes),
with at most ``max_inflight`` batches queued on the device so that arrivals during a
batch join the next one. Latency is arrival to device completion of the request's batch.

The scheduler is independent of the device: an executor launches batches, reports
their completion and keeps the clock. GpuExecutor runs them through the library;
tests drive the scheduler with a simulated executor.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass

import numpy as np

from . import abi, hydro


@dataclass
class Request:
    rid: int
    pid: int  # resident patch whose hydro source is requested
    arrival: float  # seconds since the start of the run
    cells: int = 0
    nbytes: int = 0  # device bytes held from launch to completion
    start: float = math.nan  # time the request's batch was launched
    finish: float = math.nan  # device completion time of its batch
    batch: int = -1  # index of the batch it ran in

    @property
    def latency(self):
        return self.finish - self.arrival


class BudgetError(ValueError):
    pass


class Scheduler:
    def __init__(self, executor, budget_bytes, max_inflight=2, max_batch=None):
        self.ex = executor
        self.budget = int(budget_bytes)
        self.max_inflight = int(max_inflight)
        self.max_batch = max_batch
        self.peak_bytes = 0
        self.nbatches = 0

    def run(self, requests):
        """Serve ``requests`` (arrival times relative to the executor's start) to
        completion; fills start/finish/batch in place and returns them."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in reqs:
            if r.nbytes > self.budget:
                raise BudgetError(f"request {r.rid} needs {r.nbytes} bytes, budget {self.budget}")
        ex = self.ex
        i, n = 0, len(reqs)
        waiting, inflight = deque(), deque()
        used = 0
        while i < n or waiting or inflight:
            now = ex.now()
            while i < n and reqs[i].arrival <= now:
                waiting.append(reqs[i])
                i += 1
            progressed = False
            while inflight and ex.done(inflight[0][0]):
                h, batch = inflight.popleft()
                t = ex.finish_time(h)
                for r in batch:
                    r.finish = t
                    used -= r.nbytes
                progressed = True
            if waiting and len(inflight) < self.max_inflight:
                batch = []
                while waiting and used + waiting[0].nbytes <= self.budget and (
                        self.max_batch is None or len(batch) < self.max_batch):
                    r = waiting.popleft()
                    used += r.nbytes
                    r.start = now
                    r.batch = self.nbatches
                    batch.append(r)
                if batch:
                    self.peak_bytes = max(self.peak_bytes, used)
                    inflight.append((ex.launch(batch), batch))
                    self.nbatches += 1
                    progressed = True
            if not progressed:
                nxt = reqs[i].arrival if i < n else None
                ex.idle(nxt, bool(inflight))
        return reqs


def summarize(reqs):
    lat = np.array([r.latency for r in reqs]) * 1e3
    t0 = min(r.arrival for r in reqs)
    t1 = max(r.finish for r in reqs)
    cells = sum(r.cells for r in reqs)
    return {"requests": len(reqs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max()), "makespan_s": t1 - t0,
            "cell_updates_per_s": cells / (t1 - t0) if t1 > t0 else math.nan,
            "batches": len({r.batch for r in reqs})}


def poisson_arrivals(n, rate, seed):
    """n arrival times of a Poisson process of ``rate`` per second (rate inf: all at 0)."""
    if math.isinf(rate):
        return np.zeros(n)
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


class GpuExecutor:
    """Executes batches with pcg_hydro_boxes on one stream. Patches are uploaded once
    (resident); each gets its CFL timestep (estTimeStep of the patch) and a device
    output for its hydro source."""

    def __init__(self, eos, precision=abi.PREC_MIXED, cfl=0.3, device=0, poll_s=20e-6):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        hydro.init(device)
        hydro.set_eos(eos)
        self.ns = eos.nspec
        self.nv = abi.nvar(self.ns)
        self.cfl = float(cfl)
        self.poll_s = poll_s
        self.prm = None
        self.precision = precision
        self.stream = torch.cuda.Stream(device=self.dev)
        self.boxes, self.states, self.outs, self.cells, self.nbytes = [], [], [], [], []
        self._dt = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.t0_event = torch.cuda.Event(enable_timing=True)
        self.t0_host = None

    def add_patch(self, patch):
        torch = self.torch
        u = abi.Fab(torch.from_numpy(np.ascontiguousarray(patch.fab.data)).to(self.dev), tuple(patch.fab.lo))
        n = [patch.hi[d] - patch.lo[d] + 1 for d in range(3)]
        h = abi.Fab(torch.zeros((self.nv, n[2], n[1], n[0]), dtype=torch.float64, device=self.dev), tuple(patch.lo))
        if self.prm is None:
            self.prm = abi.make_params(patch.dx, 0.0, self.ns, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0),
                                       precision_mode=self.precision)
        b = hydro.make_box(patch.lo, patch.hi, u, h, patch.dx, 0.0)
        hydro.estdt(self.ns, [b], self.cfl, self._dt)
        b.dt = float(self._dt.item())
        self.boxes.append(b)
        self.states.append(u)
        self.outs.append(h)
        self.cells.append(patch.ncells)
        self.nbytes.append(hydro.workspace_bytes(self.prm, [(patch.lo, patch.hi)]))
        return len(self.boxes) - 1

    def request(self, rid, pid, arrival):
        return Request(rid, pid, float(arrival), self.cells[pid], self.nbytes[pid])

    def start(self):
        torch = self.torch
        torch.cuda.synchronize(self.dev)
        self.t0_event.record(self.stream)
        self.t0_event.synchronize()
        self.t0_host = time.perf_counter()

    def now(self):
        return time.perf_counter() - self.t0_host

    def launch(self, batch):
        hydro.hydro_boxes(self.prm, [self.boxes[r.pid] for r in batch], self.stream)
        ev = self.torch.cuda.Event(enable_timing=True)
        ev.record(self.stream)
        return ev

    def done(self, ev):
        return ev.query()

    def finish_time(self, ev):
        return self.t0_event.elapsed_time(ev) / 1e3

    def idle(self, next_arrival, busy):
        wait = self.poll_s
        if next_arrival is not None and not busy:
            wait = max(0.0, min(next_arrival - self.now(), 1e-3))
        time.sleep(wait)

    def synchronize(self):
        self.stream.synchronize()


def serve_sweep(executor, pids, budget_bytes, loads=(0.1, 0.25, 0.5, 0.75, 0.9, 1.0), seed=11, max_inflight=2):
    """Saturated throughput (all requests at t=0), then Poisson arrivals at the given
    fractions of the saturated request rate. Returns one summary per load."""
    out = []
    ex = executor
    sat = None
    # the first saturated run grows the workspace pool to the largest batch; the second
    # is the measured one
    for rep, load in enumerate((math.inf, math.inf) + tuple(loads)):
        if load is math.inf:
            arr = np.zeros(len(pids))
        else:
            arr = poisson_arrivals(len(pids), load * sat, seed)
        reqs = [ex.request(k, p, a) for k, (p, a) in enumerate(zip(pids, arr))]
        ex.start()
        sch = Scheduler(ex, budget_bytes, max_inflight=max_inflight)
        sch.run(reqs)
        s = summarize(reqs)
        s["load"] = "saturated" if load is math.inf else load
        s["peak_bytes"] = sch.peak_bytes
        if load is math.inf:
            sat = len(pids) / s["makespan_s"]
            s["requests_per_s"] = sat
        if rep > 0:
            out.append(s)
    return out
