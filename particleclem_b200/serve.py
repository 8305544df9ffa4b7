"""Continuous-batching serving loop for ensemble patch steps.

A request asks for ONE STEP of one patch of an ensemble run: the ghost fill of the patch
(its own domain, zero-gradient faces), the hydro advance of construct_hydro_source
(Source/Hydro.cpp:4-301), S_new = S_old + dt * hydro_source with computeTemp written over
the patch's state (Source/Advance.cpp:397-417, Source/PeleC.cpp:2289-2305), and the
patch's next CFL timestep (Source/PeleC.cpp:829-960), which the patch's next request uses.
So every request evolves its patch; the states stay on the device between requests.

Admission. A waiting request is admitted when its patch is not already in a running batch
(steps of one patch stay in order) and the device bytes it needs fit the HBM budget: the
workspace of its step (pcg_hydro_workspace) plus, if its patch's state is not resident,
the state itself. To make room, idle resident states are evicted least recently used
first (copied back to host memory). Requests are taken in arrival order; a request whose
patch is busy is passed over, the first one that does not fit stops the batch.

Batching. All admitted requests, up to ``max_batch_cells`` cells, form ONE pcg_step_boxes
call (one launch per stage over all their boxes). Up to ``max_inflight`` batches run at the
same time, each on its own CUDA stream, so requests that arrive while a batch runs form
the next batch and overlap it on the device. The host waits for a batch completion or the
next arrival, whichever comes first, without polling.

Latency is arrival to the host's observation of the device completion of the request's
batch (a thread per batch blocks on the batch's CUDA event and stamps the host clock when
it returns): the time until a client could see the result, and free of the drift between
the GPU's event timer and the host clock over a long run. The scheduler is
device-independent:
an executor moves states, launches batches and keeps the clock; GpuExecutor runs them
through the library, the CPU tests drive the scheduler with a simulated executor.
"""
from __future__ import annotations

import math
import threading
import time
from collections import OrderedDict
from dataclasses import dataclass

import numpy as np

from . import abi, hydro


@dataclass
class Request:
    rid: int
    pid: int  # patch to advance by one step
    arrival: float  # seconds since the start of the run
    cells: int = 0
    nbytes: int = 0  # workspace bytes held from launch to completion
    state_bytes: int = 0  # device bytes of the patch's state while resident
    start: float = math.nan  # time the request's batch was launched
    finish: float = math.nan  # device completion time of its batch
    batch: int = -1  # index of the batch it ran in

    @property
    def latency(self):
        return self.finish - self.arrival


class BudgetError(ValueError):
    pass


class Scheduler:
    def __init__(self, executor, budget_bytes, max_inflight=2, max_batch=None, max_batch_cells=None):
        self.ex = executor
        self.budget = int(budget_bytes)
        self.max_inflight = int(max_inflight)
        self.max_batch = max_batch
        self.max_batch_cells = max_batch_cells
        self.peak_bytes = 0
        self.nbatches = 0
        self.evictions = 0
        self.uploads = 0
        # resident patch states, least recently used first: pid -> bytes
        states = executor.resident_states() if hasattr(executor, "resident_states") else []
        self.resident = OrderedDict((pid, b) for pid, b in states)
        self.used = sum(self.resident.values())

    def _evict_for(self, need, keep):
        """Evict idle resident states (LRU first) until ``need`` more bytes fit; False if
        they cannot."""
        if self.used + need <= self.budget:
            return True
        idle = sum(b for pid, b in self.resident.items() if pid not in keep)
        if self.used - idle + need > self.budget:
            return False  # evicting every idle state would not make room: evict nothing
        for pid in list(self.resident):
            if self.used + need <= self.budget:
                break
            if pid in keep:
                continue
            self.ex.evict(pid)
            self.used -= self.resident.pop(pid)
            self.evictions += 1
        return self.used + need <= self.budget

    def run(self, requests):
        """Serve ``requests`` (arrival times relative to the executor's start) to
        completion; fills start/finish/batch in place and returns them."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in reqs:
            if r.nbytes + r.state_bytes > self.budget:
                raise BudgetError(f"request {r.rid} needs {r.nbytes + r.state_bytes} bytes, budget {self.budget}")
        ex = self.ex
        i, n = 0, len(reqs)
        waiting, inflight = [], []
        busy = set()  # patches in running batches
        while i < n or waiting or inflight:
            now = ex.now()
            while i < n and reqs[i].arrival <= now:
                waiting.append(reqs[i])
                i += 1
            progressed = False
            for h, batch, slot in [x for x in inflight if ex.done(x[0])]:  # a batch on another stream may finish first
                inflight.remove((h, batch, slot))
                t = ex.finish_time(h)
                for r in batch:
                    r.finish = t
                    self.used -= r.nbytes
                    busy.discard(r.pid)
                progressed = True
            if waiting and len(inflight) < self.max_inflight:
                batch, cells, rest = [], 0, []
                stop = len(waiting)  # index of the first request the scan did not reach
                for idx, r in enumerate(waiting):
                    if r.pid in busy:
                        rest.append(r)
                        continue
                    if batch and ((self.max_batch is not None and len(batch) >= self.max_batch) or (
                            self.max_batch_cells is not None and cells + r.cells > self.max_batch_cells)):
                        stop = idx
                        break
                    need = r.nbytes + (0 if r.pid in self.resident else r.state_bytes)
                    if not self._evict_for(need, busy):
                        stop = idx  # first come first served: nothing overtakes a request that does not fit
                        break
                    if r.pid not in self.resident:
                        self.resident[r.pid] = r.state_bytes
                        self.uploads += 1
                    self.resident.move_to_end(r.pid)
                    self.used += need
                    busy.add(r.pid)
                    r.start = now
                    r.batch = self.nbatches
                    batch.append(r)
                    cells += r.cells
                waiting = rest + waiting[stop:]  # the passed-over requests keep their order
                if batch:
                    self.peak_bytes = max(self.peak_bytes, self.used)
                    slots = {s for _, _, s in inflight}
                    slot = next(k for k in range(self.max_inflight) if k not in slots)  # a stream not in use
                    inflight.append((ex.launch(batch, slot), batch, slot))
                    self.nbatches += 1
                    progressed = True
            if not progressed:
                nxt = reqs[i].arrival if i < n else None
                ex.idle(nxt, [x[0] for x in inflight])
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
    """Runs batches of patch steps with pcg_step_boxes, one CUDA stream per in-flight slot.

    Each patch keeps its state in pinned host memory while not resident and on the device
    while resident, and its current timestep in a device array (the first one is the CFL
    timestep of its initial state). Every patch is its own domain with zero-gradient
    (outflow) faces."""

    def __init__(self, eos, precision=abi.PREC_MIXED, cfl=0.3, device=0, nstreams=2):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        hydro.init(device)
        hydro.set_eos(eos)
        self.ns = eos.nspec
        self.nv = abi.nvar(self.ns)
        self.cfl = float(cfl)
        self.precision = precision
        self.prm = abi.make_params((1, 1, 1), 0.0, self.ns, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0),
                                   precision_mode=precision)
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(nstreams)]
        self.copy_stream = torch.cuda.Stream(device=self.dev)  # evictions (device to host)
        self._evicted = {}  # pid -> event of its last eviction copy
        self.patches, self.host, self.dev_state, self.boxes = [], [], [], []
        self.cells, self.nbytes, self.state_nbytes = [], [], []
        self._dts = []
        self.dts = None  # device timesteps, one per patch
        self.t0_event = torch.cuda.Event(enable_timing=True)
        self.t0_host = None
        self._wake = threading.Event()
        self._finish = {}  # batch event -> host time its completion was observed
        self._pending_free = []  # (event, tensor) of evictions whose copy is in flight

    # ---- patches
    def add_patch(self, patch):
        torch = self.torch
        host = torch.from_numpy(np.ascontiguousarray(patch.fab.data)).pin_memory()
        self.patches.append(patch)
        self.host.append(host)
        self.dev_state.append(None)
        self.boxes.append(None)
        self.cells.append(patch.ncells)
        self.state_nbytes.append(host.numel() * 8)
        self.nbytes.append(hydro.workspace_bytes(self.prm, [(patch.lo, patch.hi)]))
        # first timestep: the CFL timestep of the initial state (valid cells)
        u = abi.Fab(host.to(self.dev), tuple(patch.fab.lo))
        b = self._box(len(self.patches) - 1, u)
        dt = torch.zeros(1, dtype=torch.float64, device=self.dev)
        hydro.estdt(self.ns, [b], self.cfl, dt)
        self._dts.append(float(dt.item()))
        self.dts = None
        return len(self.patches) - 1

    def _box(self, pid, u):
        p = self.patches[pid]
        ob = (abi.BC_OUTFLOW,) * 3
        return hydro.make_box(p.lo, p.hi, u, None, p.dx, 0.0, p.lo, p.hi, ob, ob)

    def request(self, rid, pid, arrival):
        return Request(rid, pid, float(arrival), self.cells[pid], self.nbytes[pid], self.state_nbytes[pid])

    def resident_states(self):
        return [(pid, self.state_nbytes[pid]) for pid, s in enumerate(self.dev_state) if s is not None]

    def _make_resident(self, pid, stream):
        torch = self.torch
        ev = self._evicted.pop(pid, None)
        if ev is not None:
            stream.wait_event(ev)  # the host copy of an evicted state must be complete
        with torch.cuda.stream(stream):
            d = torch.empty_like(self.host[pid], device=self.dev)
            d.copy_(self.host[pid], non_blocking=True)
        u = abi.Fab(d, tuple(self.patches[pid].fab.lo))
        self.dev_state[pid] = u
        self.boxes[pid] = self._box(pid, u)

    def evict(self, pid):
        """Copy an idle patch's state back to host memory and release its device copy
        once the copy is done."""
        torch = self.torch
        u = self.dev_state[pid]
        # the patch is idle: the batches that stepped it have completed on the device
        s = self.copy_stream
        with torch.cuda.stream(s):
            self.host[pid].copy_(u.data, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        self._evicted[pid] = ev
        self._pending_free.append((ev, u.data))
        self.dev_state[pid] = None
        self.boxes[pid] = None

    def reserve(self, max_inflight, max_batch_cells=None, cap_bytes=None):
        """Grow the library's workspace pool to hold ``max_inflight`` batches of at most
        ``max_batch_cells`` cells (every patch when None), at most ``cap_bytes``, so that no
        batch waits for the driver to map memory for a workspace size it has not seen
        before."""
        per_cell = max(b / c for b, c in zip(self.nbytes, self.cells))
        cells = sum(self.cells) if max_batch_cells is None else max_batch_cells
        batch = max(per_cell * min(cells, sum(self.cells)), max(self.nbytes))
        nbytes = int(max_inflight * batch * 1.25)
        if cap_bytes is not None:
            nbytes = min(nbytes, int(cap_bytes))
        hydro.reserve_workspace(self.dev.index or 0, nbytes)

    # ---- clock and batches
    def start(self):
        torch = self.torch
        if self.dts is None:
            self.dts = torch.tensor(self._dts, dtype=torch.float64, device=self.dev)
        torch.cuda.synchronize(self.dev)
        self.t0_event.record(self.streams[0])
        self.t0_event.synchronize()
        self.t0_host = time.perf_counter()

    def now(self):
        return time.perf_counter() - self.t0_host

    def launch(self, batch, slot):
        torch = self.torch
        s = self.streams[slot % len(self.streams)]
        for r in batch:
            if self.dev_state[r.pid] is None:
                self._make_resident(r.pid, s)
        pids = [r.pid for r in batch]
        with torch.cuda.stream(s):
            idx = torch.tensor(pids, dtype=torch.int64).pin_memory().to(self.dev, non_blocking=True)
            dt = self.dts.index_select(0, idx)
            dt_next = torch.empty_like(dt)
            hydro.step_boxes(self.prm, [self.boxes[p] for p in pids], self.cfl, dt, dt_next, True, s)
            self.dts.index_copy_(0, idx, dt_next)
            ev = torch.cuda.Event(enable_timing=True, blocking=True)
            ev.record(s)
        threading.Thread(target=self._watch, args=(ev,), daemon=True).start()
        return ev

    def _watch(self, ev):
        ev.synchronize()  # blocking wait (no spinning), GIL released
        self._finish[ev] = self.now()
        self._wake.set()

    def done(self, ev):
        return ev in self._finish  # stamped by its watcher

    def finish_time(self, ev):
        return self._finish.pop(ev)

    def idle(self, next_arrival, handles):
        # sleep until a running batch completes or the next request arrives
        if self._pending_free:
            self._pending_free = [(e, t) for e, t in self._pending_free if not e.query()]
        if handles and any(self.done(h) for h in handles):
            return
        timeout = None if next_arrival is None else max(0.0, next_arrival - self.now())
        if not handles and timeout is None:
            return
        self._wake.wait(timeout)
        self._wake.clear()

    def synchronize(self):
        for s in self.streams + [self.copy_stream]:
            s.synchronize()

    def state(self, pid):
        """The patch's current state on the host (numpy), wherever it lives."""
        self.synchronize()
        if self.dev_state[pid] is not None:
            return self.dev_state[pid].data.cpu().numpy()
        return self.host[pid].numpy().copy()


def serve_sweep(executor, pids, budget_bytes, loads=(0.1, 0.25, 0.5, 0.75, 0.8, 0.9, 1.0), nreq=None, seed=11,
                max_inflight=2, max_batch_cells=None):
    """Saturated throughput (all requests at t=0), then Poisson arrivals at the given
    fractions of the saturated request rate. Each request steps a patch drawn uniformly
    (seeded) from ``pids``; ``nreq`` requests per point (default: one per patch). Returns
    one summary per load."""
    out = []
    ex = executor
    nreq = len(pids) if nreq is None else int(nreq)
    rng = np.random.default_rng(seed)
    # the first saturated run warms the memory pool and the streams; the second is measured.
    # The cyclic garbage collector is off while requests are served (its pauses would show
    # as latency outliers of the host loop), and the interpreter switches threads every
    # 0.2 ms so that a batch-completion watcher reaches the scheduler promptly.
    import gc
    import sys

    gc_was, switch = gc.isenabled(), sys.getswitchinterval()
    gc.disable()
    sys.setswitchinterval(2e-4)
    try:
        return _sweep(ex, pids, budget_bytes, loads, nreq, rng, seed, max_inflight, max_batch_cells, out)
    finally:
        sys.setswitchinterval(switch)
        if gc_was:
            gc.enable()


def _sweep(ex, pids, budget_bytes, loads, nreq, rng, seed, max_inflight, max_batch_cells, out):
    sat = None
    if hasattr(ex, "reserve"):
        ex.reserve(max_inflight, max_batch_cells, cap_bytes=budget_bytes)
    for rep, load in enumerate((math.inf, math.inf) + tuple(loads)):
        arr = np.zeros(nreq) if load is math.inf else poisson_arrivals(nreq, load * sat, seed + rep)
        choice = rng.choice(np.asarray(pids), size=nreq)
        reqs = [ex.request(k, int(p), a) for k, (p, a) in enumerate(zip(choice, arr))]
        ex.start()
        sch = Scheduler(ex, budget_bytes, max_inflight=max_inflight, max_batch_cells=max_batch_cells)
        sch.run(reqs)
        ex.synchronize()
        s = summarize(reqs)
        s["load"] = "saturated" if load is math.inf else load
        s["peak_bytes"] = sch.peak_bytes
        s["evictions"] = sch.evictions
        if load is math.inf:
            sat = nreq / s["makespan_s"]
            s["requests_per_s"] = sat
        if rep > 0:
            out.append(s)
    return out


def step_error(eos, patches, device=0):
    """Error of one mixed-form step against the plain FP64 form (bit-identical to the CPU
    oracle in the parity tests) on ``patches``, from the same state and timestep (each
    patch's FP64 CFL timestep): max over patches of the group-normalised relative L1 and
    Linf of S_new (the step's result, bound 1e-6 in L1) and of the hydro source."""
    import torch

    dev = torch.device("cuda", device)
    hydro.init(device)
    hydro.set_eos(eos)
    ns = eos.nspec
    nv = abi.nvar(ns)
    ob = (abi.BC_OUTFLOW,) * 3
    worst = {"s_new_rel_l1": 0.0, "s_new_rel_linf": 0.0, "hydro_source_rel_l1": 0.0, "hydro_source_rel_linf": 0.0}
    res = {}
    for form, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        prm = abi.make_params((1, 1, 1), 0.0, ns, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0), precision_mode=prec)
        states = [abi.Fab(torch.from_numpy(np.ascontiguousarray(p.fab.data)).to(dev), tuple(p.fab.lo))
                  for p in patches]
        srcs = [abi.Fab(torch.zeros((nv,) + tuple(p.hi[e] - p.lo[e] + 1 for e in (2, 1, 0)), dtype=torch.float64,
                                    device=dev), tuple(p.lo)) for p in patches]
        boxes = [hydro.make_box(p.lo, p.hi, s, h, p.dx, 0.0, p.lo, p.hi, ob, ob)
                 for p, s, h in zip(patches, states, srcs)]
        if form == "fp64":
            dts = torch.zeros(len(patches), dtype=torch.float64, device=dev)
            for k, b in enumerate(boxes):
                hydro.estdt(ns, [b], 0.3, dts[k:k + 1])
            dt_host = dts.cpu().numpy()
        for b, d in zip(boxes, dt_host):
            b.dt = float(d)
        dt_next = torch.zeros(len(patches), dtype=torch.float64, device=dev)
        hydro.step_boxes(prm, boxes, 0.3, dts, dt_next)  # fills the ghosts, steps S in place
        # the hydro source of the same step: from the old state with the filled ghosts
        old = [abi.Fab(torch.from_numpy(np.ascontiguousarray(p.fab.data)).to(dev), tuple(p.fab.lo)) for p in patches]
        for o, s in zip(old, states):  # ghost cells as the step filled them
            g = abi.NGROW
            mask = torch.ones_like(o.data, dtype=torch.bool)
            mask[:, g:-g, g:-g, g:-g] = False
            o.data[mask] = s.data[mask]
        ob_boxes = [hydro.make_box(p.lo, p.hi, o, h, p.dx, float(d), p.lo, p.hi, ob, ob)
                    for p, o, h, d in zip(patches, old, srcs, dt_host)]
        hydro.hydro_boxes(prm, ob_boxes)
        torch.cuda.synchronize(dev)
        res[form] = (states, srcs)
    g = abi.NGROW
    for (sa, ha), (sb, hb) in [((res["fp64"][0][k], res["fp64"][1][k]), (res["mixed"][0][k], res["mixed"][1][k]))
                               for k in range(len(patches))]:
        for key, a, b in (("s_new", sa.data[:, g:-g, g:-g, g:-g], sb.data[:, g:-g, g:-g, g:-g]),
                          ("hydro_source", ha.data, hb.data)):
            l1, li = _rel_grouped(a, b, ns)
            worst[key + "_rel_l1"] = max(worst[key + "_rel_l1"], float(l1.max()))
            worst[key + "_rel_linf"] = max(worst[key + "_rel_linf"], float(li.max()))
    worst["patches"] = len(patches)
    return worst


def _rel_grouped(a, b, nspec):
    """Per-component relative L1 and Linf of b against a (component-major CUDA tensors),
    each component normalised by the sum / max of its physical group: mass (rho and the
    species densities), momentum, energy (rho E, rho e), temperature."""
    import torch

    nv = a.shape[0]
    d = (a - b).abs().reshape(nv, -1)
    r = a.abs().reshape(nv, -1)
    s1, sinf = r.sum(1), r.max(1).values
    g1, ginf = torch.ones_like(s1), torch.ones_like(s1)
    for grp in ([abi.URHO] + list(range(abi.UFS, abi.UFS + nspec)), [abi.UMX, abi.UMY, abi.UMZ],
                [abi.UEDEN, abi.UEINT], [abi.UTEMP]):
        grp = [c for c in grp if c < nv]
        g1[grp] = s1[grp].max().clamp_min(1e-300)
        ginf[grp] = sinf[grp].max().clamp_min(1e-300)
    return (d.sum(1) / g1).cpu().numpy(), (d.max(1).values / ginf).cpu().numpy()


def ensemble_serving(eos, nruns=16, per_run=32, seed=5, nreq=5000, budget_bytes=int(120e9),
                     loads=(0.1, 0.25, 0.5, 0.75, 0.8, 0.9, 1.0), max_batch_cells=500_000, error_sample=32,
                     device=0, max_inflight=3):
    """The ensemble serving workload: ``nruns`` runs of ``per_run`` flame patches each with
    edges drawn from {16, 24, 32, 48, 64} (per axis, seeded per run), mixed precision,
    ``nreq`` step requests per load point on patches drawn uniformly, saturated throughput
    then Poisson arrivals at ``loads`` of it, under the HBM budget; plus the mixed-form
    error of one step against the FP64 form on ``error_sample`` patches."""
    from . import workloads as wl

    patches, _ = wl.serving_patches(nruns=nruns, per_run=per_run, seed=seed, eos=eos)
    ex = GpuExecutor(eos, precision=abi.PREC_MIXED, device=device, nstreams=max_inflight)
    pids = [ex.add_patch(p) for p in patches]
    res = serve_sweep(ex, pids, budget_bytes, loads=loads, nreq=nreq, max_batch_cells=max_batch_cells,
                      max_inflight=max_inflight)
    resident = sum(s for _, s in ex.resident_states())
    del ex
    err = step_error(eos, patches[:error_sample], device=device)
    return {"workload": f"{nruns} runs x {per_run} flame patches, edges in {{16,24,32,48,64}}, ns9, mixed, "
                        f"{nreq} step requests per load point",
            "budget_gb": budget_bytes / 1e9, "max_batch_cells": max_batch_cells,
            "resident_state_gb": resident / 1e9, "points": res, "error_vs_fp64_one_step": err}
