#!/usr/bin/env python
"""Benchmark of the B200 Godunov hydro advance on the production flame level.

Workload (the configuration the headline metric is quoted on): a 128^3 level tiled
into 64 boxes of 32^3 with 4 ghost cells, 9-species H2/air with the NASA-7 mixture
EOS (stand-in coefficients), tanh flame front along z, periodic x/y, outflow z, PPM,
CFL 0.3. Inputs are seeded synthetic states of that shape (no dataset exists for this
path). One step = ghost fill + CFL timestep + construct_hydro_source over all boxes
+ state update with the temperature Newton solve, all on the device.

Our arm (default): the batched mixed-precision form (FP32 trace/Riemann/transverse,
FP64 state, flux divergence, Newton and dt), one CUDA graph per step. Reported beside
it: the plain FP64 drop-in (per-box pcg_hydro_box semantics, reference operation
order), the error of the mixed step against the FP64 form, the end-to-end rate
through the public API with host buffers, per-kernel CUDA-event timings, the roofline
of the dominant kernel and of the whole step, and the reference's own CPU code timed
on the host cores.

--impl reference: the reference's hot-path sources compiled in place (oracle/_ref,
-O3 -march=native) timed on all host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s per hydro step, mixed vs FP64 GPU at ≤1e-6 L1; p50/p99 patch ms"
UNIT = "cell-updates/s"
WORKLOAD = "h2air_flame_level_128^3_as_64x32^3_ns9_ppm_cfl0.3"
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=128, help="level edge")
    ap.add_argument("--box", type=int, default=32, help="box edge")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU-baseline work budget")
    ap.add_argument("--serve-requests", type=int, default=5000, help="step requests per serving load point")
    ap.add_argument("--serve-loads", type=float, nargs="*", default=[0.1, 0.25, 0.5, 0.75, 0.8, 0.9, 1.0])
    ap.add_argument("--serve-batch-cells", type=int, default=500_000, help="cells per serving batch at most")
    ap.add_argument("--serve-inflight", type=int, default=3, help="serving batches running at once (streams)")
    ap.add_argument("--sweep-steps", type=int, default=100, help="steps of the precision sweep")
    ap.add_argument("--no-side-workloads", action="store_true",
                    help="skip the batching, precision-sweep and serving workloads (quick runs)")
    ap.add_argument("--cpu-configs", action="store_true",
                    help="only time the CPU baseline on the Sod box, the flame level and the turbulence level "
                         "(PPM and PLM), one JSON line each")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
def pci_bus_id(local):
    """The PCI bus ID ("DDDDDDDD:BB:DD.0") of CUDA device ``local`` of this process, which
    names the same physical GPU for NVML and nvidia-smi whatever CUDA_VISIBLE_DEVICES is."""
    import torch

    p = torch.cuda.get_device_properties(local)
    return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"


class ClockSampler:
    """Samples the SM clock, power and clock-event reasons of the process's GPU (found by
    its PCI bus ID) every ``period_s`` while the timed region runs: NVML from a thread
    (read-only queries), or nvidia-smi at 100 ms where NVML is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, local, period_s=0.01):
        self.bus = pci_bus_id(local)
        self.period = period_s
        self.rows = []  # (sm_mhz, sm_max_mhz, power_w, reasons)
        self.proc = self.path = self.thread = None
        self.stop = False

    def _nvml_loop(self, nv, h):
        while not self.stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1e3
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                rs = [n for n, c in self.REASONS if bits & getattr(nv, c)]
                self.rows.append((float(sm), float(mx), pw, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        try:
            import threading

            import pynvml as nv

            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByPciBusId(self.bus)
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            try:
                self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.bus}", f"--query-gpu={SMI_FIELDS}",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            except OSError:
                self.proc = None
        time.sleep(0.05)
        return self

    def __exit__(self, *exc):
        self.stop = True
        if self.thread is not None:
            self.thread.join(timeout=2)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.path:
            names = [n for n, _ in self.REASONS]
            try:
                for ln in open(self.path):
                    f = [x.strip() for x in ln.split(",")]
                    if len(f) >= 9:
                        rs = [names[i] for i in range(4) if f[5 + i].lower().startswith("active")]
                        self.rows.append((float(f[1]), float(f[2]), float(f[3]) if f[3] not in ("", "[N/A]") else 0.0,
                                          rs))
            finally:
                os.unlink(self.path)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0,
                    "gpu": self.bus}
        sm = sorted(r[0] for r in self.rows)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.rows[0][1],
                "reasons": sorted({x for r in self.rows for x in r[3]}), "samples": len(self.rows),
                "power_w_max": max(r[2] for r in self.rows), "gpu": self.bus,
                "source": "nvml" if self.thread is not None else "nvidia-smi"}


# ---------------------------------------------------------------- CPU baseline
class CpuArm:
    """The reference's own hot path (oracle/_ref: Source/Godunov.cpp and PPM.cpp compiled
    in place, -O3 -march=native) or, where that build is absent, the oracle port, run
    box-parallel on all host threads (the reference tiles boxes over OpenMP threads,
    Source/Hydro.cpp:60-71). Each measurement is a bounded sample of one step's boxes."""

    def __init__(self, level, ppm_type=1):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        from particleclem_b200 import abi

        self.kind = "reference" if pyoracle.ref_available(level.nspec, fast=True) else "port"
        self.lib = pyoracle.reference(level.nspec, fast=True) if self.kind == "reference" else pyoracle.oracle(fast=True)
        self.lib.set_eos(level.eos)
        self.cores = len(os.sched_getaffinity(0))
        self.fabs = [(lo, hi, level.box_fab(lo, hi)) for lo, hi in level.boxes]
        dt = 0.3 * min(self.lib.estdt(lo, hi, f, level.dx) for lo, hi, f in self.fabs)
        self.prm = abi.make_params(level.dx, dt, level.nspec, level.domlo, level.domhi, level.bclo, level.bchi,
                                   ppm_type=ppm_type)
        t0 = time.perf_counter()
        self.lib.hydro_box(self.prm, *self.fabs[0])
        self.t_box = time.perf_counter() - t0
        self.pool = ThreadPoolExecutor(max_workers=self.cores)

    def measure(self, seconds):
        per_round = max(1, min(len(self.fabs), self.cores))
        rounds = max(1, int(seconds / max(self.t_box * 1.2, 1e-3)))
        nbox = rounds * per_round  # the step's boxes, repeated where the step is shorter than the budget
        work = [self.fabs[b % len(self.fabs)] for b in range(nbox)]
        t0 = time.perf_counter()
        list(self.pool.map(lambda w: self.lib.hydro_box(self.prm, *w), work))
        el = time.perf_counter() - t0
        ncell = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h, _ in work)
        thr = min(self.cores, nbox)
        return {"value": ncell / el, "unit": UNIT, "cores": thr, "kind": self.kind,
                "sample": f"{nbox} box advances over the {len(self.fabs)} boxes of one step "
                          f"(construct_hydro_source incl. ctoprim, FP64), {el:.1f} s on {thr} threads"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from particleclem_b200 import workloads as wl

    arm = CpuArm(wl.flame(n=args.n, box=args.box))
    per_step = max(1.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    vals, last = [], None
    for s in range(args.warmup + args.steps):
        last = arm.measure(per_step)
        if s >= args.warmup:
            vals.append(last["value"])
    v = sum(vals) / len(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": "reference FP64 CPU path, box-parallel on host threads"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": last["cores"], "kind": last["kind"],
                             "sample": last["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- our arm
def run_cpu_configs(args):
    """The CPU baseline on every level workload: the 32^3 Sod box (one species), the
    128^3 flame level, the 256^3 turbulence level with PPM and with PLM."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    from particleclem_b200 import workloads as wl

    def sod_tiled():
        # one 32^3 box, cut into the 32x8x8 tiles the reference's OpenMP box loop uses
        # (AMReX default CPU tile size 1024x8x8), so that the box spreads over 16 threads
        lev = wl.sod(n=32)
        lev.boxes = wl.tile_boxes((32, 32, 32), (32, 8, 8))
        return lev

    cases = [("sod_32^3_ns1_ppm (32x8x8 tiles)", sod_tiled, 1),
             (WORKLOAD, lambda: wl.flame(n=128, box=32, seed=2), 1),
             ("turbulence_256^3_as_64x64^3_ns1_ppm", lambda: wl.turbulence(n=256, box=64, seed=4), 1),
             ("turbulence_256^3_as_64x64^3_ns1_plm", lambda: wl.turbulence(n=256, box=64, seed=4), 0)]
    for name, make, ppm in cases:
        arm = CpuArm(make(), ppm_type=ppm)
        arm.measure(min(2.0, args.cpu_seconds))  # warm
        vals = [arm.measure(args.cpu_seconds / 5) for _ in range(5)]
        vals.sort(key=lambda r: r["value"])
        med = vals[2]  # median of five samples
        print(json.dumps({"config": {"workload": name}, "cpu_baseline": med,
                          "runs": [round(r["value"]) for r in vals]}), flush=True)
        arm.pool.shutdown()
    return 0


def rel_grouped(a, b, nspec):
    """Per-component relative L1 and Linf of b against a (component-major CUDA tensors),
    each component normalised by the sum / max of its physical group: mass (rho and the
    species densities), momentum (three components), energy (rho E, rho e), temperature."""
    import torch

    nv = a.shape[0]
    d = (a - b).abs().reshape(nv, -1)
    r = a.abs().reshape(nv, -1)
    s1, sinf = r.sum(1), r.max(1).values
    g1, ginf = torch.ones_like(s1), torch.ones_like(s1)
    for grp in ([0] + list(range(7, 7 + nspec)), [1, 2, 3], [4, 5], [6]):
        grp = [c for c in grp if c < nv]
        g1[grp] = s1[grp].max().clamp_min(1e-300)
        ginf[grp] = sinf[grp].max().clamp_min(1e-300)
    return (d.sum(1) / g1).cpu().numpy(), (d.max(1).values / ginf).cpu().numpy()


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from particleclem_b200 import abi, autotune, hydro, workloads as wl
    from particleclem_b200.level import LevelStepper

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- headline: batched mixed form, fused plan, CUDA graphs. One GPU: the 128^3 level.
    # N GPUs: one level of n x n x (n*N) cut into z-slabs of n^3, one per rank, with the
    # 4-cell halo exchange (NCCL send/recv) and the dt all-reduce-min every step.
    if world == 1:
        lev = wl.flame(n=args.n, box=args.box, seed=2)
        st = LevelStepper(lev, precision=abi.PREC_MIXED, fuse=True, device=local)
        st.step()  # valid dt and intermediates for the launch-shape autotuner
        tuned = {"mixed": autotune.tune(st.plan, st.dt, reps=3, state=st.state.data)}
        st.capture()
        step_fn = st.replay
        parallelism = "single GPU"
    else:
        from particleclem_b200.slab import DistComm, SlabStepper, step as slab_step

        slab = wl.flame_slab(n=args.n, nz=args.n * world, nranks=world, rank=rank, box=args.box, seed=2)
        st = SlabStepper(slab, world, rank, precision=abi.PREC_MIXED, fuse=True, device=local)
        st.fill()
        st.plan.estdt(st.cfl, st.dt)  # a local dt for the launch-shape autotuner
        tuned = {"mixed": autotune.tune(st.plan, st.dt, reps=3, state=st.state.data)}
        st.capture()  # leaves the slab's state as generated
        comm = DistComm()

        def step_fn():
            slab_step([st], comm)

        parallelism = (f"z-slabs x{world}: one {args.n}x{args.n}x{args.n * world} level, {args.n}^3 per GPU, "
                       "4-cell halo exchange (NCCL send/recv) + dt all-reduce-min every step")
    ncell = st.ncells
    for _ in range(args.warmup):
        step_fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(args.steps):
            step_fn()
        e1.record()
        barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    clocks = clk.summary()
    value = world * ncell * args.steps / (ms / 1e3)
    if world > 1:
        # end to end for the decomposed level: every step uploads each slab's state from
        # pinned host memory, steps (with the exchange) and downloads it
        host_in = torch.from_numpy(slab.state).pin_memory()
        host_out1 = torch.empty_like(host_in).pin_memory()
        h2d = d2h = host_in.numel() * 8
        for _ in range(2):
            st.load_state(host_in, non_blocking=True)
            step_fn()
            host_out1.copy_(st.state.data, non_blocking=True)
        barrier()
        kp = ke = max(2, min(args.steps, 5))
        e0.record()
        for _ in range(kp):
            st.load_state(host_in, non_blocking=True)
            step_fn()
            host_out1.copy_(st.state.data, non_blocking=True)
        e1.record()
        barrier()
        mse = mse_serial = max_over_ranks(e0.elapsed_time(e1))
        e2e_value = e2e_serial = world * ncell * kp / (mse / 1e3)
        lev = wl.flame(n=args.n, box=args.box, seed=2 + rank)  # per-GPU level for the side measurements

    # ---- fixed cost of the step's launch sequence: the same CUDA graph (ghost fill, 6
    # hydro stages, fused tail, final minimum) on an 8^3 level, whose kernels do almost no
    # work; it bounds what merging the launches into one persistent kernel could save
    tiny = LevelStepper(wl.flame(n=8, box=8, seed=2), precision=abi.PREC_MIXED, fuse=True, device=local)
    tiny.capture()
    for _ in range(20):
        tiny.replay()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(200):
        tiny.replay()
    e1.record()
    torch.cuda.synchronize()
    graph_overhead = {"workload": "flame level 8^3, one box", "launches": LevelStepper.launches_per_step,
                      "ms_per_step": e0.elapsed_time(e1) / 200}
    tiny.close()

    # ---- per-stage CUDA-event timings of the same step (not graph-captured)
    # "advance" is the launch sequence the level step uses: the hydro stages up to flux2,
    # then flux divergence + update + computeTemp + next CFL minimum in one pass
    names = ["fill", "estdt"] + ["hydro." + s for s in hydro.Plan.STAGES] + ["update", "advance"]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)]
    stage_ms = np.zeros(len(names))
    dt_next = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(args.steps):
        ev[0].record()
        st.fill()
        ev[1].record()
        st.plan.estdt(st.cfl, st.dt)
        ev[2].record()
        for s in range(7):
            st.plan.stages(s, s, st.dt)
            ev[3 + s].record()
        st.plan.update(st.dt)
        ev[10].record()
        st.plan.advance(st.cfl, st.dt, dt_next)
        ev[11].record()
        torch.cuda.synchronize()
        stage_ms += [ev[i].elapsed_time(ev[i + 1]) for i in range(len(names))]
    stage_ms /= args.steps
    st.close()

    # ---- plain FP64 drop-in: per-box (reference) semantics, reference operation order
    lev64 = wl.flame(n=args.n, box=args.box, seed=2 + rank)
    st64 = LevelStepper(lev64, precision=abi.PREC_FP64, fuse=False, device=local)
    st64.step()
    tuned["fp64"] = autotune.tune(st64.plan, st64.dt, reps=3)
    st64.capture()
    st64.replay()
    barrier()
    k64 = max(1, min(args.steps, 5))
    e0.record()
    for _ in range(k64):
        st64.replay()
    e1.record()
    barrier()
    ms64 = max_over_ranks(e0.elapsed_time(e1))
    fp64_value = world * ncell * k64 / (ms64 / 1e3)
    st64.close()

    # ---- error of one mixed step against the plain FP64 form. The FP64 form (reference
    # operation order, per box) is the one the parity tests show bit-identical to the CPU
    # oracle (hydro source and fluxes, 32^3 flame boxes of this level included), so these are
    # errors against the oracle's arithmetic. Both outputs are compared: the updated state
    # S_new (the bound 1e-6 applies to it) and the hydro source of the step.
    sa = LevelStepper(wl.flame(n=args.n, box=args.box, seed=2 + rank), precision=abi.PREC_FP64, fuse=False,
                      device=local)
    sb = LevelStepper(wl.flame(n=args.n, box=args.box, seed=2 + rank), precision=abi.PREC_MIXED, fuse=True,
                      device=local)
    sa.fill()
    sb.fill()
    sa.plan.estdt(sa.cfl, sa.dt)
    sb.dt.copy_(sa.dt)  # the same timestep on both sides: the difference is precision only
    sa.plan.hydro(sa.dt)
    sb.plan.hydro(sb.dt)
    torch.cuda.synchronize()
    src_l1, src_linf = rel_grouped(sa.hsrc.data, sb.hsrc.data, 9)
    sa.plan.update(sa.dt)
    sb.plan.update(sb.dt)
    torch.cuda.synchronize()
    g = 4
    A = sa.state.data[:, g:-g, g:-g, g:-g]
    B = sb.state.data[:, g:-g, g:-g, g:-g]
    l1, linf = rel_grouped(A, B, 9)
    comp = ["rho", "mx", "my", "mz", "rhoE", "rhoe", "T"] + [f"rhoY{k}" for k in range(9)]
    err = {"reference_side": "plain FP64 GPU form, per box, reference operation order: bit-identical to the CPU "
                             "oracle in the parity tests",
           "normalisation": "per component, by the sum (L1) / max (Linf) of its physical group (mass, momentum, "
                            "energy, temperature)",
           "s_new": {"max_rel_l1": float(l1.max()), "max_rel_linf": float(linf.max()),
                     "per_component_rel_l1": {c: float(v) for c, v in zip(comp, l1)}},
           "hydro_source": {"max_rel_l1": float(src_l1.max()), "max_rel_linf": float(src_linf.max())},
           "bound": "max_rel_l1 of s_new <= 1e-6"}
    sa.close()
    sb.close()

    # ---- end to end through the public API with host buffers: every step uploads its
    # state from pinned host memory and downloads the advanced state. Serial form first
    # (one stepper: copy in, step, copy out), then the pipelined form (HostPipeline: the
    # upload of step k+1 and the download of step k-1 overlap the step k).
    from particleclem_b200.level import HostPipeline

    lev_e = wl.flame(n=args.n, box=args.box, seed=2 + rank) if world == 1 else None
    if world == 1:
        host_in = torch.from_numpy(lev_e.state).pin_memory()
        host_out = [torch.empty_like(host_in).pin_memory() for _ in range(2)]
        se = LevelStepper(lev_e, precision=abi.PREC_MIXED, fuse=True, device=local)
        h2d = d2h = se.row_bytes  # the valid rows each way; the step's ghost fill forms the rest
        for _ in range(2):
            se.upload(host_in)
            se.step()
            se.download(host_out[0])
        barrier()
        ke = max(1, min(args.steps, 5))
        e0.record()
        for _ in range(ke):
            se.upload(host_in)
            se.step()
            se.download(host_out[0])
        e1.record()
        barrier()
        mse_serial = max_over_ranks(e0.elapsed_time(e1))
        e2e_serial = world * ncell * ke / (mse_serial / 1e3)
        se.close()

        pipe = HostPipeline(lev_e, depth=3, precision=abi.PREC_MIXED, fuse=True, device=local)
        assert (pipe.h2d_bytes, pipe.d2h_bytes) == (h2d, d2h)
        for i in range(3):
            pipe.submit(host_in, host_out[i % 2])
        pipe.synchronize()
        barrier()
        kp = max(20, args.steps)  # enough submissions that filling and draining the pipeline is amortised
        e0.record(pipe.up)
        for i in range(kp):
            pipe.submit(host_in, host_out[i % 2])
        e1.record(pipe.down)
        pipe.synchronize()
        barrier()
        mse = max_over_ranks(e0.elapsed_time(e1))
        e2e_value = world * ncell * kp / (mse / 1e3)
        pipe.close()

    # ---- serving: patch-step latency under Poisson arrivals with continuous batching
    # (16 ensemble runs x 32 flame patches of edges in {16..64}; every request one step of
    # a resident, evolving patch; HBM budget 120 GB; batches of at most --serve-batch-cells
    # cells, --serve-inflight of them at once on their own streams)
    from particleclem_b200.serve import ensemble_serving

    serving = None
    if not args.no_side_workloads:
        serving = ensemble_serving(lev.eos, nruns=16, per_run=32, seed=5 + rank, nreq=args.serve_requests,
                                   budget_bytes=int(120e9), loads=tuple(args.serve_loads),
                                   max_batch_cells=args.serve_batch_cells, error_sample=32, device=local,
                                   max_inflight=args.serve_inflight)

    # ---- batching (512 independent flame boxes, edges log-uniform in [8, 64]) and the
    # precision sweep (256^3 periodic turbulence as 64 boxes of 64^3, PPM and PLM): mixed
    # against the plain FP64 form, step times in CUDA graphs and errors
    from particleclem_b200.suite import batch_workload, sweep_workload

    batching = sweep = None
    if not args.no_side_workloads:
        batching = batch_workload(512, steps=5, warmup=3, device=local)
        sweep = sweep_workload(256, 64, steps=args.sweep_steps, every=10, device=local)

    # ---- roofline: the dominant kernel (one fused region of the whole level) and the step
    from particleclem_b200 import roofline as rl

    pk = rl.peaks(ROOT)
    edges = [lev.domhi[d] - lev.domlo[d] + 1 for d in range(3)]
    roof = rl.dominant_kernel_roofline(edges, 9, 4, names, stage_ms, pk, "mixed", ROOT)
    box_edges = [[h[d] - l[d] + 1 for d in range(3)] for l, h in lev.boxes]
    path_roof = rl.path_roofline(box_edges, 9, ms / args.steps, pk)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cpu = CpuArm(wl.flame(n=args.n, box=args.box, seed=2)).measure(args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64 (mixed: FP32 trace/Riemann/transverse, FP64 update/Newton/dt)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells_per_gpu": ncell, "boxes_per_gpu": len(lev.boxes),
                       "form": "batched mixed precision, boxes fused into one region, CUDA graph per step",
                       "parallelism": parallelism,
                       "l2": "inputs larger than L2 (state 0.34 GB, intermediates 3.4 GB per step)"},
            "fp64_dropin": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms64 / k64,
                            "form": "plain FP64, reference operation order, per-box (64 boxes), CUDA graph"
                                    + (", one level per GPU" if world > 1 else ""),
                            "speedup_of_mixed": value / fp64_value},
            "error_vs_fp64": err,  # errors against the oracle-equal FP64 form
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": mse / kp, "steps": kp,
                    "path": ("valid rows of a pinned host state -> H2D -> fill/estdt/hydro/update via C ABI -> "
                             "valid rows D2H, every step; level.HostPipeline (3 device slots) overlaps the step of "
                             "one submission with the upload of the next and the download of the previous")
                            if world == 1 else
                            "per rank: pinned host slab -> H2D -> slab step with halo exchange and dt all-reduce "
                            "-> D2H, every step",
                    "serial": {"value": e2e_serial, "ms_per_step": mse_serial / ke,
                               "path": "same copies and step, one after another"}},
            "serving": None if serving is None else {"workload": serving["workload"], "budget_gb": serving["budget_gb"],
                        "max_batch_cells": serving["max_batch_cells"], "max_inflight": args.serve_inflight,
                        "latency": "arrival to the host's observation of the batch's device completion",
                        "resident_state_gb": serving["resident_state_gb"],
                        "saturated_cell_updates_per_s": serving["points"][0]["cell_updates_per_s"],
                        "saturated_requests_per_s": serving["points"][0]["requests_per_s"],
                        "loads": [{k: r[k] for k in ("load", "requests", "p50_ms", "p99_ms", "cell_updates_per_s",
                                                     "batches", "peak_bytes")}
                                  for r in serving["points"][1:]],
                        "error_vs_fp64_one_step": serving["error_vs_fp64_one_step"]},
            "graph_step_overhead": graph_overhead,
            "batching": batching,
            "precision_sweep": sweep,
            "gpu_launches": LevelStepper.launches_per_step * args.steps,  # fill 1, stages 6, fused tail 1, final dt 1
            "launch_variants": {f: {k: v["variant"] for k, v in t.items()} for f, t in tuned.items()},
            "launch_tuning": tuned,
            "stage_ms": {n: float(v) for n, v in zip(names, stage_ms)},
            "roofline": roof,
            "path_roofline": path_roof,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.cpu_configs:
        return run_cpu_configs(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
