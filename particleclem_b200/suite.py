"""Measurement driver for the workloads beside the headline level step.

  python -m particleclem_b200.suite batch   512 independent flame boxes, edges log-uniform
                                            in [8, 64] per axis (9 species): one batched step
                                            (CUDA graph), mixed and plain FP64,
                                            per-component error of mixed against FP64
  python -m particleclem_b200.suite sweep   256^3 periodic turbulence in 64 boxes of 64^3
                                            (gamma law): PPM and PLM x {FP64, mixed}, error
                                            growth of mixed against FP64 over the steps
  python -m particleclem_b200.suite options the headline flame level with each reconstruction
                                            option (PPM, hybrid WENO-JS5/Z5/Z7/Z3) and with
                                            an inflow low-z face (low-order boundary fluxes),
                                            and the 32^3 Sod box: FP64 and mixed step times,
                                            mixed error
  python -m particleclem_b200.suite serve   16 ensemble runs of flame patches with edges in
                                            {16,24,32,48,64}, each request one step of a patch
                                            (states evolve and stay resident): saturated
                                            throughput and p50/p99 latency under Poisson
                                            arrivals at 10..100 % of it, HBM admission budget

  python -m particleclem_b200.suite step    a few eager steps of one level in one form (the
                                            workload of the kernel profiles)

Each prints one JSON line per result. All inputs are synthetic (seeded generators of
particleclem_b200.workloads). The plain FP64 form is bit-identical to the CPU
restatement of the reference (the GPU parity tests), so errors against it are errors
against the reference arithmetic.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

from . import abi, autotune, roofline as rl, workloads as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _timed(torch, fn, steps, warmup):
    for _ in range(warmup):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _rel_grouped(torch, a, b, nspec):
    """Per-component relative L1 and Linf of b against a, each component normalised by
    its physical group's scale (mass: rho and the species densities; momentum: the three
    components; energy: rho E and rho e; temperature), so that a near-zero component (the
    transverse momenta of a nearly planar Sod problem) is not measured against itself."""
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


def _rel(torch, a, b):
    """Per-component relative L1 and Linf of b against a (component-major tensors)."""
    d = (a - b).abs().reshape(a.shape[0], -1)
    r = a.abs().reshape(a.shape[0], -1)
    l1 = (d.sum(1) / r.sum(1).clamp_min(1e-300)).cpu().numpy()
    li = (d.max(1).values / r.max(1).values.clamp_min(1e-300)).cpu().numpy()
    return l1, li


def batch_workload(nbox=512, steps=10, warmup=3, device=0):
    """The batching workload: ``nbox`` independent flame boxes with edges log-uniform in
    [8, 64] per axis (9 species), one plan over all boxes, one CUDA graph per step; mixed
    and plain FP64 step times and the error of one mixed step against the FP64 one
    (group-normalised relative L1 / Linf of S_new)."""
    import torch

    from .batch import BoxBatch

    eos = wl.load_nasa7()
    patches = wl.flame_boxes(nbox, seed=3, eos=eos, lo=8, hi=64)
    ncell = sum(p.ncells for p in patches)
    pk = rl.peaks(ROOT)
    edges = [[p.hi[d] - p.lo[d] + 1 for d in range(3)] for p in patches]
    balg = sum(rl.b_alg_box(e, 9) for e in edges)
    res = {}
    states = {}
    launches = None
    tuned = {}
    for name, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
        bb = BoxBatch(patches, eos, precision=prec, device=device)
        bb.step()  # one step from the initial state, kept for the error
        torch.cuda.synchronize()
        states[name] = [s.data.clone() for s in bb.states]
        # launch shapes tuned for this batch's box sizes (both forms), the previous
        # table restored afterwards
        keep = {st: autotune.get_variant(prec, 9, st) for st in autotune.TUNED_STAGES + (autotune.TAIL_STAGE,)}
        tuned[name] = autotune.tune(bb.plan, bb.dt, reps=3, state=[s.data for s in bb.states])
        bb.capture()
        launches = bb.launches_per_step
        ms = _timed(torch, bb.replay, steps, warmup)
        res[name] = {"ms_per_step": ms, "cell_updates_per_s": ncell / (ms / 1e3),
                     "path_hbm_frac": balg / (ms / 1e3) / 1e9 / pk["hbm_gbs"]}
        bb.close()
        del bb
        for st, v in keep.items():
            autotune.set_variant(prec, 9, st, v)
        torch.cuda.empty_cache()
    g = abi.NGROW
    a = torch.cat([x[:, g:-g, g:-g, g:-g].reshape(x.shape[0], -1) for x in states["fp64"]], dim=1)
    b = torch.cat([x[:, g:-g, g:-g, g:-g].reshape(x.shape[0], -1) for x in states["mixed"]], dim=1)
    l1, li = _rel_grouped(torch, a, b, 9)
    return {"workload": f"flame_boxes_{nbox}_loguniform_8_64_ns9", "boxes": nbox, "cells": ncell,
            "mixed": res["mixed"], "fp64": res["fp64"],
            "speedup_mixed_over_fp64": res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"],
            "error_mixed_vs_fp64_one_step": {"s_new_max_rel_l1": float(l1.max()), "s_new_max_rel_linf": float(li.max()),
                                             "normalisation": "per physical group"},
            "launches_per_step": launches, "b_alg_bytes_per_step": balg, "peak_source": pk["source"],
            "launch_tuning": tuned}


def run_batch(args):
    print(json.dumps(batch_workload(args.nbox, args.steps, args.warmup)), flush=True)


def sweep_workload(n=256, box=64, steps=100, every=10, schemes=(1, 0), device=0):
    """The precision sweep: the periodic decaying-turbulence level (gamma law), PPM
    (scheme 1) and PLM (0), plain FP64 per box against mixed fused, step times (CUDA graphs)
    and the error growth of the mixed state against the FP64 one over ``steps`` steps taken
    with the FP64 run's timestep sequence (so the difference is precision only)."""
    import torch

    from .level import LevelStepper

    lev0 = wl.turbulence(n=n, box=box, seed=4)
    out = []
    for ppm in schemes:
        a = LevelStepper(lev0, precision=abi.PREC_FP64, fuse=False, ppm_type=ppm, device=device)
        b = LevelStepper(lev0, precision=abi.PREC_MIXED, fuse=True, ppm_type=ppm, device=device)
        # launch shapes tuned on each form's own plan for this level (one species), the
        # previous table restored after the measurement
        keep, tuned = {}, {}
        for name, st in (("fp64", a), ("mixed", b)):
            prec = st.prm.precision_mode
            keep[prec] = {k: autotune.get_variant(prec, 1, k) for k in autotune.TUNED_STAGES + (autotune.TAIL_STAGE,)}
            st.step()
            tuned[name] = autotune.tune(st.plan, st.dt, reps=3, state=st.state.data)
        a.capture()
        b.capture()
        ms_a = _timed(torch, a.replay, 3, 2)
        ms_b = _timed(torch, b.replay, 3, 2)
        a.graph = b.graph = None
        a.state.data.copy_(torch.from_numpy(lev0.state).to(a.dev))
        b.state.data.copy_(a.state.data)
        growth = []
        g = abi.NGROW
        for s in range(1, steps + 1):
            a.fill()
            a.plan.estdt(a.cfl, a.dt)
            a.plan.hydro(a.dt)
            a.plan.update(a.dt)
            b.fill()
            b.dt.copy_(a.dt)  # the same timestep sequence: the difference is precision only
            b.plan.hydro(b.dt)
            b.plan.update(b.dt)
            if s in (1, 2, 5) or s % every == 0:
                l1, li = _rel_grouped(torch, a.state.data[:, g:-g, g:-g, g:-g], b.state.data[:, g:-g, g:-g, g:-g], 1)
                growth.append({"step": s, "max_rel_l1": float(l1[:5].max()), "max_rel_linf": float(li[:5].max())})
        out.append({"workload": f"turbulence_{n}^3_as_{box}^3_boxes_ns1_mach0.3", "scheme": "PPM" if ppm else "PLM",
                    "fp64_ms_per_step": ms_a, "mixed_ms_per_step": ms_b,
                    "fp64_cell_updates_per_s": lev0.ncells() / (ms_a / 1e3),
                    "mixed_cell_updates_per_s": lev0.ncells() / (ms_b / 1e3),
                    "speedup_mixed_over_fp64": ms_a / ms_b, "launch_tuning": tuned,
                    "error_components": "rho, rho u, rho v, rho w, rho E (per physical group)", "growth": growth})
        for prec, table in keep.items():
            for k, v in table.items():
                autotune.set_variant(prec, 1, k, v)
        a.close()
        b.close()
        del a, b
        torch.cuda.empty_cache()
    return out


def run_sweep(args):
    for r in sweep_workload(args.n, args.box, args.steps, args.every):
        print(json.dumps(r), flush=True)


def run_serve(args):
    from .serve import ensemble_serving

    out = ensemble_serving(wl.load_nasa7(), nruns=args.runs, per_run=args.per_run, nreq=args.requests,
                           budget_bytes=int(args.budget_gb * 1e9), loads=tuple(args.loads),
                           max_batch_cells=args.max_batch_cells, error_sample=args.error_sample,
                           max_inflight=args.max_inflight)
    for r in out["points"]:
        r.update({"workload": out["workload"], "budget_gb": args.budget_gb, "precision": "mixed"})
        print(json.dumps(r), flush=True)
    print(json.dumps({"serving_error_mixed_vs_fp64": out["error_vs_fp64_one_step"],
                      "resident_state_gb": out["resident_state_gb"]}), flush=True)


def run_options(args):
    """The 128^3 flame level step (FP64 per box as the drop-in, mixed fused, CUDA graphs)
    with the reference's remaining reconstruction and boundary options, and the single
    32^3 Sod box (one species) the same way."""
    import torch

    from .level import LevelStepper

    flame = f"flame_level_{args.n}^3_"
    cases = [(flame + "ppm", {}, False)] + [
        (flame + f"hybrid_weno_{n}", {"use_hybrid_weno": True, "weno_scheme": s}, False)
        for s, n in ((0, "js5"), (1, "z5"), (2, "z7"), (3, "z3"))] + [(flame + "ppm_inflow_zlo", {}, True),
                                                                      ("sod_32^3_one_box_ppm", {}, None)]
    g = abi.NGROW
    for name, kw, inflow in cases:
        lev = wl.sod(n=32) if inflow is None else wl.flame(n=args.n, box=args.box, seed=2)
        if inflow:
            lev.bclo = (lev.bclo[0], lev.bclo[1], abi.BC_INFLOW)
        ms, states = {}, {}
        for form, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
            st = LevelStepper(lev, precision=prec, fuse=prec == abi.PREC_MIXED, **kw)
            st.step()  # one step from the generated state, kept for the error
            torch.cuda.synchronize()
            states[form] = st.state.data[:, g:-g, g:-g, g:-g].clone()
            st.capture()
            ms[form] = _timed(torch, st.replay, args.steps, args.warmup)
            st.close()
            del st
            torch.cuda.empty_cache()
        l1, li = _rel_grouped(torch, states["fp64"], states["mixed"], lev.nspec)
        print(json.dumps({"workload": name, "fp64_ms_per_step": ms["fp64"],
                          "mixed_ms_per_step": ms["mixed"], "speedup_mixed_over_fp64": ms["fp64"] / ms["mixed"],
                          "mixed_cell_updates_per_s": lev.ncells() / (ms["mixed"] / 1e3),
                          "error_mixed_vs_fp64_one_step": {"max_rel_l1": float(l1.max()),
                                                           "max_rel_linf": float(li.max())}}), flush=True)
        del states


def run_step(args):
    """A few eager steps of one level (the profiling workload): the flame level of edge n
    (9 species) or the turbulence level (one species), one form."""
    import torch

    from .level import LevelStepper

    from . import autotune

    lev = wl.flame(n=args.n, box=args.box, seed=2) if args.level == "flame" else wl.turbulence(n=args.n, box=args.box)
    prec = {"mixed": abi.PREC_MIXED, "fp64": abi.PREC_FP64, "fast": abi.PREC_FP64_FAST}[args.form]
    for sv in args.variant:  # launch variants to profile, stage=variant (autotune.STAGE_NAMES)
        name, v = sv.split("=")
        autotune.set_variant(prec, lev.nspec, autotune.STAGE_NAMES.index(name), int(v))
    st = LevelStepper(lev, precision=prec, fuse=not args.per_box, ppm_type=args.ppm)
    for _ in range(args.steps):
        st.step()
    torch.cuda.synchronize()
    print(json.dumps({"level": args.level, "n": args.n, "form": args.form, "steps": args.steps,
                      "dt": float(st.dt.item())}), flush=True)
    st.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("batch")
    b.add_argument("--nbox", type=int, default=512)
    b.add_argument("--steps", type=int, default=10)
    b.add_argument("--warmup", type=int, default=3)
    s = sub.add_parser("sweep")
    s.add_argument("--n", type=int, default=256)
    s.add_argument("--box", type=int, default=64)
    s.add_argument("--steps", type=int, default=100)
    s.add_argument("--every", type=int, default=10)
    v = sub.add_parser("serve")
    v.add_argument("--runs", type=int, default=16)
    v.add_argument("--per-run", type=int, default=32)
    v.add_argument("--budget-gb", type=float, default=120.0)
    v.add_argument("--loads", type=float, nargs="*", default=[0.1, 0.25, 0.5, 0.75, 0.8, 0.9, 1.0])
    v.add_argument("--requests", type=int, default=5000, help="step requests per load point")
    v.add_argument("--max-batch-cells", type=int, default=500_000)
    v.add_argument("--max-inflight", type=int, default=3)
    v.add_argument("--error-sample", type=int, default=32)
    t = sub.add_parser("step")
    t.add_argument("--level", choices=("flame", "turbulence"), default="flame")
    t.add_argument("--n", type=int, default=64)
    t.add_argument("--box", type=int, default=32)
    t.add_argument("--form", choices=("mixed", "fp64", "fast"), default="mixed")
    t.add_argument("--variant", nargs="*", default=[], help="launch variants, e.g. trace=5")
    t.add_argument("--ppm", type=int, default=1)
    t.add_argument("--per-box", action="store_true", help="advance the boxes as separate regions")
    t.add_argument("--steps", type=int, default=2)
    o = sub.add_parser("options")
    o.add_argument("--n", type=int, default=128)
    o.add_argument("--box", type=int, default=32)
    o.add_argument("--steps", type=int, default=10)
    o.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args(argv)
    {"batch": run_batch, "sweep": run_sweep, "serve": run_serve, "options": run_options,
     "step": run_step}[args.cmd](args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
