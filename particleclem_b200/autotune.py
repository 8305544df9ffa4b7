"""Launch-shape autotuner for the hydro stages.

Every heavy stage (ctoprim, trace, the three Riemann stages, and the fused step tail
that the consup slot selects for ``pcg_plan_advance``) is compiled in three register
budgets (``kMinBlocks`` in csrc/pcg_kernels.cuh: no cap, moderate, tight),
which trades registers per thread against resident warps per SM; the trace of the
mixed form also exists as the TMA-staged tiled trace in the same three budgets
(variants 3-5). The best choice
depends on the precision form (FP32 or FP64 arithmetic), the species count and the GPU,
so it is measured: :func:`tune` runs each variant of each stage on a live plan with
CUDA events, keeps the fastest, installs it with ``pcg_set_launch_variant`` and
returns the table, which :func:`save` / :func:`load` persist as JSON.
"""
from __future__ import annotations

import json
import os

from . import native

TUNED_STAGES = (0, 2, 3, 4, 5)  # ctoprim, trace, flux0, flux1, flux2
STAGE_NAMES = ("ctoprim", "prep", "trace", "flux0", "flux1", "flux2", "consup")
TAIL_STAGE = 6  # the consup slot: its variant selects the fused step tail's register cap
NVARIANT = 3
TRACE_STAGE = 2
TILED_TRACE_VARIANTS = 6  # the mixed form's trace: 0-2 untiled, 3-5 TMA-staged tiles


def n_variants(prec, stage):
    return TILED_TRACE_VARIANTS if (prec == 2 and stage == TRACE_STAGE) else NVARIANT


CAPS = ("no register cap", "moderate register cap", "tight register cap")


def describe(prec, stage, variant):
    """What launch variant ``variant`` of ``stage`` is: its register budget, and for the
    mixed form's trace whether it runs on TMA-staged tiles (32 x 4 cells per block for
    the x and y traces, 32 x 1 x 4 for z) or one cell per thread from global memory."""
    if stage == TRACE_STAGE and prec == 2:
        shape = "TMA-staged tiles" if variant >= NVARIANT else "cell per thread"
        return f"{shape}, {CAPS[variant % NVARIANT]}"
    return CAPS[variant]


def get_variant(prec, nspec, stage):
    v = native.load().pcg_get_launch_variant(int(prec), int(nspec), int(stage))
    if v < 0:
        raise native.PcgError("pcg_get_launch_variant", v, native.load().pcg_last_error().decode())
    return v


def set_variant(prec, nspec, stage, variant):
    native.call("pcg_set_launch_variant", int(prec), int(nspec), int(stage), int(variant))


def tune(plan, dt_dev=None, reps=5, stages=TUNED_STAGES, state=None):
    """Time every variant of ``stages`` on ``plan`` (a hydro.Plan whose workspace holds
    a valid state; stages before each tuned one are run once first) and install the
    fastest. With ``state`` (the device tensor, or list of tensors, the plan's boxes
    update) the fused step tail is tuned too: whole ``plan.advance`` calls per variant,
    the state restored afterwards. Returns {stage_name: {"variant": v, "ms": [ms per variant]}}."""
    import torch

    prec, ns = plan.prm.precision_mode, plan.prm.nspec
    plan.hydro(dt_dev)  # fills every intermediate
    torch.cuda.synchronize()
    result = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    states = [] if state is None else list(state) if isinstance(state, (list, tuple)) else [state]
    if states:
        stages = tuple(stages) + (TAIL_STAGE,)
        saved = [s.clone() for s in states]
        dt_next = torch.zeros(1, dtype=torch.float64, device=states[0].device)
    for st in stages:
        times = []
        nv = n_variants(prec, st)
        for v in range(nv):
            set_variant(prec, ns, st, v)
            if st == TAIL_STAGE:
                run = lambda: plan.advance(1.0, dt_dev, dt_next)  # noqa: E731
            else:
                run = lambda: plan.stages(st, st, dt_dev)  # noqa: E731
            run()  # warm
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / reps)
            if st == TAIL_STAGE:
                for s, v0 in zip(states, saved):
                    s.copy_(v0)
        best = min(range(nv), key=lambda v: times[v])
        set_variant(prec, ns, st, best)
        result[STAGE_NAMES[st]] = {"variant": best, "shape": describe(prec, st, best),
                                   "ms": [round(t, 4) for t in times]}
    return result


def save(path, prec, nspec, table, gpu_name=None):
    data = json.load(open(path)) if os.path.exists(path) else {}
    data[f"prec{prec}_ns{nspec}"] = {"gpu": gpu_name, "stages": table}
    with open(path, "w") as f:
        json.dump(data, f, indent=1)


def load(path):
    """Install every table of a JSON file written by :func:`save`."""
    data = json.load(open(path))
    for key, entry in data.items():
        prec = int(key.split("_")[0][4:])
        ns = int(key.split("_")[1][2:])
        for name, rec in entry["stages"].items():
            set_variant(prec, ns, STAGE_NAMES.index(name), rec["variant"])
    return data
