"""GPU tests of pcg_step_boxes: one full step of independent patches, each its own domain
with its own timestep (the step the serving loop runs per request).

Per patch the oracle does what PeleC's level advance does around construct_hydro_source
for a one-box level (Source/Advance.cpp:266-352): fill the ghost cells (zero-gradient at
outflow faces, Source/Advance.cpp:307-309), construct_hydro_source with the patch's dt,
S_new = S_old + dt * hydro_source with computeTemp (Source/Advance.cpp:397-417,
Source/PeleC.cpp:2289-2305), and the next CFL timestep of S_new (Source/PeleC.cpp:829-960).
The plain FP64 form must reproduce it bit for bit over two consecutive steps, the second
taking the device's own next timestep; a patch stepped alone and inside a batch of others
must give the same state bit for bit in every form.
"""
import numpy as np
import pytest

from common import MIXED_TOL, eos9, oracle, rel_err
from particleclem_b200 import abi, hydro, workloads as wl

pytestmark = pytest.mark.gpu
EDGES = [(8, 12, 6), (16, 8, 8), (5, 7, 11), (12, 12, 12)]
OUTFLOW = (abi.BC_OUTFLOW,) * 3


def _patches(seed, edges=EDGES):
    eos = eos9()
    return [wl.flame_patch(e, seed + k, eos) for k, e in enumerate(edges)], eos


def _oracle_step(o, p, fab, dt):
    """One step of patch p (state FAB fab, ghosts included) on the CPU oracle."""
    data = fab.data.copy()
    wl.fill_ghosts(data, (False, False, False))
    f = abi.Fab(data, fab.lo)
    prm = abi.make_params(p.dx, dt, 9, p.lo, p.hi, OUTFLOW, OUTFLOW)
    hs, _ = o.hydro_box(prm, p.lo, p.hi, f)
    upd = o.update_state(p.lo, p.hi, f, hs, dt)
    sn = abi.Fab(data.copy(), fab.lo)  # ghost cells as filled, valid cells updated
    sn.view(p.lo, p.hi)[:] = upd.view(p.lo, p.hi)
    return sn, 0.3 * o.estdt(p.lo, p.hi, sn, p.dx)


def _device(patches, prec):
    import torch

    states = [abi.Fab(torch.from_numpy(np.ascontiguousarray(p.fab.data)).cuda(), tuple(p.fab.lo)) for p in patches]
    boxes = [hydro.make_box(p.lo, p.hi, s, None, p.dx, 0.0, p.lo, p.hi, OUTFLOW, OUTFLOW)
             for p, s in zip(patches, states)]
    prm = abi.make_params((1, 1, 1), 0.0, 9, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0), precision_mode=prec)
    return states, boxes, prm


def test_step_boxes_fp64_equals_oracle_over_two_steps():
    import torch

    patches, eos = _patches(300)
    hydro.init(0)
    hydro.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    states, boxes, prm = _device(patches, abi.PREC_FP64)
    # each patch its own first timestep: the CFL of its filled initial state, scaled per patch
    cpu = [abi.Fab(p.fab.data.copy(), p.fab.lo) for p in patches]
    for f in cpu:
        wl.fill_ghosts(f.data, (False, False, False))
    dts = [(0.2 + 0.05 * k) * o.estdt(p.lo, p.hi, f, p.dx) for k, (p, f) in enumerate(zip(patches, cpu))]
    dt = torch.tensor(dts, dtype=torch.float64, device="cuda")
    dt_next = torch.zeros_like(dt)
    for step in range(2):
        hydro.step_boxes(prm, boxes, 0.3, dt, dt_next)
        torch.cuda.synchronize()
        got_dt = dt_next.cpu().numpy()
        for k, p in enumerate(patches):
            sn, dtn = _oracle_step(o, p, cpu[k], float(dt[k].item()))
            got = abi.Fab(states[k].data.cpu().numpy(), states[k].lo)
            np.testing.assert_array_equal(got.view(p.lo, p.hi), sn.view(p.lo, p.hi))
            assert got_dt[k] == dtn, (step, k, got_dt[k], dtn)
            cpu[k] = abi.Fab(got.data.copy(), got.lo)
        dt.copy_(dt_next)


def test_step_boxes_mixed_within_tolerance():
    import torch

    patches, eos = _patches(320)
    hydro.init(0)
    hydro.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    states, boxes, prm = _device(patches, abi.PREC_MIXED)
    cpu = [abi.Fab(p.fab.data.copy(), p.fab.lo) for p in patches]
    for f in cpu:
        wl.fill_ghosts(f.data, (False, False, False))
    dts = [0.3 * o.estdt(p.lo, p.hi, f, p.dx) for p, f in zip(patches, cpu)]
    dt = torch.tensor(dts, dtype=torch.float64, device="cuda")
    dt_next = torch.zeros_like(dt)
    hydro.step_boxes(prm, boxes, 0.3, dt, dt_next)
    torch.cuda.synchronize()
    for k, p in enumerate(patches):
        sn, dtn = _oracle_step(o, p, cpu[k], dts[k])
        got = abi.Fab(states[k].data.cpu().numpy(), states[k].lo)
        l1, _ = rel_err(got.view(p.lo, p.hi), sn.view(p.lo, p.hi))
        assert l1 <= MIXED_TOL, (k, l1)
        assert abs(float(dt_next[k].item()) - dtn) <= 1e-6 * dtn


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP64_FAST, abi.PREC_MIXED])
def test_patch_alone_equals_patch_in_a_batch(prec):
    import torch

    patches, eos = _patches(340)
    hydro.init(0)
    hydro.set_eos(eos)
    s_all, b_all, prm = _device(patches, prec)
    s_one, b_one, _ = _device(patches[2:3], prec)
    dt_all = torch.full((len(patches),), 1e-8, dtype=torch.float64, device="cuda")
    dt_one = dt_all[2:3].clone()
    dn_all, dn_one = torch.zeros_like(dt_all), torch.zeros_like(dt_one)
    for _ in range(3):  # three evolving steps, each with the patch's own next timestep
        hydro.step_boxes(prm, b_all, 0.3, dt_all, dn_all)
        hydro.step_boxes(prm, b_one, 0.3, dt_one, dn_one)
        dt_all.copy_(dn_all)
        dt_one.copy_(dn_one)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(s_all[2].data.cpu().numpy(), s_one[0].data.cpu().numpy())
    assert float(dn_all[2].item()) == float(dn_one[0].item())
