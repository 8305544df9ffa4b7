"""GPU tests of the batched box advance and of the serving loop: a batch of uneven
independent flame boxes advanced one step (CFL dt over the batch, hydro, update with the
T(e) Newton solve) equals the oracle in the plain FP64 form; a request served alone and
the same request served inside a mix of other requests give the same hydro source bit for
bit, in every precision form; a short serving sweep keeps its HBM budget."""
import numpy as np
import pytest

from common import eos9, oracle
from particleclem_b200 import abi, workloads as wl
from particleclem_b200.batch import BoxBatch
from particleclem_b200.serve import GpuExecutor, Request, Scheduler, serve_sweep

pytestmark = pytest.mark.gpu

EDGES = [(8, 12, 6), (16, 8, 8), (5, 7, 11), (12, 12, 12), (9, 16, 4), (6, 6, 20)]


def _patches(edges, seed):
    eos = eos9()
    return [wl.flame_patch(e, seed + k, eos) for k, e in enumerate(edges)], eos


def test_box_batch_step_fp64_equals_oracle():
    patches, eos = _patches(EDGES, 70)
    bb = BoxBatch(patches, eos, precision=abi.PREC_FP64, cfl=0.3)
    bb.step()
    o = oracle()
    o.set_eos(eos)
    dt = 0.3 * min(o.estdt(p.lo, p.hi, p.fab, p.dx) for p in patches)
    assert float(bb.dt.item()) == dt
    for p, st in zip(patches, bb.states):
        prm = abi.make_params(p.dx, dt, 9, (-(1 << 30),) * 3, ((1 << 30),) * 3, (0, 0, 0), (0, 0, 0))
        hs, _ = o.hydro_box(prm, p.lo, p.hi, p.fab)
        sn = o.update_state(p.lo, p.hi, p.fab, hs, dt)
        got = st.data.cpu().numpy()
        np.testing.assert_array_equal(abi.Fab(got, st.lo).view(p.lo, p.hi), sn.view(p.lo, p.hi))
    bb.close()


def test_box_batch_graph_replay_equals_eager():
    patches, eos = _patches(EDGES[:4], 90)
    a = BoxBatch(patches, eos, precision=abi.PREC_MIXED)
    b = BoxBatch(patches, eos, precision=abi.PREC_MIXED)
    a.capture()  # runs one eager step before capturing
    b.step()
    a.replay()
    b.step()
    for x, y in zip(a.states, b.states):
        np.testing.assert_array_equal(x.data.cpu().numpy(), y.data.cpu().numpy())
    a.close()
    b.close()


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP64_FAST, abi.PREC_MIXED])
def test_request_alone_equals_request_in_a_mix(prec):
    patches, eos = _patches(EDGES, 110)
    ex = GpuExecutor(eos, precision=prec)
    pids = [ex.add_patch(p) for p in patches]
    budget = 10 * max(ex.nbytes)
    ex.start()
    Scheduler(ex, budget).run([ex.request(0, pids[3], 0.0)])
    ex.synchronize()
    alone = ex.outs[pids[3]].data.clone()
    ex.outs[pids[3]].data.zero_()
    ex.start()
    mix = [ex.request(k, pid, 0.0) for k, pid in enumerate([pids[1], pids[3], pids[0], pids[5], pids[2]])]
    sch = Scheduler(ex, budget)
    sch.run(mix)
    ex.synchronize()
    assert sch.nbatches == 1
    assert bool((alone == ex.outs[pids[3]].data).all())
    if prec == abi.PREC_FP64:
        o = oracle()
        o.set_eos(eos)
        p = patches[3]
        prm = abi.make_params(p.dx, ex.boxes[pids[3]].dt, 9, (-(1 << 30),) * 3, ((1 << 30),) * 3, (0, 0, 0),
                              (0, 0, 0))
        hs, _ = o.hydro_box(prm, p.lo, p.hi, p.fab)
        np.testing.assert_array_equal(alone.cpu().numpy(), hs.data)


def test_serving_sweep_respects_budget():
    patches, eos = _patches(EDGES * 3, 130)
    ex = GpuExecutor(eos, precision=abi.PREC_MIXED)
    pids = [ex.add_patch(p) for p in patches]
    budget = 3 * max(ex.nbytes)
    res = serve_sweep(ex, pids, budget, loads=(0.5,))
    assert [r["load"] for r in res] == ["saturated", 0.5]
    for r in res:
        assert r["requests"] == len(pids) and 0 < r["p50_ms"] <= r["p99_ms"] and r["peak_bytes"] <= budget


def test_box_batch_fused_tail_equals_separate_passes_fp64():
    """Three steps of an uneven batch with the fused step tail (the update pass forms
    the batch's next CFL minimum) equal the separate CFL, hydro and update passes bit for
    bit in the plain FP64 form, eager and graph-replayed."""
    patches, eos = _patches(EDGES[:4], 150)
    a = BoxBatch(patches, eos, precision=abi.PREC_FP64)
    b = BoxBatch(patches, eos, precision=abi.PREC_FP64, fused_tail=False)
    c = BoxBatch(patches, eos, precision=abi.PREC_FP64)
    c.capture()  # one eager step before capturing
    for k in range(3):
        a.step()
        b.step()
        if k == 0:
            continue
        c.replay()
        assert float(a.dt.item()) == float(b.dt.item())
    for x, y in zip(a.states, b.states):
        np.testing.assert_array_equal(x.data.cpu().numpy(), y.data.cpu().numpy())
    for x, y in zip(a.states, c.states):
        np.testing.assert_array_equal(x.data.cpu().numpy(), y.data.cpu().numpy())
    for s in (a, b, c):
        s.close()
