"""GPU tests of the batched box advance and of the serving loop: a batch of uneven
independent flame boxes advanced one step (CFL dt over the batch, hydro, update with the
T(e) Newton solve) equals the oracle in the plain FP64 form; a patch stepped by requests
served alone and by the same requests inside a mix of others ends in the same state bit
for bit, in every precision form; eviction of resident states under a small budget does
not change results; a short serving sweep keeps its HBM budget."""
import numpy as np
import pytest

from common import eos9, oracle
from particleclem_b200 import abi, workloads as wl
from particleclem_b200.batch import BoxBatch
from particleclem_b200.serve import GpuExecutor, Scheduler, serve_sweep

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
    """Three steps of one patch served alone, and the same three steps served inside a mix
    of requests for other patches (batched with them, two streams, the patch's steps in
    order), leave the patch in the same state bit for bit: the states evolve, and nothing
    couples the boxes of a batch. In the plain FP64 form the steps equal the oracle's."""
    patches, eos = _patches(EDGES, 110)
    solo = GpuExecutor(eos, precision=prec)
    p_solo = solo.add_patch(patches[3])
    solo.start()
    Scheduler(solo, 10**10).run([solo.request(k, p_solo, 0.0) for k in range(3)])
    alone = solo.state(p_solo)
    ex = GpuExecutor(eos, precision=prec)
    pids = [ex.add_patch(p) for p in patches]
    ex.start()
    order = [1, 3, 0, 5, 3, 2, 4, 1, 3, 0]  # patch 3 three times, interleaved with others
    sch = Scheduler(ex, 10**10)
    sch.run([ex.request(k, pids[q], 1e-4 * k) for k, q in enumerate(order)])
    np.testing.assert_array_equal(ex.state(pids[3]), alone)
    if prec == abi.PREC_FP64:
        from test_gpu_step_boxes import _oracle_step

        o = oracle()
        o.set_eos(eos)
        p = patches[3]
        f = abi.Fab(p.fab.data.copy(), p.fab.lo)
        for _ in range(3):
            g = abi.Fab(f.data.copy(), f.lo)
            wl.fill_ghosts(g.data, (False, False, False))
            dt = 0.3 * o.estdt(p.lo, p.hi, g, p.dx) if _ == 0 else dtn
            f, dtn = _oracle_step(o, p, f, dt)
        np.testing.assert_array_equal(abi.Fab(alone, f.lo).view(p.lo, p.hi), f.view(p.lo, p.hi))


def test_eviction_under_a_small_budget_does_not_change_results():
    """The same request sequence under a budget that holds every state and under one that
    holds about two (idle states go back to host memory and return on their next request)
    gives the same patch states bit for bit, and the small budget is never exceeded."""
    patches, eos = _patches(EDGES, 120)
    order = [0, 1, 2, 3, 4, 5, 0, 2, 4, 1, 3, 5, 0]
    finals = []
    for small in (False, True):
        ex = GpuExecutor(eos, precision=abi.PREC_MIXED)
        pids = [ex.add_patch(p) for p in patches]
        big = max(ex.nbytes[q] + ex.state_nbytes[q] for q in pids)
        budget = 2 * big + max(ex.state_nbytes) if small else 10**11
        ex.start()
        sch = Scheduler(ex, budget, max_inflight=2)
        sch.run([ex.request(k, pids[q], 2e-4 * k) for k, q in enumerate(order)])
        assert sch.peak_bytes <= budget
        if small:
            assert sch.evictions > 0
        finals.append([ex.state(q) for q in pids])
    for a, b in zip(*finals):
        np.testing.assert_array_equal(a, b)


def test_serving_sweep_respects_budget():
    patches, eos = _patches(EDGES * 3, 130)
    ex = GpuExecutor(eos, precision=abi.PREC_MIXED)
    pids = [ex.add_patch(p) for p in patches]
    budget = 3 * max(w + s for w, s in zip(ex.nbytes, ex.state_nbytes))
    res = serve_sweep(ex, pids, budget, loads=(0.5, 0.8), nreq=60)
    assert [r["load"] for r in res] == ["saturated", 0.5, 0.8]
    for r in res:
        assert r["requests"] == 60 and 0 < r["p50_ms"] <= r["p99_ms"] and r["peak_bytes"] <= budget


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
