"""GPU parity on degenerate and ragged inputs: boxes one or two cells thick in any
direction (face rows of length one or two, march chunks shorter than the march length,
a single cell), alone and batched with larger boxes, in the three precision forms; a
fused level one cell thick in z stepped against the oracle's level loop; an empty box
list."""
import numpy as np
import pytest

from common import FP64_TOL, MIXED_TOL, eos9, gpu_zeros, oracle, rel_err, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, workloads as wl
from particleclem_b200.level import LevelStepper
from test_gpu_batched import _oracle_steps

pytestmark = pytest.mark.gpu
BIG = 1 << 30
THIN = [(1, 1, 1), (1, 5, 3), (4, 1, 2), (2, 3, 1), (1, 2, 9), (2, 2, 2), (7, 6, 5)]


def _run_batch(nspec, prec, edges, seed):
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    hydro.init(0)
    hydro.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    patches = [wl.random_patch(e, seed + n, eos if nspec == 9 else None) for n, e in enumerate(edges)]
    nv = abi.nvar(nspec)
    boxes, ins, outs, dts = [], [], [], []
    for p in patches:
        dt = 0.3 * o.estdt(p.lo, p.hi, p.fab, p.dx)
        uin = to_gpu(p.fab)  # the descriptor holds a raw pointer: keep the tensor alive
        out = gpu_zeros(nv, p.lo, p.hi)
        boxes.append(hydro.make_box(p.lo, p.hi, uin, out, p.dx, dt))
        ins.append(uin)
        outs.append(out)
        dts.append(dt)
    prm = abi.make_params((1, 1, 1), 0.0, nspec, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0), precision_mode=prec)
    hydro.hydro_boxes(prm, boxes)
    return o, patches, dts, [to_cpu(x) for x in outs]


@pytest.mark.parametrize("nspec", [1, 9])
def test_thin_boxes_fp64_bitexact(nspec):
    o, patches, dts, got = _run_batch(nspec, abi.PREC_FP64, THIN, 500)
    for p, dt, g in zip(patches, dts, got):
        prm = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0))
        ref, _ = o.hydro_box(prm, p.lo, p.hi, p.fab)
        np.testing.assert_array_equal(g, ref.data)


@pytest.mark.parametrize("nspec", [1, 9])
def test_thin_boxes_fast_and_mixed(nspec):
    for prec in (abi.PREC_FP64_FAST, abi.PREC_MIXED):
        o, patches, dts, got = _run_batch(nspec, prec, THIN, 520)
        for p, dt, g in zip(patches, dts, got):
            prm = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0))
            ref, _ = o.hydro_box(prm, p.lo, p.hi, p.fab)
            if prec == abi.PREC_FP64_FAST:
                l1, linf = rel_err(g, ref.data)
                assert l1 <= FP64_TOL and linf <= FP64_TOL, (p.hi, l1, linf)
            else:
                s_ref = o.update_state(p.lo, p.hi, p.fab, ref, dt)
                s_got = o.update_state(p.lo, p.hi, p.fab, abi.Fab(g, tuple(p.lo)), dt)
                l1, _ = rel_err(s_got.view(p.lo, p.hi), s_ref.view(p.lo, p.hi))
                assert l1 <= MIXED_TOL, (p.hi, l1)


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_level_one_cell_thick(prec):
    """A 12x8x1 level (periodic x and y, outflow z) in boxes of 4x8x1 and 8x8x1, fused into
    one region, three steps against the oracle's level loop."""
    p = wl.random_patch((12, 8, 1), 77)
    lev = wl.Level(wl.GammaLaw(), p.dx, (0, 0, 0), (11, 7, 0), (abi.BC_INTERIOR, abi.BC_INTERIOR, abi.BC_OUTFLOW),
                   (abi.BC_INTERIOR, abi.BC_INTERIOR, abi.BC_OUTFLOW), p.fab.data.copy(),
                   [((0, 0, 0), (3, 7, 0)), ((4, 0, 0), (11, 7, 0))], (True, True, False))
    ref_state, dts = _oracle_steps(lev, 3)
    st = LevelStepper(lev, precision=prec, fuse=True)
    got_dts = []
    for _ in range(3):
        st.step()
        got_dts.append(float(st.dt.item()))
    st.fill()
    got = st.host_state()
    if prec == abi.PREC_FP64:
        assert got_dts == dts
        np.testing.assert_array_equal(got, ref_state)
    else:
        l1, _ = rel_err(got, ref_state)
        assert l1 <= MIXED_TOL, l1
    st.close()


def test_empty_box_list_is_a_no_op():
    hydro.init(0)
    hydro.set_eos(wl.GammaLaw())
    prm = abi.make_params((1, 1, 1), 0.0, 1, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0))
    hydro.hydro_boxes(prm, [])
