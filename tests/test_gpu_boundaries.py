"""GPU parity on boxes whose faces are domain boundaries: the Riemann boundary overrides
of pc_cmpflx for walls, symmetry and outflow, and the low-order recomputation of inflow /
user_bc faces (pc_low_order_boundary, Source/Godunov.cpp:6-55, :440-468), in the three
precision forms; and a level whose low z face is an inflow, stepped as fused and per-box
plans, against the oracle's level loop."""
import numpy as np
import pytest

from common import FP64_TOL, MIXED_TOL, eos9, gpu_zeros, oracle, rel_err, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, workloads as wl
from particleclem_b200.level import LevelStepper
from test_gpu_batched import _oracle_steps

pytestmark = pytest.mark.gpu

BCS = {
    "inflow_lo_outflow_hi": ((1, 0, 0), (2, 0, 0)),
    "user_hi_walls": ((4, 3, 0), (6, 5, 0)),
    "inflow_everywhere": ((1, 1, 1), (1, 6, 1)),
}


def _run(prec, bc, nspec, ppm):
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    hydro.init(0)
    hydro.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    p = wl.random_patch((9, 7, 6), 311, eos if nspec == 9 else None)
    dt = 0.3 * o.estdt(p.lo, p.hi, p.fab, p.dx)
    bclo, bchi = BCS[bc]
    prm = abi.make_params(p.dx, dt, nspec, p.lo, p.hi, bclo, bchi, ppm_type=ppm, precision_mode=prec)
    ref, ref_flx = o.hydro_box(prm, p.lo, p.hi, p.fab)
    nv = abi.nvar(nspec)
    uout = gpu_zeros(nv, p.lo, p.hi)
    flx = [gpu_zeros(nv, *abi.nodes(p.lo, p.hi, d)) for d in range(3)]
    hydro.hydro_box(prm, p.lo, p.hi, to_gpu(p.fab), uout, flx)
    return p, o, dt, ref, ref_flx, to_cpu(uout), [to_cpu(f) for f in flx]


@pytest.mark.parametrize("bc", sorted(BCS))
@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("ppm", [1, 0])
def test_domain_boundaries_fp64_bitexact(bc, nspec, ppm):
    _, _, _, ref, ref_flx, got, got_flx = _run(abi.PREC_FP64, bc, nspec, ppm)
    np.testing.assert_array_equal(got, ref.data)
    for d in range(3):
        np.testing.assert_array_equal(got_flx[d], ref_flx[d].data)


@pytest.mark.parametrize("bc", sorted(BCS))
@pytest.mark.parametrize("nspec", [1, 9])
def test_domain_boundaries_fast_and_mixed(bc, nspec):
    _, _, _, ref, _, got, _ = _run(abi.PREC_FP64_FAST, bc, nspec, 1)
    l1, linf = rel_err(got, ref.data)
    assert l1 <= FP64_TOL and linf <= FP64_TOL, (l1, linf)
    p, o, dt, ref, _, got, _ = _run(abi.PREC_MIXED, bc, nspec, 1)
    s_ref = o.update_state(p.lo, p.hi, p.fab, ref, dt)
    s_got = o.update_state(p.lo, p.hi, p.fab, abi.Fab(got, tuple(p.lo)), dt)
    l1, _ = rel_err(s_got.view(p.lo, p.hi), s_ref.view(p.lo, p.hi))
    assert l1 <= MIXED_TOL, l1


@pytest.mark.parametrize("fuse", [False, True])
def test_level_with_inflow_face_equals_oracle(fuse):
    """The flame level with its low z face an inflow (ghost cells hold the given inflow
    state: here the zero-gradient fill of the generator) for three steps."""
    lev = wl.flame(n=16, box=8)
    lev.bclo = (lev.bclo[0], lev.bclo[1], abi.BC_INFLOW)
    ref_state, dts = _oracle_steps(lev, 3)
    st = LevelStepper(lev, precision=abi.PREC_FP64, fuse=fuse)
    got_dts = []
    for _ in range(3):
        st.step()
        got_dts.append(float(st.dt.item()))
    st.fill()
    assert got_dts == dts
    np.testing.assert_array_equal(st.host_state(), ref_state)
    st.close()
