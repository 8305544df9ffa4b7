"""GPU parity for the species counts other than 1 and 9 that the library is built for
(NUM_SPECIES is a compile-time constant of the reference's mechanism,
Source/IndexDefines.H:50-89; the build compiles kernels for a list of counts). Tables:
the synthetic NASA-7 mixtures of thermo.standin_mixture. Per count: one box through the
plain FP64 form bit for bit against the oracle, a batch of uneven boxes through the FMA
and mixed forms within their tolerances, and three level steps (ghost fill, CFL timestep,
hydro, the fused update with the FP64 Newton solve for T) against the oracle's level
loop."""
import numpy as np
import pytest

from common import FP64_TOL, MIXED_TOL, gpu_zeros, oracle, rel_err, rel_errors, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, thermo, workloads as wl

pytestmark = pytest.mark.gpu
BIG = 1 << 30


def _counts():
    hydro.init(0)
    return [n for n in hydro.species_counts() if n not in (1, 9)]


def _setup(nspec):
    eos = thermo.standin_mixture(nspec)
    hydro.init(0)
    hydro.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    return eos, o


def _prm(p, dt, nspec, prec=abi.PREC_FP64):
    return abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), precision_mode=prec)


def test_build_has_other_species_counts():
    assert _counts(), "the build holds kernels for 1 and 9 species only"


@pytest.mark.parametrize("nspec", [2, 3, 21])
def test_box_fp64_bitexact(nspec):
    if nspec not in _counts():
        pytest.skip(f"library built without {nspec} species")
    eos, o = _setup(nspec)
    for seed, edges, ppm in ((700, (12, 10, 9), 1), (701, (7, 5, 6), 0)):
        p = wl.random_patch(edges, seed + nspec, eos)
        dt = 0.3 * o.estdt(p.lo, p.hi, p.fab, p.dx)
        prm = _prm(p, dt, nspec)
        prm.ppm_type = ppm
        ref, _ = o.hydro_box(prm, p.lo, p.hi, p.fab)
        uin = to_gpu(p.fab)
        out = gpu_zeros(abi.nvar(nspec), p.lo, p.hi)
        hydro.hydro_box(prm, p.lo, p.hi, uin, out)
        np.testing.assert_array_equal(to_cpu(out), ref.data)


@pytest.mark.parametrize("nspec", [2, 3, 21])
def test_batch_fast_and_mixed(nspec):
    if nspec not in _counts():
        pytest.skip(f"library built without {nspec} species")
    eos, o = _setup(nspec)
    patches = [wl.random_patch(e, 720 + n + nspec, eos) for n, e in enumerate(((16, 12, 8), (5, 9, 7), (10, 10, 10)))]
    dts = [0.3 * o.estdt(p.lo, p.hi, p.fab, p.dx) for p in patches]
    refs = [o.hydro_box(_prm(p, dt, nspec), p.lo, p.hi, p.fab)[0].data for p, dt in zip(patches, dts)]
    for prec in (abi.PREC_FP64_FAST, abi.PREC_MIXED):
        boxes, keep, outs = [], [], []
        for p, dt in zip(patches, dts):
            uin = to_gpu(p.fab)
            out = gpu_zeros(abi.nvar(nspec), p.lo, p.hi)
            boxes.append(hydro.make_box(p.lo, p.hi, uin, out, p.dx, dt))
            keep.append(uin)
            outs.append(out)
        prm = abi.make_params((1, 1, 1), 0.0, nspec, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0),
                              precision_mode=prec)
        hydro.hydro_boxes(prm, boxes)
        for p, dt, ref, out in zip(patches, dts, refs, outs):
            got = to_cpu(out)
            if prec == abi.PREC_FP64_FAST:
                l1, linf = rel_err(got, ref)
                assert l1 <= FP64_TOL and linf <= FP64_TOL, (nspec, p.hi, l1, linf)
            else:
                # the mixed form's bound is on S_new = S_old + dt * hydro_source
                s_old = p.fab.view(p.lo, p.hi)
                l1, _ = rel_errors(s_old + dt * got, s_old + dt * ref, nspec)
                assert l1.max() <= MIXED_TOL, (nspec, p.hi, l1.max())


def _level(eos, seed):
    """A 16x12x8 level cut into four boxes (periodic x and y, outflow z) whose state is a
    random mixture patch."""
    p = wl.random_patch((16, 12, 8), seed, eos)
    boxes = [((0, 0, 0), (7, 5, 7)), ((8, 0, 0), (15, 5, 7)), ((0, 6, 0), (7, 11, 7)), ((8, 6, 0), (15, 11, 7))]
    lev = wl.Level(eos, p.dx, (0, 0, 0), (15, 11, 7), (0, 0, 2), (0, 0, 2), p.fab.data.copy(), boxes,
                   (True, True, False))
    lev.fill_ghosts()
    return lev


@pytest.mark.parametrize("nspec", [2, 3, 21])
def test_level_steps(nspec):
    """Three level steps (ghost fill, CFL timestep, hydro, S_new with the FP64 Newton
    solve for T, the fused step tail) with this many species: the plain FP64 form, per
    box and fused, equals the oracle's level loop bit for bit; the mixed form stays
    within its tolerance."""
    if nspec not in _counts():
        pytest.skip(f"library built without {nspec} species")
    from particleclem_b200.level import LevelStepper
    from test_gpu_batched import _oracle_steps

    eos, o = _setup(nspec)
    lev = _level(eos, 760 + nspec)
    ref_state, dts = _oracle_steps(lev, 3)
    for prec, fuse in ((abi.PREC_FP64, False), (abi.PREC_FP64, True), (abi.PREC_MIXED, True)):
        st = LevelStepper(lev, precision=prec, fuse=fuse)
        got_dts = []
        for _ in range(3):
            st.step()
            got_dts.append(float(st.dt.item()))
        st.fill()
        got = st.host_state()
        st.close()
        if prec == abi.PREC_FP64:
            assert got_dts == dts, (nspec, fuse, got_dts, dts)
            np.testing.assert_array_equal(got, ref_state)
        else:
            l1, _ = rel_errors(got, ref_state, nspec)
            assert l1.max() <= MIXED_TOL, (nspec, l1.max())
