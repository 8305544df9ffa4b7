"""GPU parity of the PPM trace with hybrid-WENO edge values (use_hybrid_weno,
Source/PPM.cpp:120-172, Source/WENO.H) for the four schemes: plain FP64 bit-identical to
the oracle (itself pinned to the reference build), FMA and mixed forms within tolerance,
including the 7-point scheme whose FP32 primitive copy covers grow(box,4), through
pcg_hydro_box, pcg_umdrv (caller q) and a fused level plan."""
import numpy as np
import pytest

from common import FP64_TOL, MIXED_TOL, eos9, gpu_zeros, oracle, rel_err, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, workloads as wl
from particleclem_b200.level import LevelStepper

pytestmark = pytest.mark.gpu
BIG = 1 << 30


def _prm(p, dt, nspec, scheme, prec):
    prm = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=1,
                          precision_mode=prec)
    prm.use_hybrid_weno = 1
    prm.weno_scheme = scheme
    return prm


def _case(nspec, seed=501):
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    hydro.init(0)
    hydro.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    p = wl.random_patch((10, 7, 8), seed, eos if nspec == 9 else None)
    return p, o, 0.3 * o.estdt(p.lo, p.hi, p.fab, p.dx)


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
@pytest.mark.parametrize("nspec", [1, 9])
def test_hybrid_weno_fp64_bitexact(scheme, nspec):
    p, o, dt = _case(nspec)
    prm = _prm(p, dt, nspec, scheme, abi.PREC_FP64)
    ref, ref_flx = o.hydro_box(prm, p.lo, p.hi, p.fab)
    nv = abi.nvar(nspec)
    uout = gpu_zeros(nv, p.lo, p.hi)
    flx = [gpu_zeros(nv, *abi.nodes(p.lo, p.hi, d)) for d in range(3)]
    hydro.hydro_box(prm, p.lo, p.hi, to_gpu(p.fab), uout, flx)
    np.testing.assert_array_equal(to_cpu(uout), ref.data)
    for d in range(3):
        np.testing.assert_array_equal(to_cpu(flx[d]), ref_flx[d].data)


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
@pytest.mark.parametrize("nspec", [1, 9])
def test_hybrid_weno_fast_and_mixed(scheme, nspec):
    p, o, dt = _case(nspec)
    nv = abi.nvar(nspec)
    ref, _ = o.hydro_box(_prm(p, dt, nspec, scheme, abi.PREC_FP64), p.lo, p.hi, p.fab)
    for prec in (abi.PREC_FP64_FAST, abi.PREC_MIXED):
        uout = gpu_zeros(nv, p.lo, p.hi)
        hydro.hydro_box(_prm(p, dt, nspec, scheme, prec), p.lo, p.hi, to_gpu(p.fab), uout)
        got = to_cpu(uout)
        if prec == abi.PREC_FP64_FAST:
            l1, linf = rel_err(got, ref.data)
            assert l1 <= FP64_TOL and linf <= FP64_TOL, (l1, linf)
        else:
            s_ref = o.update_state(p.lo, p.hi, p.fab, ref, dt)
            s_got = o.update_state(p.lo, p.hi, p.fab, abi.Fab(got, tuple(p.lo)), dt)
            l1, _ = rel_err(s_got.view(p.lo, p.hi), s_ref.view(p.lo, p.hi))
            assert l1 <= MIXED_TOL, l1


def test_hybrid_weno7_mixed_umdrv_with_caller_q():
    """pcg_umdrv with the caller's q: the FP32 copy is made by k_prep over grow(box,4)."""
    p, o, dt = _case(9, 503)
    lo, hi = p.lo, p.hi
    g4lo, g4hi = abi.grow(lo, hi, 4)
    q_ref, qa_ref = o.ctoprim(g4lo, g4hi, p.fab)
    nv = abi.nvar(9)
    ref, _ = o.hydro_box(_prm(p, dt, 9, 2, abi.PREC_FP64), lo, hi, p.fab)
    import pyoracle

    area, vol = pyoracle.uniform_geometry(lo, hi, p.dx)
    uout = gpu_zeros(nv, lo, hi)
    flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
    hydro.umdrv(_prm(p, dt, 9, 2, abi.PREC_MIXED), lo, hi, to_gpu(p.fab), uout, to_gpu(q_ref), to_gpu(qa_ref), None,
                flx, [to_gpu(a) for a in area], to_gpu(vol))
    s_ref = o.update_state(lo, hi, p.fab, ref, dt)
    s_got = o.update_state(lo, hi, p.fab, abi.Fab(to_cpu(uout), tuple(lo)), dt)
    l1, _ = rel_err(s_got.view(lo, hi), s_ref.view(lo, hi))
    assert l1 <= MIXED_TOL, l1


@pytest.mark.parametrize("scheme", [2, 1])
def test_hybrid_weno_fused_level_mixed_vs_fp64(scheme):
    lev = wl.flame(n=16, box=8)
    out = []
    for prec, fuse in ((abi.PREC_FP64, False), (abi.PREC_MIXED, True)):
        st = LevelStepper(lev, precision=prec, fuse=fuse)
        st.prm.use_hybrid_weno = 1
        st.prm.weno_scheme = scheme
        st.plan.close()
        st.plan = hydro.Plan(st.prm, st.boxes, fuse=fuse)
        st.step()
        out.append(st.host_state()[:, 4:-4, 4:-4, 4:-4])
        st.close()
    l1, _ = rel_err(out[1], out[0])
    assert l1 <= MIXED_TOL, l1
