"""GPU parity of the hydro path against the CPU FP64 oracle, through the C ABI.

The plain FP64 form (PCG_PREC_FP64: reference operation order, no FMA contraction)
must reproduce the oracle bit for bit; the FMA form must stay within 1e-12 relative
L1/Linf per conserved component; the mixed form within 1e-6 relative L1 on the updated
state. Cases follow the reference's Godunov regression inputs: Sod with PPM
(Exec/RegTests/Sod/sod-2.inp), PLM defaults (plm_iorder 4), outflow boundaries, and the
9-species mixture EOS, plus generic random states with a pressure jump so every
limiter, flattening and Riemann branch is visited.
"""
import numpy as np
import pytest

from common import FP64_TOL, MIXED_TOL, eos9, gpu_zeros, np_zeros, oracle, params_for, rel_err, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, workloads as wl

pytestmark = pytest.mark.gpu


def _setup(eos):
    hydro.init(0)
    hydro.set_eos(eos)
    oracle().set_eos(eos)


def _gpu_hydro_box(prm, lo, hi, uin_fab, with_flx=True):
    nv = abi.nvar(prm.nspec)
    uin = to_gpu(uin_fab)
    uout = gpu_zeros(nv, lo, hi)
    flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)] if with_flx else None
    hydro.hydro_box(prm, lo, hi, uin, uout, flx)
    return to_cpu(uout), ([to_cpu(f) for f in flx] if with_flx else None)


def _dt(fab, lo, hi, dx, cfl=0.3):
    return cfl * oracle().estdt(lo, hi, fab, dx)


CASES = [
    ("sod", 1, 4),
    ("random_gamma", 1, 4),
    ("random_gamma", 0, 4),
    ("random_gamma", 0, 2),
    ("random_nasa7", 1, 4),
    ("random_nasa7", 0, 4),
    ("flame", 1, 4),
]


def _case(name):
    if name == "sod":
        lev = wl.sod(16)
        lo, hi = lev.boxes[0]
        return lev, lo, hi, lev.box_fab(lo, hi), lev.eos
    if name == "flame":
        lev = wl.flame(n=16, box=16)
        lo, hi = lev.boxes[0]
        return lev, lo, hi, lev.box_fab(lo, hi), lev.eos
    if name == "random_gamma":
        p = wl.random_patch((11, 9, 7), 5)
        return p, p.lo, p.hi, p.fab, wl.GammaLaw()
    p = wl.random_patch((9, 7, 6), 6, eos9())
    return p, p.lo, p.hi, p.fab, eos9()


@pytest.mark.parametrize("name,ppm,order", CASES)
def test_hydro_box_fp64_bitexact(name, ppm, order):
    src, lo, hi, uin, eos = _case(name)
    _setup(eos)
    dt = _dt(uin, lo, hi, src.dx)
    prm = params_for(src, dt, ppm_type=ppm, plm_iorder=order, nspec=eos.nspec)
    ref_out, ref_flx = oracle().hydro_box(prm, lo, hi, uin)
    got_out, got_flx = _gpu_hydro_box(prm, lo, hi, uin)
    assert np.isfinite(got_out).all()
    np.testing.assert_array_equal(got_out, ref_out.data)
    for d in range(3):
        np.testing.assert_array_equal(got_flx[d], ref_flx[d].data)


@pytest.mark.parametrize("name,ppm,order", CASES)
def test_hydro_box_fp64_fast_within_tolerance(name, ppm, order):
    src, lo, hi, uin, eos = _case(name)
    _setup(eos)
    dt = _dt(uin, lo, hi, src.dx)
    prm = params_for(src, dt, ppm_type=ppm, plm_iorder=order, prec=abi.PREC_FP64_FAST, nspec=eos.nspec)
    ref_out, _ = oracle().hydro_box(prm, lo, hi, uin)
    got_out, _ = _gpu_hydro_box(prm, lo, hi, uin, with_flx=False)
    l1, linf = rel_err(got_out, ref_out.data)
    assert l1 <= FP64_TOL and linf <= FP64_TOL, (l1, linf)


@pytest.mark.parametrize("name,ppm,order", CASES)
def test_hydro_box_mixed_within_tolerance(name, ppm, order):
    src, lo, hi, uin, eos = _case(name)
    _setup(eos)
    dt = _dt(uin, lo, hi, src.dx)
    prm = params_for(src, dt, ppm_type=ppm, plm_iorder=order, prec=abi.PREC_MIXED, nspec=eos.nspec)
    ref_out, _ = oracle().hydro_box(prm, lo, hi, uin)
    got_out, _ = _gpu_hydro_box(prm, lo, hi, uin, with_flx=False)
    assert np.isfinite(got_out).all()
    s_ref = oracle().update_state(lo, hi, uin, ref_out, dt)
    s_got = oracle().update_state(lo, hi, uin, abi.Fab(got_out, tuple(lo)), dt)
    l1, _ = rel_err(s_got.view(lo, hi), s_ref.view(lo, hi))
    assert l1 <= MIXED_TOL, l1


def test_ctoprim_and_umdrv_dropin_bitexact():
    """pcg_ctoprim + pcg_umdrv with caller-owned q/qaux/flx/area/vol, uout accumulated."""
    p = wl.random_patch((10, 8, 7), 11)
    eos = wl.GammaLaw()
    _setup(eos)
    lo, hi = p.lo, p.hi
    g4lo, g4hi = abi.grow(lo, hi, 4)
    dt = _dt(p.fab, lo, hi, p.dx)
    prm = params_for(p, dt, nspec=1)
    o = oracle()
    q_ref, qa_ref = o.ctoprim(g4lo, g4hi, p.fab)
    uin = to_gpu(p.fab)
    q = gpu_zeros(abi.qvar(1), g4lo, g4hi)
    qa = gpu_zeros(abi.NQAUX, g4lo, g4hi)
    hydro.ctoprim(prm, g4lo, g4hi, uin, q, qa)
    np.testing.assert_array_equal(to_cpu(q), q_ref.data)
    np.testing.assert_array_equal(to_cpu(qa), qa_ref.data)
    import pyoracle

    area, vol = pyoracle.uniform_geometry(lo, hi, p.dx)
    rng = np.random.default_rng(0)
    nv = abi.nvar(1)
    shp = (nv,) + tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
    u0 = rng.standard_normal(shp)
    ref_out = abi.Fab(u0.copy(), tuple(lo))
    ref_flx = [np_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
    import ctypes as C

    rc = o._umdrv(C.byref(prm), abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(p.fab)), C.byref(abi.array4(ref_out)),
                  C.byref(abi.array4(q_ref)), C.byref(abi.array4(qa_ref)), None, abi.array4_list(ref_flx),
                  abi.array4_list(area), C.byref(abi.array4(vol)))
    assert rc == 0
    uout = to_gpu(abi.Fab(u0.copy(), tuple(lo)))
    flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
    hydro.umdrv(prm, lo, hi, uin, uout, q, qa, None, flx, [to_gpu(a) for a in area], to_gpu(vol))
    np.testing.assert_array_equal(to_cpu(uout), ref_out.data)
    for d in range(3):
        np.testing.assert_array_equal(to_cpu(flx[d]), ref_flx[d].data)
