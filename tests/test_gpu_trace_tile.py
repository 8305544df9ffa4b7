"""The tiled trace of the mixed form (trace launch variants 3-5) against the untiled one.

The tiled trace stages each tile of 128 cells of the FP32 primitive copy and its halo in
shared memory with one TMA load, forms each PPM interface value once per interface (the
untiled trace forms both of a cell's interfaces per cell) and traces the strips that full
tiles leave over one cell per thread; the untiled trace reads the array in global memory.
Both must meet the mixed form's bounds against the FP64 oracle, on boxes whose extents
are not multiples of the tile (strips on every side, x origins that are not multiples of
4), with PPM and PLM, with the ghost cells' primitive state formed by ctoprim (hydro_box)
or passed in (umdrv), and on a fused region of four boxes; each test prints the
difference between the two.
"""
import dataclasses

import numpy as np
import pytest

import pyoracle
from common import MIXED_TOL, eos9, gpu_zeros, oracle, params_for, rel_errors, to_cpu, to_gpu
from particleclem_b200 import abi, autotune, hydro, workloads as wl

pytestmark = pytest.mark.gpu

TRACE = autotune.TRACE_STAGE
MIXED_SRC_TOL = 5e-4  # the hydro source's own bound (see test_gpu_config_parity)


@pytest.fixture
def trace_variant():
    """Restore every mixed trace variant after the test."""
    saved = {ns: autotune.get_variant(abi.PREC_MIXED, ns, TRACE) for ns in (1, 9)}
    yield lambda ns, v: autotune.set_variant(abi.PREC_MIXED, ns, TRACE, v)
    for ns, v in saved.items():
        autotune.set_variant(abi.PREC_MIXED, ns, TRACE, v)


def _patch(nspec, edges, seed):
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    p = wl.random_patch(edges, seed, eos if nspec == 9 else None)
    sh = lambda t: tuple(int(v) + 3 for v in t)  # noqa: E731  (an x origin not a multiple of 4)
    return dataclasses.replace(p, lo=sh(p.lo), hi=sh(p.hi), fab=abi.Fab(p.fab.data, sh(p.fab.lo))), eos


def _run(prm, p):
    out = gpu_zeros(abi.nvar(prm.nspec), p.lo, p.hi)
    hydro.hydro_box(prm, p.lo, p.hi, to_gpu(p.fab), out)
    return to_cpu(out)


def _check_vs_oracle(p, prm64, got, dt):
    ref, _ = oracle().hydro_box(prm64, p.lo, p.hi, p.fab)
    s_ref = oracle().update_state(p.lo, p.hi, p.fab, ref, dt).view(p.lo, p.hi)
    s_got = oracle().update_state(p.lo, p.hi, p.fab, abi.Fab(got, tuple(p.lo)), dt).view(p.lo, p.hi)
    s_l1 = rel_errors(s_got, s_ref)[0].max()
    h_l1 = rel_errors(got, ref.data)[0].max()
    assert s_l1 <= MIXED_TOL and h_l1 <= MIXED_SRC_TOL, (s_l1, h_l1)
    return s_l1, h_l1


@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("ppm", [1, 0])
@pytest.mark.parametrize("edges", [(37, 9, 6), (5, 13, 11)])
def test_tiled_trace_matches_untiled(nspec, ppm, edges, trace_variant):
    p, eos = _patch(nspec, edges, 700 + nspec + 3 * ppm + edges[0])
    hydro.init(0)
    hydro.set_eos(eos)
    oracle().set_eos(eos)
    dt = 0.3 * oracle().estdt(p.lo, p.hi, p.fab, p.dx)
    prm = params_for(p, dt, ppm_type=ppm, nspec=nspec, prec=abi.PREC_MIXED)
    trace_variant(nspec, 2)
    untiled = _run(prm, p)
    trace_variant(nspec, 5)
    tiled = _run(prm, p)
    assert np.isfinite(tiled).all()
    diff = rel_errors(tiled, untiled)[0].max()
    print(f"\nnspec {nspec} ppm {ppm} {edges}: tiled vs untiled rel L1 {diff:.3e}")
    prm64 = params_for(p, dt, ppm_type=ppm, nspec=nspec)
    for got in (untiled, tiled):
        _check_vs_oracle(p, prm64, got, dt)


@pytest.mark.parametrize("nspec", [1, 9])
def test_tiled_trace_with_caller_primitives(nspec, trace_variant):
    """umdrv with q, qaux from ctoprim: the FP32 copy covers grow(box, 3) only."""
    p, eos = _patch(nspec, (19, 6, 10), 820 + nspec)
    hydro.init(0)
    hydro.set_eos(eos)
    oracle().set_eos(eos)
    dt = 0.3 * oracle().estdt(p.lo, p.hi, p.fab, p.dx)
    prm = params_for(p, dt, nspec=nspec, prec=abi.PREC_MIXED)
    g4lo, g4hi = abi.grow(p.lo, p.hi, 4)
    nv, nq = abi.nvar(nspec), abi.qvar(nspec)
    res = []
    for v in (2, 5):
        trace_variant(nspec, v)
        uin = to_gpu(p.fab)
        q, qa = gpu_zeros(nq, g4lo, g4hi), gpu_zeros(abi.NQAUX, g4lo, g4hi)
        hydro.ctoprim(prm, g4lo, g4hi, uin, q, qa)
        sq = gpu_zeros(nq, g4lo, g4hi)
        out = gpu_zeros(nv, p.lo, p.hi)
        flx = [gpu_zeros(nv, *abi.nodes(p.lo, p.hi, d)) for d in range(3)]
        area, vol = pyoracle.uniform_geometry(p.lo, p.hi, p.dx)
        area, vol = [to_gpu(a) for a in area], to_gpu(vol)
        hydro.umdrv(prm, p.lo, p.hi, uin, out, q, qa, sq, flx, area, vol)
        res.append(to_cpu(out))
    diff = rel_errors(res[1], res[0])[0].max()
    print(f"\numdrv nspec {nspec}: tiled vs untiled rel L1 {diff:.3e}")
    prm64 = params_for(p, dt, nspec=nspec)
    for got in res:
        _check_vs_oracle(p, prm64, got, dt)


def test_tiled_trace_fused_region(trace_variant):
    """Four boxes of a 48^3 flame level fused into one region (one tensor map set)."""
    import torch

    lev = wl.flame(n=48, box=24, seed=3)
    hydro.init(0)
    hydro.set_eos(lev.eos)
    oracle().set_eos(lev.eos)
    block = [(lo, hi) for lo, hi in lev.boxes if lo[2] == 0]
    assert len(block) == 4
    fabs = [lev.box_fab(lo, hi) for lo, hi in block]
    dt = 0.3 * min(oracle().estdt(lo, hi, f, lev.dx) for (lo, hi), f in zip(block, fabs))
    n = [lev.domhi[d] - lev.domlo[d] + 1 for d in range(3)]
    res = []
    for v in (2, 5):
        trace_variant(9, v)
        state = abi.Fab(torch.from_numpy(np.ascontiguousarray(lev.state)).cuda(), lev.fab.lo)
        hsrc = abi.Fab(torch.zeros((abi.nvar(9), n[2], n[1], n[0]), dtype=torch.float64, device="cuda"),
                       tuple(lev.domlo))
        boxes = [hydro.make_box(lo, hi, state, hsrc, lev.dx, dt, lev.domlo, lev.domhi, lev.bclo, lev.bchi)
                 for lo, hi in block]
        plan = hydro.Plan(params_for(lev, dt, prec=abi.PREC_MIXED), boxes, fuse=True)
        assert plan.info()["nregions"] == 1
        plan.hydro()
        res.append(to_cpu(hsrc))
        plan.close()
    diff = rel_errors(res[1], res[0])[0].max()
    print(f"\nfused 2x2x1 flame block: tiled vs untiled rel L1 {diff:.3e}")
    assert diff <= MIXED_SRC_TOL
