"""GPU parity of the source path and of the pc_umeth_3D operator surface, through the C ABI.

* pcg_srctoprim (pc_srctoprim, Source/Hydro.H:14-68) on non-zero conserved sources equals
  the oracle bit for bit;
* pcg_umdrv fed with those primitive sources (the hdt * srcQ terms of pc_transdd,
  Source/Godunov.H:639-845) equals the oracle's pc_umdrv bit for bit in the plain FP64
  form, and stays within the mixed form's bound;
* pcg_umeth (pc_umeth_3D alone, Source/Godunov.H:1142-1162) returns the unadjusted final
  fluxes, the face states qec and p div u bit for bit, with and without sources, and on a
  box whose low faces are inflow boundaries (the low-order boundary faces).

The oracle's srctoprim and umeth are themselves pinned to the reference build
(tests/test_oracle_vs_reference.py).
"""
import numpy as np
import pytest

import pyoracle
from common import MIXED_TOL, eos9, gpu_zeros, oracle, random_sources, rel_err, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, workloads as wl

pytestmark = pytest.mark.gpu
BIG = 1 << 30


def _setup(nspec):
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    hydro.init(0)
    hydro.set_eos(eos)
    oracle().set_eos(eos)
    return eos


def _inputs(nspec, seed, edges=(9, 7, 6)):
    eos = _setup(nspec)
    p = wl.random_patch(edges, seed, eos if nspec == 9 else None)
    g4lo, g4hi = abi.grow(p.lo, p.hi, 4)
    q, qa = oracle().ctoprim(g4lo, g4hi, p.fab)
    src = random_sources(p.fab, seed + 1, scale=20.0 if nspec == 1 else 1e4)
    sq = oracle().srctoprim(g4lo, g4hi, q, qa, src)
    dt = 0.3 * oracle().estdt(p.lo, p.hi, p.fab, p.dx)
    return p, g4lo, g4hi, q, qa, src, sq, dt


@pytest.mark.parametrize("nspec", [1, 9])
def test_srctoprim_bitexact(nspec):
    p, g4lo, g4hi, q, qa, src, sq_ref, _ = _inputs(nspec, 801)
    prm = abi.make_params(p.dx, 0.0, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0))
    out = gpu_zeros(abi.qvar(nspec), g4lo, g4hi)
    hydro.srctoprim(prm, g4lo, g4hi, to_gpu(q), to_gpu(qa), to_gpu(src), out)
    got = to_cpu(out)
    assert np.abs(got).max() > 0
    np.testing.assert_array_equal(got, sq_ref.data)


@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("ppm", [1, 0])
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_umdrv_with_sources(nspec, ppm, prec):
    p, g4lo, g4hi, q, qa, src, sq, dt = _inputs(nspec, 811 + 2 * ppm)
    lo, hi = p.lo, p.hi
    nv = abi.nvar(nspec)
    prm64 = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=ppm)
    area, vol = pyoracle.uniform_geometry(lo, hi, p.dx)
    ref_out = abi.Fab(np.zeros((nv,) + tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))), tuple(lo))
    ref_flx = [abi.Fab(np.zeros((nv,) + tuple(b[e] - a[e] + 1 for e in (2, 1, 0))), a)
               for a, b in (abi.nodes(lo, hi, d) for d in range(3))]
    import ctypes as C

    rc = oracle()._umdrv(C.byref(prm64), abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(p.fab)),
                         C.byref(abi.array4(ref_out)), C.byref(abi.array4(q)), C.byref(abi.array4(qa)),
                         C.byref(abi.array4(sq)), abi.array4_list(ref_flx), abi.array4_list(area),
                         C.byref(abi.array4(vol)))
    assert rc == 0
    prm = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=ppm,
                          precision_mode=prec)
    uout = gpu_zeros(nv, lo, hi)
    flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
    hydro.umdrv(prm, lo, hi, to_gpu(p.fab), uout, to_gpu(q), to_gpu(qa), to_gpu(sq), flx,
                [to_gpu(a) for a in area], to_gpu(vol))
    got = to_cpu(uout)
    if prec == abi.PREC_FP64:
        np.testing.assert_array_equal(got, ref_out.data)
        for d in range(3):
            np.testing.assert_array_equal(to_cpu(flx[d]), ref_flx[d].data)
        # the sources entered: without them the result differs
        out0 = gpu_zeros(nv, lo, hi)
        hydro.umdrv(prm, lo, hi, to_gpu(p.fab), out0, to_gpu(q), to_gpu(qa), None,
                    [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)], [to_gpu(a) for a in area],
                    to_gpu(vol))
        assert not np.array_equal(to_cpu(out0), got)
    else:
        s_ref = oracle().update_state(lo, hi, p.fab, ref_out, dt)
        s_got = oracle().update_state(lo, hi, p.fab, abi.Fab(got, tuple(lo)), dt)
        l1, _ = rel_err(s_got.view(lo, hi), s_ref.view(lo, hi))
        assert l1 <= MIXED_TOL, l1


UMETH_CASES = [
    # (nspec, ppm, with sources, bclo, bchi): the inflow low faces take the low-order path
    (1, 1, False, (0, 0, 0), (0, 0, 0)),
    (1, 0, True, (0, 0, 0), (0, 0, 0)),
    (9, 1, True, (0, 0, 0), (0, 0, 0)),
    (9, 0, False, (0, 0, 0), (0, 0, 0)),
    (1, 1, True, (1, 1, 0), (2, 5, 0)),
    (9, 1, False, (1, 0, 1), (2, 0, 6)),
]


@pytest.mark.parametrize("nspec,ppm,with_src,bclo,bchi", UMETH_CASES)
def test_umeth_bitexact(nspec, ppm, with_src, bclo, bchi):
    p, g4lo, g4hi, q, qa, src, sq, dt = _inputs(nspec, 831 + nspec + ppm, edges=(7, 6, 8))
    lo, hi = p.lo, p.hi
    boundary = any(bclo) or any(bchi)
    dom = (lo, hi) if boundary else ((-BIG,) * 3, (BIG,) * 3)
    prm = abi.make_params(p.dx, dt, nspec, dom[0], dom[1], bclo, bchi, ppm_type=ppm)
    area, vol = pyoracle.uniform_geometry(lo, hi, p.dx)
    rflx, rqec, rpdivu = oracle().umeth(prm, lo, hi, q, qa, sq if with_src else None, area, vol)
    nv = abi.nvar(nspec)
    flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
    qec = [gpu_zeros(abi.NGDNV, *abi.nodes(lo, hi, d)) for d in range(3)]
    pdivu = gpu_zeros(1, lo, hi)
    hydro.umeth(prm, lo, hi, to_gpu(q), to_gpu(qa), to_gpu(sq) if with_src else None, flx, qec,
                [to_gpu(a) for a in area], pdivu, to_gpu(vol))
    for d in range(3):
        np.testing.assert_array_equal(to_cpu(flx[d]), rflx[d].data)
        np.testing.assert_array_equal(to_cpu(qec[d]), rqec[d].data)
    np.testing.assert_array_equal(to_cpu(pdivu), rpdivu.data)
    assert np.abs(rpdivu.data).max() > 0
