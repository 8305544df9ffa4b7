"""pcg_hydro_box_noalloc: one box's hydro advance for callers that must not allocate
device memory.

A PeleC run on GPUs normally lets the AMReX arena reserve most of the device memory at
start-up, so a library that calls cudaMalloc inside the run can fail or fragment what
the arena left, and some hosts forbid the implicit synchronisation of cudaMalloc/cudaFree
in their step loop. This entry point keeps its tables and workspace in a fixed 32 MiB
device array of the library. The test calls it through the C ABI twice in a row on
different boxes (the second call runs on the scratch contents the first one left) and
compares each result with pcg_hydro_box, which allocates its workspace; in the plain FP64
form the two must agree bit for bit. It also checks that a box needing more scratch than
the array holds is refused with PCG_EINVAL.
"""
import ctypes as C

import numpy as np
import pytest

from common import eos9, gpu_zeros, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, native, workloads as wl

pytestmark = pytest.mark.gpu
BIG = 1 << 30


def _call_noalloc(prm, lo, hi, uin, uout, flx):
    lib = native.load()
    return lib.pcg_hydro_box_noalloc(C.byref(prm), abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(uin)),
                                     C.byref(abi.array4(uout)), abi.array4_list(flx) if flx else None,
                                     hydro._stream_ptr(None))


def _case(kind):
    if kind == "flame":
        lev = wl.flame(n=16, box=16)
        lo, hi = lev.boxes[0]
        prm = abi.make_params(lev.dx, 2e-8, 9, lev.domlo, lev.domhi, lev.bclo, lev.bchi)
        return prm, lo, hi, lev.box_fab(lo, hi)
    p = wl.random_patch((13, 9, 11), 77)
    prm = abi.make_params(p.dx, 2e-3, 1, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=0)
    return prm, p.lo, p.hi, p.fab


def test_noalloc_matches_allocating_entry_on_two_calls_in_a_row():
    hydro.init(0)
    hydro.set_eos(eos9())
    hydro.set_eos(wl.GammaLaw())
    results = []
    for kind in ("flame", "random_gamma"):
        prm, lo, hi, fab = _case(kind)
        nv = abi.nvar(prm.nspec)
        uin = to_gpu(fab)
        out = gpu_zeros(nv, lo, hi)
        flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
        rc = _call_noalloc(prm, lo, hi, uin, out, flx)
        assert rc == 0, native.load().pcg_last_error().decode()
        results.append((prm, lo, hi, uin, out, flx))
    for prm, lo, hi, uin, out, flx in results:
        nv = abi.nvar(prm.nspec)
        ref_out = gpu_zeros(nv, lo, hi)
        ref_flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
        hydro.hydro_box(prm, lo, hi, uin, ref_out, ref_flx)
        np.testing.assert_array_equal(to_cpu(out), to_cpu(ref_out))
        for d in range(3):
            np.testing.assert_array_equal(to_cpu(flx[d]), to_cpu(ref_flx[d]))


def test_noalloc_refuses_boxes_beyond_its_scratch():
    hydro.init(0)
    hydro.set_eos(eos9())
    p = wl.flame_patch((32, 32, 32), 5)
    prm = abi.make_params(p.dx, 2e-8, 9, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0))
    uin = to_gpu(p.fab)
    out = gpu_zeros(abi.nvar(9), p.lo, p.hi)
    rc = _call_noalloc(prm, p.lo, p.hi, uin, out, None)
    assert rc == -1
    msg = native.load().pcg_last_error().decode()
    assert "scratch" in msg and "pcg_hydro_box" in msg


@pytest.mark.parametrize("prec,edge", [(abi.PREC_FP64, 21), (abi.PREC_MIXED, 27)])
def test_noalloc_accepts_the_largest_stated_box_and_refuses_the_next(prec, edge):
    """The stated limits with 9 species and no flux export: 21^3 in FP64 and 27^3 in the
    mixed form run (and equal pcg_hydro_box bit for bit), one cell more per edge is refused."""
    hydro.init(0)
    hydro.set_eos(eos9())
    nv = abi.nvar(9)
    p = wl.flame_patch((edge, edge, edge), 9)
    prm = abi.make_params(p.dx, 2e-8, 9, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), precision_mode=prec)
    uin = to_gpu(p.fab)
    out = gpu_zeros(nv, p.lo, p.hi)
    rc = _call_noalloc(prm, p.lo, p.hi, uin, out, None)
    assert rc == 0, native.load().pcg_last_error().decode()
    ref = gpu_zeros(nv, p.lo, p.hi)
    hydro.hydro_box(prm, p.lo, p.hi, uin, ref)
    np.testing.assert_array_equal(to_cpu(out), to_cpu(ref))
    big = wl.flame_patch((edge + 1, edge + 1, edge + 1), 10)
    uin2 = to_gpu(big.fab)
    out2 = gpu_zeros(nv, big.lo, big.hi)
    assert _call_noalloc(prm, big.lo, big.hi, uin2, out2, None) == -1
