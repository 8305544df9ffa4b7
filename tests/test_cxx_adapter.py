"""The PeleC-side C++ binding (include/pcg_pelec_adapter.H) exercised from C++.

tests/cxx/adapter_test.cpp is the body of construct_hydro_source's box loop
(Source/Hydro.cpp:70-249) written against the AMReX Array4 API, with pc_ctoprim,
pc_srctoprim and pc_umdrv replaced by the library through the adapter, on device memory.
It builds against the repository's AMReX-API shim in place of AMReX. The CPU test checks
that it compiles and links against the library; the GPU test runs it on a box with
non-zero sources and compares hydro source and fluxes bit for bit with the same box loop
run by the reference's own sources compiled on the CPU (oracle/_ref; the oracle
restatement, which is pinned to that build, where the build is absent).
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import pyoracle
from common import eos9, oracle, random_sources
from particleclem_b200 import abi, workloads as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CXX = os.path.join(ROOT, "tests", "cxx")
EXE = os.path.join(CXX, "_build", "adapter_test")


def _build():
    if shutil.which("g++") is None or not os.path.exists("/usr/local/cuda/include/cuda_runtime.h"):
        pytest.skip("g++ or the CUDA headers are missing")
    from particleclem_b200 import native

    native.load()  # builds the library in place if needed
    subprocess.run(["make", "-s", "-C", CXX], check=True)
    return EXE


def test_adapter_compiles_and_links():
    assert os.path.exists(_build())


def _write_input(path, nspec, ppm, lo, hi, dx, dt, difmag, eos, fab, src):
    with open(path, "wb") as f:
        np.array([nspec, ppm, 4, *lo, *hi], dtype=np.int32).tofile(f)
        np.array([*dx, dt, difmag], dtype=np.float64).tofile(f)
        if nspec == 1:
            np.array([eos.gamma, eos.mw], dtype=np.float64).tofile(f)
        else:
            for a in (eos.mw, eos.tmid, eos.a_lo, eos.a_hi):
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        np.ascontiguousarray(fab.data).tofile(f)
        np.ascontiguousarray(src.data).tofile(f)


@pytest.mark.gpu
@pytest.mark.parametrize("nspec,ppm", [(1, 1), (9, 1), (9, 0)])
def test_adapter_box_loop_equals_reference_build(nspec, ppm, tmp_path):
    exe = _build()
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    p = wl.random_patch((10, 7, 8), 901 + nspec + ppm, eos if nspec == 9 else None)
    lo, hi = p.lo, p.hi
    src = random_sources(p.fab, 903 + nspec, scale=20.0 if nspec == 1 else 1e4)
    ref = pyoracle.reference(nspec) if pyoracle.ref_available(nspec) else oracle()
    ref.set_eos(eos)
    dt = 0.3 * ref.estdt(lo, hi, p.fab, p.dx)
    difmag = 0.1
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write_input(inp, nspec, ppm, lo, hi, p.dx, dt, difmag, eos, p.fab, src)
    r = subprocess.run([exe, inp, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

    # the same box loop on the CPU: ctoprim, srctoprim, umdrv of the reference build
    big = 1 << 30
    prm = abi.make_params(p.dx, dt, nspec, (-big,) * 3, (big,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=ppm,
                          plm_iorder=4, difmag=difmag)
    g4lo, g4hi = abi.grow(lo, hi, 4)
    q, qa = ref.ctoprim(g4lo, g4hi, p.fab)
    sq = ref.srctoprim(g4lo, g4hi, q, qa, src)
    nv = abi.nvar(nspec)
    shp = lambda a, b: tuple(b[e] - a[e] + 1 for e in (2, 1, 0))  # noqa: E731
    uout = abi.Fab(np.zeros((nv,) + shp(lo, hi)), tuple(lo))
    flx = [abi.Fab(np.zeros((nv,) + shp(*abi.nodes(lo, hi, d))), abi.nodes(lo, hi, d)[0]) for d in range(3)]
    area, vol = pyoracle.uniform_geometry(lo, hi, p.dx)
    rc = ref._umdrv(C.byref(prm), abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(p.fab)), C.byref(abi.array4(uout)),
                    C.byref(abi.array4(q)), C.byref(abi.array4(qa)), C.byref(abi.array4(sq)), abi.array4_list(flx),
                    abi.array4_list(area), C.byref(abi.array4(vol)))
    assert rc == 0

    got = np.fromfile(out, dtype=np.float64)
    n0 = uout.data.size
    np.testing.assert_array_equal(got[:n0].reshape(uout.data.shape), uout.data)
    off = n0
    for d in range(3):
        n = flx[d].data.size
        np.testing.assert_array_equal(got[off:off + n].reshape(flx[d].data.shape), flx[d].data)
        off += n
    assert off == got.size
