"""The flux-register binding of the PeleC-side C++ adapter (include/pcg_pelec_adapter.H:
update_flux_registers and reflux on the library's register) exercised from C++.

tests/cxx/fluxreg_test.cpp does one coarse step's refluxing as PeleC does it
(Source/Hydro.cpp:281-287 -> update_flux_registers, Source/PeleC.cpp:1343-1400; reflux,
:1403-1414) against the AMReX Array4 API of the repository's shim, on device memory. The
CPU test checks that it compiles and links; the GPU test feeds it random coarse and fine
fluxes and compares the refluxed coarse state bit for bit with the register of the CPU
oracle (oracle/fluxreg_oracle.py) on the same fluxes.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import fluxreg_oracle as fro
from particleclem_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CXX = os.path.join(ROOT, "tests", "cxx")
EXE = os.path.join(CXX, "_build", "fluxreg_test")


def _build():
    if shutil.which("g++") is None or not os.path.exists("/usr/local/cuda/include/cuda_runtime.h"):
        pytest.skip("g++ or the CUDA headers are missing")
    from particleclem_b200 import native

    native.load()  # builds the library in place if needed
    subprocess.run(["make", "-s", "-C", CXX], check=True)
    return EXE


def test_fluxreg_binding_compiles_and_links():
    assert os.path.exists(_build())


def _faces(rng, lo, hi, nc):
    out = []
    for d in range(3):
        nlo, nhi = abi.nodes(lo, hi, d)
        shp = (nc,) + tuple(nhi[e] - nlo[e] + 1 for e in (2, 1, 0))
        out.append(abi.Fab(rng.standard_normal(shp), tuple(nlo)))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("ratio,flo,fhi,periodic", [(2, (0, 8, 4), (7, 15, 11), (1, 1, 1)),
                                                    (4, (16, 12, 20), (27, 23, 31), (0, 1, 1))])
def test_fluxreg_binding_equals_oracle(tmp_path, ratio, flo, fhi, periodic):
    exe = _build()
    n, nc, nsub = 12, 8, ratio
    rng = np.random.default_rng(17 + ratio)
    dt_c, vol = 1.3e-3, (1.0 / n) ** 3
    dt_f = dt_c / ratio
    cflx = _faces(rng, (0, 0, 0), (n - 1,) * 3, nc)
    fflx = [_faces(rng, flo, fhi, nc) for _ in range(nsub)]
    state = abi.Fab(rng.standard_normal((nc, n, n, n)), (0, 0, 0))
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([nc, ratio, n, nsub, *flo, *fhi, *periodic], dtype=np.int32).tofile(f)
        np.array([dt_c, dt_f, vol], dtype=np.float64).tofile(f)
        for fab in cflx:
            np.ascontiguousarray(fab.data).tofile(f)
        for sub in fflx:
            for fab in sub:
                np.ascontiguousarray(fab.data).tofile(f)
        np.ascontiguousarray(state.data).tofile(f)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(tmp_path / "out.bin", dtype=np.float64).reshape(state.data.shape)
    reg = fro.FluxRegister(nc, (0, 0, 0), (n - 1,) * 3, periodic, ratio, [(flo, fhi)])
    reg.crse_add((0, 0, 0), (n - 1,) * 3, cflx, dt_c)
    for sub in fflx:
        reg.fine_add(flo, fhi, sub, dt_f)
    expect = abi.Fab(state.data.copy(), (0, 0, 0))
    reg.reflux(expect, vol)
    np.testing.assert_array_equal(got, expect.data)
    assert not np.array_equal(got, state.data)  # the register corrected some cells
