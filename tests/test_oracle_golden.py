"""The CPU oracle against golden vectors produced by the reference's own hot-path
sources (Source/Godunov.cpp, PPM.cpp and the Godunov/PPM/PLM/Riemann/Hydro headers,
compiled in place; see tests/golden/make_golden.py). Bit-exact: the oracle restates
the reference with the same operation order."""
import glob
import os

import numpy as np
import pytest

from common import oracle
from particleclem_b200 import abi, thermo, workloads as wl

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load_case(path):
    z = np.load(path)
    nspec = int(z["nspec"])
    eos = wl.GammaLaw() if nspec == 1 else thermo.load_nasa7()
    lo, hi = tuple(int(v) for v in z["lo"]), tuple(int(v) for v in z["hi"])
    uin = abi.Fab(np.ascontiguousarray(z["uin"]), tuple(int(v) for v in z["uin_lo"]))
    prm = abi.make_params(z["dx"], float(z["dt"]), nspec, z["domlo"], z["domhi"], z["bclo"], z["bchi"],
                          ppm_type=int(z["ppm_type"]), plm_iorder=int(z["plm_iorder"]))
    return z, eos, lo, hi, uin, prm


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 8


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_golden(path):
    z, eos, lo, hi, uin, prm = load_case(path)
    o = oracle()
    o.set_eos(eos)
    assert o.estdt(lo, hi, uin, tuple(z["dx"])) == float(z["estdt"])
    hs, flx = o.hydro_box(prm, lo, hi, uin)
    np.testing.assert_array_equal(hs.data, z["hydro_source"])
    for d in range(3):
        np.testing.assert_array_equal(flx[d].data, z[f"flx{d}"])
    snew = o.update_state(lo, hi, uin, hs, float(z["dt"]))
    np.testing.assert_array_equal(snew.view(lo, hi), z["snew"])
