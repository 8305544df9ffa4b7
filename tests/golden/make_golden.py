"""Generate the golden fixtures of the hydro path from the reference's own code.

The reference's Godunov/PPM/PLM/Riemann sources are compiled in place by
oracle/ref/Makefile (needs the reference checkout) into oracle/_ref. This script runs
them on small seeded inputs and stores inputs and outputs as compressed .npz files
beside it, so the CPU oracle and the GPU path can be checked against the reference
where the reference checkout is not available.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from particleclem_b200 import abi, thermo, workloads as wl  # noqa: E402

BIG = 1 << 30


def cases():
    eos9 = thermo.load_nasa7()
    lev = wl.sod(8)
    lo, hi = lev.boxes[0]
    yield "sod8_ppm", lev.eos, lo, hi, lev.box_fab(lo, hi), lev.dx, lev.domlo, lev.domhi, lev.bclo, lev.bchi, 1, 4
    p = wl.random_patch((7, 6, 5), 21)
    for ppm, order in ((1, 4), (0, 4), (0, 2)):
        yield (f"random_gamma_ppm{ppm}_o{order}", wl.GammaLaw(), p.lo, p.hi, p.fab, p.dx, (-BIG,) * 3, (BIG,) * 3,
               (0, 0, 0), (0, 0, 0), ppm, order)
    p = wl.random_patch((6, 5, 5), 22, eos9)
    for ppm in (1, 0):
        yield (f"random_nasa7_ppm{ppm}", eos9, p.lo, p.hi, p.fab, p.dx, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0),
               (0, 0, 0), ppm, 4)
    # walls: symmetry/slip/no-slip faces exercise the Riemann boundary overrides
    p = wl.random_patch((6, 6, 6), 23)
    yield ("random_gamma_walls", wl.GammaLaw(), p.lo, p.hi, p.fab, p.dx, (0, 0, 0), (5, 5, 5),
           (abi.BC_NO_SLIP_WALL, abi.BC_SLIP_WALL, abi.BC_SYMMETRY), (abi.BC_OUTFLOW, abi.BC_NO_SLIP_WALL, abi.BC_SLIP_WALL),
           1, 4)
    lev = wl.flame(n=8, box=8)
    lo, hi = lev.boxes[0]
    yield "flame8_ppm", lev.eos, lo, hi, lev.box_fab(lo, hi), lev.dx, lev.domlo, lev.domhi, lev.bclo, lev.bchi, 1, 4


def main():
    for name, eos, lo, hi, uin, dx, domlo, domhi, bclo, bchi, ppm, order in cases():
        ref = pyoracle.reference(eos.nspec)
        ref.set_eos(eos)
        dt0 = ref.estdt(lo, hi, uin, dx)
        dt = 0.3 * dt0
        prm = abi.make_params(dx, dt, eos.nspec, domlo, domhi, bclo, bchi, ppm_type=ppm, plm_iorder=order)
        hs, flx = ref.hydro_box(prm, lo, hi, uin)
        snew = ref.update_state(lo, hi, uin, hs, dt)
        out = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(out, uin=uin.data, uin_lo=np.array(uin.lo), lo=np.array(lo), hi=np.array(hi),
                            dx=np.array(dx), dt=dt, estdt=dt0, domlo=np.array(domlo), domhi=np.array(domhi),
                            bclo=np.array(bclo), bchi=np.array(bchi), ppm_type=ppm, plm_iorder=order,
                            nspec=eos.nspec, hydro_source=hs.data, flx0=flx[0].data, flx1=flx[1].data,
                            flx2=flx[2].data, snew=snew.view(lo, hi))
        print(name, os.path.getsize(out))


if __name__ == "__main__":
    main()
