"""Property checks of the oracle that mirror the reference's verification tests:
conservation (Tests/test_masscons.py checks total mass and rho E to rtol 1e-13) and
the species-flux normalisation of pc_norm_spec_flx (Source/Hydro.H:835-849)."""
import numpy as np
import pytest

from common import eos9, oracle
from particleclem_b200 import abi, workloads as wl


def _periodic_level(nspec, n=10):
    lev = wl.turbulence(n=n, box=n, seed=7, kmax=3) if nspec == 1 else wl.flame(n=n, box=n)
    if nspec == 9:  # make z periodic too so that the box is a closed system
        lev.periodic = (True, True, True)
        lev.bclo = lev.bchi = (0, 0, 0)
        lev.fill_ghosts()
    return lev


@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("ppm", [1, 0])
def test_periodic_box_conserves_mass_momentum_energy(nspec, ppm):
    lev = _periodic_level(nspec)
    o = oracle()
    o.set_eos(lev.eos)
    lo, hi = lev.boxes[0]
    uin = lev.box_fab(lo, hi)
    dt = 0.3 * o.estdt(lo, hi, uin, lev.dx)
    big = 1 << 30
    prm = abi.make_params(lev.dx, dt, nspec, (-big,) * 3, (big,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=ppm)
    hs, _ = o.hydro_box(prm, lo, hi, uin)
    vol = np.prod(lev.dx)
    u = uin.view(lo, hi)
    for c in (abi.URHO, abi.UMX, abi.UMY, abi.UMZ, abi.UEDEN):
        total = np.abs(u[c]).sum() * vol
        net = hs.data[c].sum() * vol * dt
        assert abs(net) <= 1e-13 * total, (c, net, total)


def test_species_fluxes_sum_to_mass_flux():
    p = wl.random_patch((6, 5, 4), 31, eos9())
    o = oracle()
    o.set_eos(eos9())
    dt = 0.3 * o.estdt(p.lo, p.hi, p.fab, p.dx)
    big = 1 << 30
    prm = abi.make_params(p.dx, dt, 9, (-big,) * 3, (big,) * 3, (0, 0, 0), (0, 0, 0))
    _, flx = o.hydro_box(prm, p.lo, p.hi, p.fab)
    for f in flx:
        s = f.data[abi.UFS:].sum(axis=0)
        np.testing.assert_allclose(s, f.data[abi.URHO], rtol=1e-12, atol=1e-12 * np.abs(f.data[abi.URHO]).max())
