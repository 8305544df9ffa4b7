"""The oracle restatement against the reference's own code on fresh random inputs
(runs where oracle/_ref was built from the reference checkout)."""
import numpy as np
import pytest

import pyoracle
from common import eos9, oracle
from particleclem_b200 import abi, workloads as wl

BIG = 1 << 30


@pytest.mark.parametrize("seed", [101, 102, 103])
@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("ppm", [1, 0])
def test_oracle_equals_reference_build(seed, nspec, ppm):
    if not pyoracle.ref_available(nspec):
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    p = wl.random_patch((5, 4, 6), seed, eos if nspec == 9 else None)
    ref = pyoracle.reference(nspec)
    ref.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    dt = 0.3 * ref.estdt(p.lo, p.hi, p.fab, p.dx)
    prm = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=ppm)
    a, fa = o.hydro_box(prm, p.lo, p.hi, p.fab)
    b, fb = ref.hydro_box(prm, p.lo, p.hi, p.fab)
    np.testing.assert_array_equal(a.data, b.data)
    for d in range(3):
        np.testing.assert_array_equal(fa[d].data, fb[d].data)


BCS = {
    # (bclo, bchi) per direction: interior 0, inflow 1, outflow 2, symmetry 3, slip wall 4,
    # no-slip wall 5, user_bc 6 (Source/PeleC.H:49-57)
    "inflow_lo_outflow_hi": ((1, 0, 0), (2, 0, 0)),
    "user_hi_walls": ((4, 3, 0), (6, 5, 0)),
    "inflow_everywhere": ((1, 1, 1), (1, 6, 1)),
}


@pytest.mark.parametrize("bc", sorted(BCS))
@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("ppm", [1, 0])
def test_oracle_equals_reference_build_with_domain_boundaries(bc, nspec, ppm):
    """A box filling its domain, so that every face plane of the box is a domain face:
    the boundary-condition overrides of pc_cmpflx and the low-order recomputation of
    inflow / user_bc faces (Source/Godunov.cpp:6-55, :440-468)."""
    if not pyoracle.ref_available(nspec):
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    p = wl.random_patch((5, 4, 6), 211, eos if nspec == 9 else None)
    ref = pyoracle.reference(nspec)
    ref.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    dt = 0.3 * ref.estdt(p.lo, p.hi, p.fab, p.dx)
    bclo, bchi = BCS[bc]
    prm = abi.make_params(p.dx, dt, nspec, p.lo, p.hi, bclo, bchi, ppm_type=ppm)
    a, fa = o.hydro_box(prm, p.lo, p.hi, p.fab)
    b, fb = ref.hydro_box(prm, p.lo, p.hi, p.fab)
    np.testing.assert_array_equal(a.data, b.data)
    for d in range(3):
        np.testing.assert_array_equal(fa[d].data, fb[d].data)


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("seed", [401, 402])
def test_oracle_equals_reference_build_hybrid_weno(scheme, nspec, seed):
    """PPM with hybrid WENO edge values (Source/PPM.cpp:120-172, Source/WENO.H):
    WENO-JS5 (0), WENO-Z5 (1), WENO-Z7 (2), WENO-Z3 (3)."""
    if not pyoracle.ref_available(nspec):
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    p = wl.random_patch((6, 5, 7), seed, eos if nspec == 9 else None)
    ref = pyoracle.reference(nspec)
    ref.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    dt = 0.3 * ref.estdt(p.lo, p.hi, p.fab, p.dx)
    prm = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=1)
    prm.use_hybrid_weno = 1
    prm.weno_scheme = scheme
    a, fa = o.hydro_box(prm, p.lo, p.hi, p.fab)
    b, fb = ref.hydro_box(prm, p.lo, p.hi, p.fab)
    np.testing.assert_array_equal(a.data, b.data)
    for d in range(3):
        np.testing.assert_array_equal(fa[d].data, fb[d].data)
    prm.use_hybrid_weno = 0
    c, _ = o.hydro_box(prm, p.lo, p.hi, p.fab)
    assert not np.array_equal(a.data, c.data)  # the WENO branch was taken
