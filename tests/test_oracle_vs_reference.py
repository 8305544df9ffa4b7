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


@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("ppm", [1, 0])
def test_oracle_equals_reference_build_srctoprim_and_umeth_with_sources(nspec, ppm):
    """pc_srctoprim (Source/Hydro.H:14-68) of non-zero sources, then pc_umeth_3D
    (Source/Godunov.cpp:59-476) with those primitive sources, so that the hdt * srcQ terms
    of pc_transdd (Source/Godunov.H:639-845) are taken: final fluxes, the face states qec
    (components GDU..GDGAME) and p div u agree bit for bit, and pc_umdrv with the same
    srcQ too."""
    if not pyoracle.ref_available(nspec):
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    from common import random_sources

    eos = wl.GammaLaw() if nspec == 1 else eos9()
    p = wl.random_patch((6, 5, 4), 611 + nspec, eos if nspec == 9 else None)
    ref = pyoracle.reference(nspec)
    ref.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    g4lo, g4hi = abi.grow(p.lo, p.hi, 4)
    dt = 0.3 * ref.estdt(p.lo, p.hi, p.fab, p.dx)
    prm = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), ppm_type=ppm)
    q, qa = ref.ctoprim(g4lo, g4hi, p.fab)
    src = random_sources(p.fab, 7 + nspec, scale=20.0 if nspec == 1 else 1e4)
    sq_ref = ref.srctoprim(g4lo, g4hi, q, qa, src)
    sq_orc = o.srctoprim(g4lo, g4hi, q, qa, src)
    np.testing.assert_array_equal(sq_orc.data, sq_ref.data)
    assert np.abs(sq_ref.data).max() > 0
    fa, ga, pa = o.umeth(prm, p.lo, p.hi, q, qa, sq_orc)
    fb, gb, pb = ref.umeth(prm, p.lo, p.hi, q, qa, sq_ref)
    for d in range(3):
        np.testing.assert_array_equal(fa[d].data, fb[d].data)
        np.testing.assert_array_equal(ga[d].data[1:], gb[d].data[1:])
    np.testing.assert_array_equal(pa.data, pb.data)
    f0, _, _ = o.umeth(prm, p.lo, p.hi, q, qa, None)
    assert not np.array_equal(f0[0].data, fa[0].data)  # the sources entered the fluxes
