"""GPU checks at the full sizes of the measured workloads, through properties that do not
depend on size: one step of a closed (periodic) level conserves total mass, momentum,
energy and every species' mass to round-off, in the plain FP64 and the mixed form (each
face flux is stored once and read by both of its cells, so the flux divergence telescopes
over the domain; the reference's own check is Tests/test_masscons.py, rtol 1e-13). The
256^3 periodic turbulence level (64 boxes of 64^3, one species; PPM and PLM) and the 128^3
flame level (64 boxes of 32^3, 9 species) closed in z (PPM and hybrid WENO-Z5)."""
import pytest
import torch

from particleclem_b200 import abi, workloads as wl
from particleclem_b200.level import LevelStepper

pytestmark = pytest.mark.gpu
G = abi.NGROW


def _closed_flame():
    lev = wl.flame(n=128, box=32, seed=2)
    lev.periodic = (True, True, True)
    lev.bclo = lev.bchi = (abi.BC_INTERIOR,) * 3
    lev.fill_ghosts()
    return lev


def _totals(st):
    v = st.state.data[:, G:-G, G:-G, G:-G]
    return v.sum(dim=(1, 2, 3)), v.abs().sum(dim=(1, 2, 3))


CASES = [("turbulence_256", {}), ("flame_128_closed", {}), ("turbulence_256_plm", {"ppm_type": 0}),
         ("flame_128_closed_weno_z5", {"use_hybrid_weno": True, "weno_scheme": 1})]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_one_step_of_a_closed_level_conserves(name, kw, prec):
    lev = wl.turbulence(n=256, box=64, seed=4) if name.startswith("turbulence") else _closed_flame()
    st = LevelStepper(lev, precision=prec, fuse=prec == abi.PREC_MIXED, **kw)
    before, scale = _totals(st)
    st.step()
    torch.cuda.synchronize()
    after, _ = _totals(st)
    comps = [abi.URHO, abi.UMX, abi.UMY, abi.UMZ, abi.UEDEN] + list(range(abi.UFS, abi.UFS + lev.nspec))
    if lev.nspec == 1:
        comps = comps[:5]
    # momentum components are compared against the momentum magnitude (their totals can be ~0)
    mom = float(scale[abi.UMX:abi.UMZ + 1].sum())
    for c in comps:
        ref = mom if c in (abi.UMX, abi.UMY, abi.UMZ) else float(scale[c])
        drift = abs(float(after[c] - before[c]))
        assert drift <= 1e-12 * ref, (name, c, drift, ref)
    assert float(st.dt.item()) > 0.0
    st.close()


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_fused_level_equals_per_box_at_full_size(prec):
    """The 128^3 flame level advanced as one fused region (whose final-flux stage runs
    its directions interleaved in z-slabs and whose prep, flux0 and flux2 launches run in
    reverse order, the launch order of regions larger than L2) gives the hydro source of
    the 64 boxes advanced as separate regions bit for bit in the plain FP64 form (box
    independence: every output of a box depends on grow(box, 4) only, and the plain FP64
    per-box form equals the oracle). In the mixed form, whose FP32 pressure offset p0 is
    a per-region constant, within the mixed form's resolution."""
    lev = wl.flame(n=128, box=32, seed=2)
    out = []
    for fuse in (False, True):
        st = LevelStepper(lev, precision=prec, fuse=fuse, fused_tail=False)
        st.fill()
        st.plan.estdt(st.cfl, st.dt)
        st.plan.hydro(st.dt)
        torch.cuda.synchronize()
        out.append(st.hsrc.data.clone())
        st.close()
        del st
        torch.cuda.empty_cache()
    if prec == abi.PREC_FP64:
        assert torch.equal(out[0], out[1])
    else:
        from common import rel_errors

        l1, _ = rel_errors(out[1].cpu().numpy(), out[0].cpu().numpy(), lev.nspec)
        assert float(l1.max()) < 5e-4, l1  # the hydro-source bound of the mixed form
