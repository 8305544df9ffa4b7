"""The coarse/fine calls on the GPU (pcg_fluxreg_*, pcg_average_down) against the CPU
oracle (oracle/fluxreg_oracle.py): the same two-level advance (one coarse step of a
periodic level, `ratio` fine substeps, reflux, average-down; tests/test_fluxreg_oracle.py)
with the hydro fluxes from the GPU (pcg_hydro_box with flux export, FP64) and the
register on the device ends bit for bit on the oracle's coarse state, which conserves
mass, momentum and energy; the register calls replayed on the oracle's own fluxes give
the oracle's state bit for bit; a reset register accumulates from zero again."""
import numpy as np
import pytest

from common import gpu_zeros, to_cpu, to_gpu
from particleclem_b200 import abi, amr, hydro, workloads as wl
from test_fluxreg_oracle import CASES, CONSERVED, CpuLevels, totals, two_level

pytestmark = pytest.mark.gpu


class _GpuRegister:
    """amr.FluxRegister behind the oracle register's interface: host FABs in, host FABs
    out (fluxes already on the device are passed through)."""

    def __init__(self, *args):
        self.r = amr.FluxRegister(*args)

    def _dev(self, flx):
        return [f if not isinstance(f.data, np.ndarray) else to_gpu(f) for f in flx]

    def crse_add(self, lo, hi, flx, dt):
        self.r.crse_add(lo, hi, self._dev(flx), dt)

    def fine_add(self, lo, hi, flx, dt):
        self.r.fine_add(lo, hi, self._dev(flx), dt)

    def reflux(self, crse, vol):
        g = to_gpu(crse)
        self.r.reflux(g, vol)
        crse.data[...] = to_cpu(g)


def _gpu_average_down(fine, crse, lo, hi, ratio, nc):
    g = to_gpu(crse)
    amr.average_down(to_gpu(fine), g, lo, hi, ratio, nc)
    crse.data[...] = to_cpu(g)


class GpuLevels(CpuLevels):
    """Hydro on the GPU (FP64, fluxes exported on the device), the register and
    average-down on the GPU; the state update from the oracle (the GPU update equals it
    bit for bit, tests/test_gpu_batched.py)."""

    def __init__(self, eos):
        super().__init__(eos)
        hydro.init(0)
        hydro.set_eos(eos)
        self.Register = _GpuRegister
        self.average_down = _gpu_average_down

    def hydro(self, prm, lo, hi, fab):
        uin = to_gpu(fab)
        out = gpu_zeros(abi.nvar(1), lo, hi)
        flx = [gpu_zeros(abi.nvar(1), *abi.nodes(lo, hi, d)) for d in range(3)]
        hydro.hydro_box(prm, lo, hi, uin, out, flx)
        return abi.Fab(to_cpu(out), tuple(lo)), flx


@pytest.mark.parametrize("case", sorted(CASES))
def test_two_level_step_equals_oracle(case):
    before, ref, _ = two_level(case)
    _, got, _ = two_level(case, backend=GpuLevels(wl.GammaLaw()))
    np.testing.assert_array_equal(got, ref)
    scale = np.array([np.abs(before[c]).sum() for c in CONSERVED])
    assert np.all(np.abs(totals(got) - totals(before)) <= 1e-13 * scale)


@pytest.mark.parametrize("case", ["wrap_and_abutting", "ratio4"])
def test_register_replay_and_reset(case):
    """The register calls of the oracle's run replayed on the device with the oracle's
    own fluxes: reflux gives the oracle's corrected state bit for bit, twice in a row
    with a reset between (accumulators restart from zero)."""
    rec = []
    _, _, oreg = two_level(case, record=rec)
    n, ratio, fine = CASES[case]
    hydro.init(0)
    reg = amr.FluxRegister(abi.nvar(1), (0, 0, 0), (n - 1,) * 3, (1, 1, 1), ratio, fine)
    assert reg.info()["faces"] == len(oreg.entries)
    state, _, vol = rec[-1][1:]
    expect = abi.Fab(state.copy(), (-abi.NGROW,) * 3)
    oreg.reflux(expect, vol)
    for rep in range(2):
        reg.reset()
        for kind, lo, hi, flx, dt in [r for r in rec if r[0] in ("crse", "fine")]:
            dflx = [to_gpu(f) for f in flx]
            (reg.crse_add if kind == "crse" else reg.fine_add)(lo, hi, dflx, dt)
        g = to_gpu(abi.Fab(state.copy(), (-abi.NGROW,) * 3))
        reg.reflux(g, vol)
        np.testing.assert_array_equal(to_cpu(g), expect.data)
    reg.close()
