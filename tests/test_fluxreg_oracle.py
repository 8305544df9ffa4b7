"""The coarse/fine oracle (oracle/fluxreg_oracle.py) on two-level advances: one coarse
step of a periodic level and `ratio` fine substeps of the boxes above it, with the flux
register filled from the exported hydro fluxes (Source/Hydro.cpp:281-287), reflux
(Source/PeleC.cpp:1403-1414) and average-down. Conservation pins the algorithm: after
reflux and average-down the coarse level holds exactly (to rounding) the mass, momentum
and energy it started with, as a single-level periodic step does; without reflux it does
not. Also the register's face set (domain wrap, faces between fine boxes) and the
library's refusal of bad register arguments, before any device work."""
import ctypes as C

import numpy as np
import pytest

import fluxreg_oracle as fro
from common import oracle
from particleclem_b200 import abi, native, workloads as wl

NG = abi.NGROW
CASES = {
    # coarse edge, ratio, fine boxes (fine index space)
    "one_box": (12, 2, [((6, 4, 8), (17, 19, 15))]),
    "wrap_and_abutting": (12, 2, [((0, 8, 4), (7, 15, 11)), ((8, 8, 4), (15, 15, 11))]),
    "ratio4": (12, 4, [((16, 12, 20), (27, 23, 31))]),
    # the coarse level in four boxes (CrseAdd per coarse box), the fine box across them
    "coarse_boxes": (12, 2, [((8, 8, 4), (15, 15, 11))]),
}
COARSE_SPLIT = {"coarse_boxes": 2}  # boxes per direction in x and y
CONSERVED = (abi.URHO, abi.UMX, abi.UMY, abi.UMZ, abi.UEDEN)


def inject(crse_state, n, lo, hi, ratio, ng=NG):
    """A fine FAB over grow([lo, hi], ng) whose cells copy the (periodic) coarse cell
    they lie in: conservative piecewise-constant prolongation."""
    nv = crse_state.shape[0]
    glo, ghi = abi.grow(lo, hi, ng)
    I = np.arange(glo[0], ghi[0] + 1) // ratio % n + NG
    J = np.arange(glo[1], ghi[1] + 1) // ratio % n + NG
    K = np.arange(glo[2], ghi[2] + 1) // ratio % n + NG
    data = crse_state[:, K[:, None, None], J[None, :, None], I[None, None, :]]
    return abi.Fab(np.ascontiguousarray(data.reshape(nv, len(K), len(J), len(I))), glo)


def fill_fine(s0, n, ratio, fine, fstate, b):
    """The grown FAB of fine box b: its valid cells and every ghost cell that lies in a
    fine box (periodic images included) from the fine states, the rest injected from the
    old coarse state (as FillPatch takes fine data where it exists)."""
    lo, hi = fine[b]
    fab = inject(s0, n, lo, hi, ratio)
    glo, ghi = abi.grow(lo, hi, NG)
    N = n * ratio
    shifts = [(a, c, e) for a in (-N, 0, N) for c in (-N, 0, N) for e in (-N, 0, N)]
    for b2, (lo2, hi2) in enumerate(fine):
        for sh in shifts:
            olo = [max(glo[d], lo2[d] + sh[d]) for d in range(3)]
            ohi = [min(ghi[d], hi2[d] + sh[d]) for d in range(3)]
            if any(olo[d] > ohi[d] for d in range(3)):
                continue
            src = fstate[b2][:, olo[2] - sh[2] - lo2[2]:ohi[2] - sh[2] - lo2[2] + 1,
                             olo[1] - sh[1] - lo2[1]:ohi[1] - sh[1] - lo2[1] + 1,
                             olo[0] - sh[0] - lo2[0]:ohi[0] - sh[0] - lo2[0] + 1]
            fab.view(olo, ohi)[...] = src
    return fab


class CpuLevels:
    """Hydro and update on the CPU oracle; register and average-down from the oracle."""

    def __init__(self, eos):
        self.o = oracle()
        self.o.set_eos(eos)
        self.Register = fro.FluxRegister
        self.average_down = fro.average_down

    def hydro(self, prm, lo, hi, fab):
        hs, flx = self.o.hydro_box(prm, lo, hi, fab)
        return hs, flx

    def update(self, lo, hi, fab, hs, dt):
        return self.o.update_state(lo, hi, fab, hs, dt).view(lo, hi).copy()


def two_level(case, seed=11, backend=None, do_reflux=True, record=None):
    """One coarse step and `ratio` fine substeps; returns (coarse state before, after)."""
    n, ratio, fine = CASES[case]
    eos = wl.GammaLaw()
    be = backend or CpuLevels(eos)
    p = wl.random_patch((n, n, n), seed, None)
    dom = ((0, 0, 0), (n - 1, n - 1, n - 1))
    lev = wl.Level(eos, p.dx, dom[0], dom[1], (0, 0, 0), (0, 0, 0), p.fab.data.copy(), [dom], (True, True, True))
    lev.fill_ghosts()
    s0 = lev.state.copy()
    dx_c = tuple(p.dx)
    dx_f = tuple(d / ratio for d in dx_c)
    vol_c = dx_c[0] * dx_c[1] * dx_c[2]
    big = 1 << 30
    o = oracle()
    o.set_eos(eos)
    dt_c = 0.3 * o.estdt(dom[0], dom[1], lev.box_fab(*dom), dx_c)
    reg = be.Register(abi.nvar(1), dom[0], dom[1], (1, 1, 1), ratio, fine)
    # coarse step, box by box
    prm_c = abi.make_params(dx_c, dt_c, 1, dom[0], dom[1], (0, 0, 0), (0, 0, 0))
    m = COARSE_SPLIT.get(case, 1)
    e = n // m
    cboxes = [((a * e, b * e, 0), (a * e + e - 1, b * e + e - 1, n - 1)) for b in range(m) for a in range(m)]
    new_c = np.empty_like(lev.fab.view(*dom))
    for lo, hi in cboxes:
        hs, flx = be.hydro(prm_c, lo, hi, lev.box_fab(lo, hi))
        reg.crse_add(lo, hi, flx, dt_c)
        if record is not None:
            record.append(("crse", lo, hi, flx, dt_c))
        new_c[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = be.update(lo, hi, lev.box_fab(lo, hi), hs, dt_c)
    # fine substeps: ghost cells from the fine boxes where they exist, else injected from
    # the old coarse state
    dt_f = dt_c / ratio
    prm_f = abi.make_params(dx_f, dt_f, 1, (-big,) * 3, (big,) * 3, (0, 0, 0), (0, 0, 0))
    fstate = {b: inject(s0, n, lo, hi, ratio).view(lo, hi).copy() for b, (lo, hi) in enumerate(fine)}
    for _ in range(ratio):
        fabs = [fill_fine(s0, n, ratio, fine, fstate, b) for b in range(len(fine))]
        for b, (lo, hi) in enumerate(fine):
            fab = fabs[b]
            hs_f, flx_f = be.hydro(prm_f, lo, hi, fab)
            reg.fine_add(lo, hi, flx_f, dt_f)
            if record is not None:
                record.append(("fine", lo, hi, flx_f, dt_f))
            fstate[b] = be.update(lo, hi, fab, hs_f, dt_f)
    crse = abi.Fab(s0.copy(), (-NG,) * 3)
    crse.view(*dom)[...] = new_c
    if record is not None:
        record.append(("state", crse.data.copy(), fstate, vol_c))
    if do_reflux:
        reg.reflux(crse, vol_c)
    for b, (lo, hi) in enumerate(fine):
        be.average_down(abi.Fab(fstate[b], lo), crse, lo, hi, ratio, abi.nvar(1))
    return abi.Fab(s0, (-NG,) * 3).view(*dom), crse.view(*dom), reg


def totals(valid):
    return np.array([valid[c].sum() for c in CONSERVED])


@pytest.mark.parametrize("case", sorted(CASES))
def test_two_level_step_conserves_with_reflux(case):
    before, after, _ = two_level(case)
    t0, t1 = totals(before), totals(after)
    scale = np.array([np.abs(before[c]).sum() for c in CONSERVED])
    assert np.all(np.abs(t1 - t0) <= 1e-13 * scale), (case, (t1 - t0) / scale)


def test_two_level_step_without_reflux_loses_conservation():
    before, after, _ = two_level("one_box", do_reflux=False)
    scale = np.array([np.abs(before[c]).sum() for c in CONSERVED])
    assert np.max(np.abs(totals(after) - totals(before)) / scale) > 1e-10


def test_register_faces():
    """Faces on the coarse/fine boundary only: for one box, its surface in coarse faces;
    two abutting boxes lose their shared faces; faces across the periodic boundary land on
    the wrapped coarse cell."""
    n, r, fine = CASES["one_box"]
    reg = fro.FluxRegister(8, (0, 0, 0), (n - 1,) * 3, (1, 1, 1), r, fine)
    e = [(hi[d] - lo[d] + 1) // r for lo, hi in fine for d in range(3)]
    assert len(reg.entries) == 2 * (e[0] * e[1] + e[1] * e[2] + e[0] * e[2])
    n, r, fine = CASES["wrap_and_abutting"]
    reg = fro.FluxRegister(8, (0, 0, 0), (n - 1,) * 3, (1, 1, 1), r, fine)
    # the union is 8 x 4 x 4 coarse cells
    assert len(reg.entries) == 2 * (8 * 4 + 4 * 4 + 8 * 4)
    assert any(x["c"][0] == n - 1 and x["dir"] == 0 for x in reg.entries)  # wrapped below x = 0
    reg_np = fro.FluxRegister(8, (0, 0, 0), (n - 1,) * 3, (0, 1, 1), r, fine)
    assert len(reg_np.entries) == len(reg.entries) - 4 * 4  # no faces on the x domain face


def _create(ncomp, domlo, domhi, periodic, ratio, boxes):
    lo = [v for b in boxes for v in b[0]]
    hi = [v for b in boxes for v in b[1]]
    h = C.c_void_p()
    return native.load().pcg_fluxreg_create(ncomp, abi.ivec(domlo), abi.ivec(domhi), abi.ivec(periodic), ratio,
                                            len(boxes), (C.c_int32 * len(lo))(*lo), (C.c_int32 * len(hi))(*hi),
                                            C.byref(h))


def test_fluxreg_argument_errors():
    """Misaligned, overlapping or out-of-domain fine boxes and bad ratios are refused with
    PCG_EINVAL before any device work."""
    dom = ((0, 0, 0), (11, 11, 11))
    assert _create(8, *dom, (1, 1, 1), 2, [((1, 0, 0), (4, 3, 3))]) == -1  # lo not on the ratio grid
    assert "aligned" in native.load().pcg_last_error().decode()
    assert _create(8, *dom, (1, 1, 1), 2, [((0, 0, 0), (4, 3, 3))]) == -1  # hi + 1 not on it
    assert _create(8, *dom, (1, 1, 1), 2, [((0, 0, 0), (7, 7, 7)), ((4, 4, 4), (11, 11, 11))]) == -1
    assert "overlap" in native.load().pcg_last_error().decode()
    assert _create(8, *dom, (1, 1, 1), 2, [((20, 0, 0), (27, 7, 7))]) == -1  # outside the coarse domain
    assert _create(8, *dom, (1, 1, 1), 1, [((0, 0, 0), (7, 7, 7))]) == -1
    assert _create(0, *dom, (1, 1, 1), 2, [((0, 0, 0), (7, 7, 7))]) == -1


def test_average_down_argument_errors():
    """pcg_average_down refuses a fine box off the ratio grid, a bad ratio or component
    count, and arrays that do not cover the boxes, before any device work."""
    lib = native.load()
    fine = abi.Fab(np.zeros((8, 8, 8, 8)), (0, 0, 0))
    crse = abi.Fab(np.zeros((8, 4, 4, 4)), (0, 0, 0))

    def rc(flo, fhi, ratio=2, nc=8, f=fine, c=crse):
        return lib.pcg_average_down(C.byref(abi.array4(f)), C.byref(abi.array4(c)), abi.ivec(flo), abi.ivec(fhi),
                                    ratio, nc, None)

    assert rc((1, 0, 0), (6, 7, 7)) == -1
    assert "aligned" in lib.pcg_last_error().decode()
    assert rc((0, 0, 0), (7, 7, 7), ratio=1) == -1
    assert rc((0, 0, 0), (7, 7, 7), nc=0) == -1
    assert rc((0, 0, 0), (7, 7, 7), nc=9) == -1  # more components than the arrays hold
    assert rc((0, 0, 0), (15, 7, 7)) == -1  # the fine array does not cover the box
    small = abi.Fab(np.zeros((8, 2, 2, 2)), (0, 0, 0))
    assert rc((0, 0, 0), (7, 7, 7), c=small) == -1  # the coarse array does not cover it
