"""GPU tests of the batched form and of the level loop around the hydro path:
reference golden vectors, uneven box batches, fused levels, multi-step advances with
the CFL timestep and the temperature Newton solve, CUDA-graph replay, ghost filling."""
import glob
import os

import numpy as np
import pytest

from common import FP64_TOL, eos9, gpu_zeros, oracle, rel_err, to_cpu, to_gpu
from particleclem_b200 import abi, hydro, workloads as wl
from particleclem_b200.level import LevelStepper
from test_oracle_golden import GOLDEN, load_case

NG = abi.NGROW

pytestmark = pytest.mark.gpu
BIG = 1 << 30


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_gpu_fp64_matches_reference_golden(path):
    z, eos, lo, hi, uin, prm = load_case(path)
    hydro.init(0)
    hydro.set_eos(eos)
    nv = abi.nvar(eos.nspec)
    g_in = to_gpu(uin)
    g_out = gpu_zeros(nv, lo, hi)
    flx = [gpu_zeros(nv, *abi.nodes(lo, hi, d)) for d in range(3)]
    hydro.hydro_box(prm, lo, hi, g_in, g_out, flx)
    np.testing.assert_array_equal(to_cpu(g_out), z["hydro_source"])
    for d in range(3):
        np.testing.assert_array_equal(to_cpu(flx[d]), z[f"flx{d}"])


def _patches(nspec, edges, seed):
    eos = eos9() if nspec == 9 else None
    return [wl.random_patch(e, seed + i, eos) for i, e in enumerate(edges)]


@pytest.mark.parametrize("nspec", [1, 9])
@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP64_FAST, abi.PREC_MIXED])
def test_uneven_batch_equals_single_boxes(nspec, prec):
    """Boxes of different sizes and dt in one pcg_hydro_boxes call give exactly the
    per-box results (no cross-box coupling), and the FP64 form equals the oracle."""
    eos = wl.GammaLaw() if nspec == 1 else eos9()
    hydro.init(0)
    hydro.set_eos(eos)
    o = oracle()
    o.set_eos(eos)
    patches = _patches(nspec, [(8, 5, 6), (3, 9, 4), (12, 7, 5), (6, 6, 6)], 40)
    nv = abi.nvar(nspec)
    boxes, outs, ins, dts = [], [], [], []
    for p in patches:
        dt = (0.2 + 0.1 * len(dts)) * o.estdt(p.lo, p.hi, p.fab, p.dx)
        dts.append(dt)
        uin = to_gpu(p.fab)
        out = gpu_zeros(nv, p.lo, p.hi)
        ins.append(uin)
        outs.append(out)
        boxes.append(hydro.make_box(p.lo, p.hi, uin, out, p.dx, dt))
    prm = abi.make_params((1, 1, 1), 0.0, nspec, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0), precision_mode=prec)
    hydro.hydro_boxes(prm, boxes)
    for p, dt, uin, out in zip(patches, dts, ins, outs):
        single = gpu_zeros(nv, p.lo, p.hi)
        prm1 = abi.make_params(p.dx, dt, nspec, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0), precision_mode=prec)
        hydro.hydro_box(prm1, p.lo, p.hi, uin, single)
        got = to_cpu(out)
        np.testing.assert_array_equal(got, to_cpu(single))
        if prec == abi.PREC_FP64:
            ref, _ = o.hydro_box(prm1, p.lo, p.hi, p.fab)
            np.testing.assert_array_equal(got, ref.data)


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_fused_level_equals_per_box(prec):
    """A level cut into boxes advanced as one fused region gives the per-box results
    bit for bit (results do not depend on the box decomposition)."""
    lev = wl.flame(n=24, box=8)
    hydro.init(0)
    hydro.set_eos(lev.eos)
    st_f = LevelStepper(lev, precision=prec, fuse=True)
    st_b = LevelStepper(lev, precision=prec, fuse=False)
    assert st_f.plan.info()["nregions"] == 1 and st_b.plan.info()["nregions"] == 27
    import torch

    dt = torch.full((1,), 2e-8, dtype=torch.float64, device="cuda")
    st_f.plan.hydro(dt)
    st_b.plan.hydro(dt)
    if prec == abi.PREC_FP64:
        np.testing.assert_array_equal(to_cpu(st_f.hsrc), to_cpu(st_b.hsrc))
    else:
        # the FP32 pressure offset is rho*R/W*T of each region's first cell, so a
        # fused level and its boxes agree to FP32 rounding of the offset only
        l1, linf = rel_err(to_cpu(st_f.hsrc), to_cpu(st_b.hsrc))
        assert l1 <= 1e-8 and linf <= 1e-7, (l1, linf)
    if prec == abi.PREC_FP64:
        o = oracle()
        o.set_eos(lev.eos)
        prm = abi.make_params(lev.dx, 2e-8, 9, lev.domlo, lev.domhi, lev.bclo, lev.bchi)
        hs = to_cpu(st_f.hsrc)
        for lo, hi in lev.boxes[:4]:
            ref, _ = o.hydro_box(prm, lo, hi, lev.box_fab(lo, hi))
            sub = hs[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
            np.testing.assert_array_equal(sub, ref.data)
    st_f.close()
    st_b.close()


def _oracle_steps(lev, nsteps, cfl=0.3):
    """The level loop on the CPU oracle: ghost fill, estdt, per-box hydro, update."""
    o = oracle()
    o.set_eos(lev.eos)
    lev = wl.Level(lev.eos, lev.dx, lev.domlo, lev.domhi, lev.bclo, lev.bchi, lev.state.copy(), list(lev.boxes),
                   lev.periodic)
    dts = []
    for _ in range(nsteps):
        lev.fill_ghosts()
        fabs = [(lo, hi, lev.box_fab(lo, hi)) for lo, hi in lev.boxes]
        dt = cfl * min(o.estdt(lo, hi, f, lev.dx) for lo, hi, f in fabs)
        prm = abi.make_params(lev.dx, dt, lev.nspec, lev.domlo, lev.domhi, lev.bclo, lev.bchi)
        new = lev.state.copy()
        g = abi.NGROW
        for lo, hi, f in fabs:
            hs, _ = o.hydro_box(prm, lo, hi, f)
            sn = o.update_state(lo, hi, f, hs, dt)
            new[:, lo[2] + g:hi[2] + g + 1, lo[1] + g:hi[1] + g + 1, lo[0] + g:hi[0] + g + 1] = sn.view(lo, hi)
        lev.state = new
        dts.append(dt)
    lev.fill_ghosts()
    return lev.state, dts


@pytest.mark.parametrize("name", ["sod", "flame"])
def test_level_steps_fp64_equal_oracle(name):
    """Three full level steps (ghost fill, CFL dt on the device, hydro, update with
    the T(e) Newton solve) in the plain FP64 form equal the oracle's level loop."""
    lev = wl.sod(16) if name == "sod" else wl.flame(n=16, box=8)
    ref_state, dts = _oracle_steps(lev, 3)
    st = LevelStepper(lev, precision=abi.PREC_FP64, fuse=(name == "flame"))
    got_dts = []
    for _ in range(3):
        st.step()
        got_dts.append(float(st.dt.item()))
    st.fill()
    got = st.host_state()
    assert got_dts == dts
    np.testing.assert_array_equal(got, ref_state)
    st.close()


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP64_FAST, abi.PREC_MIXED])
def test_fused_step_tail_equals_separate_kernels(prec):
    """pcg_plan_advance (flux divergence, update, computeTemp and the next CFL timestep in
    one pass) against hydro + update + estdt as separate launches, over three steps. The
    plain FP64 form is bit-identical. With FMA contraction the timestep expression may
    round differently in the fused kernel (last bit), and in the FP32 stages of the mixed
    form such a difference can flip a limiter branch in a few cells: bounds of FP64
    rounding for the FMA form and of FP32 resolution for the mixed form."""
    lev = wl.flame(n=16, box=8)
    a = LevelStepper(lev, precision=prec, fuse=True, fused_tail=True)
    b = LevelStepper(lev, precision=prec, fuse=True, fused_tail=False)
    for _ in range(3):
        a.step()
        b.step()
        assert float(a.dt.item()) == float(b.dt.item()) or prec != abi.PREC_FP64
    sa, sb = a.host_state(), b.host_state()
    if prec == abi.PREC_FP64:
        np.testing.assert_array_equal(sa, sb)
    else:
        l1, linf = rel_err(sa[:, 4:-4, 4:-4, 4:-4], sb[:, 4:-4, 4:-4, 4:-4])
        l1_tol, linf_tol = (1e-12, 1e-10) if prec == abi.PREC_FP64_FAST else (1e-9, 1e-6)
        assert l1 <= l1_tol and linf <= linf_tol, (l1, linf)
    a.close()
    b.close()


def test_graph_replay_equals_eager_steps():
    lev = wl.flame(n=16, box=8)
    a = LevelStepper(lev, precision=abi.PREC_MIXED, fuse=True)
    b = LevelStepper(lev, precision=abi.PREC_MIXED, fuse=True)
    a.capture()  # the capture warm-up runs one eager step
    b.step()
    for _ in range(2):
        a.replay()
        b.step()
    np.testing.assert_array_equal(a.host_state(), b.host_state())
    a.close()
    b.close()


@pytest.mark.parametrize("depth,valid_only", [(2, False), (3, True)])
def test_host_pipeline_equals_serial_steps(depth, valid_only):
    """Pipelined host->device->host advances equal one-at-a-time steps bit for bit, for
    inputs that differ per submission and with more submissions than device slots; with
    ``valid_only`` the valid rows cross the bus and the other ghost cells of the output
    are left untouched."""
    import torch

    from particleclem_b200.level import HostPipeline

    levs = [wl.flame(n=16, box=8, seed=s) for s in (2, 3, 4)]
    ins = [torch.from_numpy(L.state).pin_memory() for L in levs]
    if valid_only:  # the ghost cells of the inputs must not matter
        for t in ins:
            t[:, :NG] = -7.0
    order = [0, 1, 2, 1, 0, 2, 2]
    outs = [torch.full_like(ins[0], 3.5).pin_memory() for _ in order]
    pipe = HostPipeline(levs[0], depth=depth, valid_only=valid_only, precision=abi.PREC_MIXED, fuse=True)
    for i, j in enumerate(order):
        pipe.submit(ins[j], outs[i])
    pipe.synchronize()
    ref = LevelStepper(levs[0], precision=abi.PREC_MIXED, fuse=True)
    for i, j in enumerate(order):
        ref.load_state(torch.from_numpy(levs[j].state).to(ref.dev))
        ref.step()
        got, want = outs[i].numpy(), ref.host_state()
        if valid_only:
            rows = (slice(None), slice(NG, -NG), slice(NG, -NG), slice(None))
            np.testing.assert_array_equal(got[rows], want[rows])
            ghost = np.ones(got.shape, bool)
            ghost[:, NG:-NG, NG:-NG, :] = False  # the valid rows, x ghost cells included
            assert (got[ghost] == 3.5).all()
        else:
            np.testing.assert_array_equal(got, want)
    pipe.close()
    ref.close()


@pytest.mark.parametrize("whole_rows", [False, True])
def test_copy_cells_round_trip(whole_rows):
    """pcg_copy_cells moves exactly the cells of the given box, host -> device -> host,
    for FABs of different extents and origins (strided rows), and for boxes spanning
    whole rows of both FABs (slices copied as contiguous runs)."""
    import torch

    from particleclem_b200 import hydro

    rng = np.random.default_rng(3)
    src = torch.from_numpy(rng.standard_normal((5, 9, 8, 7))).pin_memory()
    if whole_rows:
        dev = abi.Fab(torch.zeros((5, 12, 8, 7), dtype=torch.float64, device="cuda"), (0, 0, -2))
        lo, hi = (0, 0, 1), (6, 7, 5)
    else:
        dev = abi.Fab(torch.zeros((5, 12, 11, 10), dtype=torch.float64, device="cuda"), (-3, -2, -1))
        lo, hi = (1, 0, 2), (4, 5, 6)
    back = torch.zeros((5, 9, 8, 7), dtype=torch.float64).pin_memory()
    hydro.copy_cells(abi.Fab(src, (0, 0, 0)), dev, lo, hi)
    hydro.copy_cells(dev, abi.Fab(back, (0, 0, 0)), lo, hi)
    torch.cuda.synchronize()
    sel = (slice(None), slice(lo[2], hi[2] + 1), slice(lo[1], hi[1] + 1), slice(lo[0], hi[0] + 1))
    b = back.numpy()
    np.testing.assert_array_equal(b[sel], src.numpy()[sel])
    mask = np.ones(b.shape, bool)
    mask[sel] = False
    assert (b[mask] == 0).all()
    d = dev.data.cpu().numpy()
    assert np.count_nonzero(d) == np.count_nonzero(src.numpy()[sel])


def test_mixed_level_step_error_vs_fp64():
    lev = wl.flame(n=32, box=16)
    a = LevelStepper(lev, precision=abi.PREC_FP64, fuse=False)
    b = LevelStepper(lev, precision=abi.PREC_MIXED, fuse=True)
    c = LevelStepper(lev, precision=abi.PREC_FP64_FAST, fuse=True)
    for s in (a, b, c):
        s.step()
    g = abi.NGROW
    A, B, Cc = (s.host_state()[:, g:-g, g:-g, g:-g] for s in (a, b, c))
    l1, _ = rel_err(B, A)
    assert l1 <= 1e-6, l1
    l1, linf = rel_err(Cc, A)
    assert l1 <= FP64_TOL and linf <= FP64_TOL, (l1, linf)
    for s in (a, b, c):
        s.close()


def test_fill_ghosts_matches_numpy():
    import torch

    lev = wl.turbulence(n=8, box=8, seed=3, kmax=2)
    s = lev.state.copy()
    s[:, :4] = -1.0
    s[:, :, :, -4:] = -2.0
    st = abi.Fab(torch.from_numpy(s.copy()).cuda(), lev.fab.lo)
    hydro.init(0)
    hydro.fill_ghosts(st, lev.domlo, lev.domhi, (True, False, True))
    wl.fill_ghosts(s, (True, False, True))
    np.testing.assert_array_equal(to_cpu(st), s)


def test_errors_are_reported():
    from particleclem_b200.native import PcgError

    p = wl.random_patch((4, 4, 4), 1)
    hydro.init(0)
    hydro.set_eos(wl.GammaLaw())
    uin = to_gpu(p.fab)
    out = gpu_zeros(8, p.lo, p.hi)
    prm = abi.make_params(p.dx, 1e-3, 1, (-BIG,) * 3, (BIG,) * 3, (0, 0, 0), (0, 0, 0))
    small = abi.Fab(uin.data[:, 1:-1, 1:-1, 1:-1].contiguous(), (-3, -3, -3))  # only 3 ghosts
    with pytest.raises(PcgError) as e:
        hydro.hydro_box(prm, p.lo, p.hi, small, out)
    assert e.value.code == -1
    prm.plm_iorder = 3
    prm.ppm_type = 0
    with pytest.raises(PcgError):
        hydro.hydro_box(prm, p.lo, p.hi, uin, out)
