"""The z-slab decomposition's host logic on CPU: slab ranges and neighbours, and the halo
exchange between two gloo ranks (and between slabs of one process) producing exactly
the ghost cells a fill of the whole level produces, for an outflow and a periodic z."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from particleclem_b200 import workloads as wl
from particleclem_b200.slab import DistComm, LocalComm, halo_planes, neighbours

NG = wl.NG


def test_slab_ranges_and_neighbours():
    assert wl.slab_range(128, 4, 2, 32) == (64, 95)
    with pytest.raises(ValueError):
        wl.slab_range(96, 2, 0, 32)
    assert neighbours(1, 0, True) == (None, None)
    assert neighbours(3, 0, False) == (None, 1) and neighbours(3, 2, False) == (1, None)
    assert neighbours(3, 0, True) == (2, 1) and neighbours(2, 1, True) == (0, 0)


class CpuSlab:
    """Host stand-in for SlabStepper's exchange surface."""

    def __init__(self, lev, nranks, rank, box):
        self.sl = wl.split_level(lev, nranks, rank, box)
        self.state = torch.from_numpy(self.sl.state.copy())
        self.down, self.up = neighbours(nranks, rank, lev.periodic[2])
        v = halo_planes(self.state)
        self.views = v
        self.sbuf = {k: torch.empty_like(v["send_" + k]) for k in ("down", "up")}
        self.rbuf = {k: torch.empty_like(v["recv_" + k]) for k in ("down", "up")}
        self.dt = torch.tensor([1.0 + rank], dtype=torch.float64)

    def fill_and_pack(self, nranks):
        st = self.state.numpy()
        wl.fill_ghosts(st, (self.sl.periodic[0], self.sl.periodic[1], self.sl.periodic[2] and nranks == 1))
        for k in ("down", "up"):
            if getattr(self, k) is not None:
                self.sbuf[k].copy_(self.views["send_" + k])

    def unpack(self):
        for k in ("down", "up"):
            if getattr(self, k) is not None:
                self.views["recv_" + k].copy_(self.rbuf[k])


def _level(periodic_z, seed=5):
    rng = np.random.default_rng(seed)
    n, nz = 6, 16
    st = rng.standard_normal((3, nz + 2 * NG, n + 2 * NG, n + 2 * NG))
    lev = wl.Level(wl.GammaLaw(), (1.0, 1.0, 1.0), (0, 0, 0), (n - 1, n - 1, nz - 1), (0, 0, 0), (0, 0, 0), st,
                   wl.tile_boxes((n, n, nz), (n, n, 4)), (True, True, periodic_z))
    ref = st.copy()
    wl.fill_ghosts(ref, lev.periodic)
    return lev, ref


def _expected(ref, sl, lev):
    k0 = sl.k0 - lev.domlo[2]
    return ref[:, k0:k0 + (sl.k1 - sl.k0 + 1) + 2 * NG]


@pytest.mark.parametrize("periodic_z", [False, True])
@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_local_exchange_equals_global_fill(periodic_z, nranks):
    lev, ref = _level(periodic_z)
    slabs = [CpuSlab(lev, nranks, r, 4) for r in range(nranks)]
    for s in slabs:
        s.fill_and_pack(nranks)
    LocalComm().exchange(slabs)
    for s in slabs:
        s.unpack()
        np.testing.assert_array_equal(s.state.numpy(), _expected(ref, s.sl, lev))
    LocalComm().min_dt(slabs)
    assert all(float(s.dt) == 1.0 for s in slabs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, nranks, port, periodic_z, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        lev, ref = _level(periodic_z)
        s = CpuSlab(lev, nranks, rank, 4)
        s.fill_and_pack(nranks)
        comm = DistComm()
        comm.exchange([s])
        s.unpack()
        ok = bool(np.array_equal(s.state.numpy(), _expected(ref, s.sl, lev)))
        comm.min_dt([s])
        out[rank] = (ok, float(s.dt))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("periodic_z", [False, True])
def test_gloo_two_ranks_exchange_equals_global_fill(periodic_z):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, _free_port(), periodic_z, out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    assert res[0] == (True, 1.0) and res[1] == (True, 1.0)


# ---- the overlapped step sequence (slab.step_overlap) with a CPU stand-in for the device
# phases: a radius-4 stencil in z (the reach of the hydro advance's grow(box, 4)) plus the
# x/y neighbours as the "hydro source", an explicit update and a CFL-like timestep. The
# interior region is advanced from valid planes only while the exchange is "in flight"
# (gloo completes it before the wait returns, but the stand-in reads nothing the exchange
# writes); the bands after the unpack. The result must equal the stand-in step of the
# whole level with a global ghost fill.
_W = np.array([0.02, -0.05, 0.1, -0.3, 0.4, 0.25, -0.12, 0.06, -0.01])


def _standin_source(u, zlo, zhi):
    """Stand-in hydro source on the valid x/y cells of the planes zlo..zhi (grown-array z
    indices) of a grown state u (comps, z, y, x), reading planes zlo-4..zhi+4 only."""
    g = NG
    h = np.zeros((u.shape[0], zhi - zlo + 1, u.shape[2] - 2 * g, u.shape[3] - 2 * g))
    for m in range(-4, 5):
        h += _W[m + 4] * u[:, zlo + m:zhi + 1 + m, g:-g, g:-g]
    c = u[:, zlo:zhi + 1]
    h += 0.1 * (c[:, :, g:-g, g + 1:c.shape[3] - g + 1] + c[:, :, g:-g, g - 1:c.shape[3] - g - 1] +
                c[:, :, g + 1:c.shape[2] - g + 1, g:-g] + c[:, :, g - 1:c.shape[2] - g - 1, g:-g])
    return h


def _standin_dt(u):
    g = NG
    return 0.05 / (1.0 + np.abs(u[:, g:-g, g:-g, g:-g]).max())


class CpuOverlapSlab(CpuSlab):
    """CpuSlab with the overlapped-form phases of SlabStepper (numpy stand-ins)."""

    def __init__(self, lev, nranks, rank, box):
        super().__init__(lev, nranks, rank, box)
        self.nranks = nranks
        self.cfl = 0.3
        self.dt_next = torch.zeros(1, dtype=torch.float64)
        self._primed = False
        nz = self.sl.k1 - self.sl.k0 + 1
        self.h = np.zeros((self.state.shape[0], nz, self.state.shape[2] - 2 * NG, self.state.shape[3] - 2 * NG))
        from particleclem_b200.slab import SlabStepper

        self.int_z, self.bands = SlabStepper.regions(self.sl.k0, self.sl.k1, self.down is not None,
                                                     self.up is not None)
        self.overlap = self.int_z is not None and bool(self.bands)
        slab = self

        class _Plan:
            def estdt(self, cfl, out):
                out.fill_(_standin_dt(slab.state.numpy()))

        self.plan = _Plan()

    def fill_and_pack(self):
        super().fill_and_pack(self.nranks)

    def _unpack(self):
        self.unpack()

    def begin_step(self):
        self.dt.copy_(self.dt_next)

    def _source(self, z0, z1):  # global z range
        k0 = self.sl.k0
        self.h[:, z0 - k0:z1 - k0 + 1] = _standin_source(self.state.numpy(), z0 - k0 + NG, z1 - k0 + NG)

    def hydro_interior(self):
        self._source(*self.int_z)

    def unpack_and_hydro_bands(self):
        self.unpack()
        for b in self.bands:
            self._source(*b)

    def update_and_estdt(self):
        u = self.state.numpy()
        u[:, NG:-NG, NG:-NG, NG:-NG] += float(self.dt) * self.h
        self.dt_next.fill_(_standin_dt(u))


def _global_overlap_reference(lev, nsteps):
    u = lev.state.copy()
    for _ in range(nsteps):
        wl.fill_ghosts(u, lev.periodic)
        dt = _standin_dt(u)
        nz = u.shape[1] - 2 * NG
        u[:, NG:-NG, NG:-NG, NG:-NG] += dt * _standin_source(u, NG, NG + nz - 1)
    return u


def _overlap_level(periodic_z, seed=7):
    rng = np.random.default_rng(seed)
    n, nz = 6, 32
    st = rng.standard_normal((2, nz + 2 * NG, n + 2 * NG, n + 2 * NG))
    return wl.Level(wl.GammaLaw(), (1.0, 1.0, 1.0), (0, 0, 0), (n - 1, n - 1, nz - 1), (0, 0, 0), (0, 0, 0), st,
                    wl.tile_boxes((n, n, nz), (n, n, 8)), (True, True, periodic_z))


def _overlap_worker(rank, nranks, port, periodic_z, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        from particleclem_b200.slab import step_overlap

        lev = _overlap_level(periodic_z)
        s = CpuOverlapSlab(lev, nranks, rank, 8)
        for _ in range(3):
            step_overlap([s], DistComm())
        ref = _global_overlap_reference(lev, 3)
        k0 = s.sl.k0
        exp = ref[:, NG + k0:NG + s.sl.k1 + 1, NG:-NG, NG:-NG]
        got = s.state.numpy()[:, NG:-NG, NG:-NG, NG:-NG]
        out[rank] = bool(np.allclose(got, exp, rtol=0, atol=1e-13)), s.int_z, s.bands
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("periodic_z", [False, True])
def test_gloo_two_ranks_overlapped_steps_equal_whole_level(periodic_z):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_overlap_worker, args=(2, _free_port(), periodic_z, out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    for r in (0, 1):
        ok, int_z, bands = res[r]
        assert ok, (r, int_z, bands)
    # rank 0 of an outflow level has no neighbour below: one band (above) only
    assert len(res[0][2]) == (2 if periodic_z else 1)


def test_local_overlapped_steps_equal_whole_level():
    from particleclem_b200.slab import step_overlap

    lev = _overlap_level(False)
    slabs = [CpuOverlapSlab(lev, 2, r, 8) for r in range(2)]
    assert all(s.overlap for s in slabs)
    for _ in range(3):
        step_overlap(slabs, LocalComm())
    ref = _global_overlap_reference(lev, 3)
    got = np.concatenate([s.state.numpy()[:, NG:-NG, NG:-NG, NG:-NG] for s in slabs], axis=1)
    np.testing.assert_allclose(got, ref[:, NG:-NG, NG:-NG, NG:-NG], rtol=0, atol=1e-13)
