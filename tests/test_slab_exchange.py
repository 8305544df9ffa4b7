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
