"""One level decomposed into z-slabs, one per rank.

PeleC distributes a level's boxes over MPI ranks and, once per step, fills the ghost
cells of every box from its neighbours (FillPatch / FillBoundary, Source/Advance.cpp:
307-309) and reduces the CFL timestep over all ranks (ParallelDescriptor::ReduceRealMin
in estTimeStep, Source/PeleC.cpp:929). Here each rank owns the slab [k0, k1] of the
level (all of x and y, whole boxes in z) as one device FAB, and a step is

  1. local ghost fill of the slab: periodic x/y, zero-gradient z        (one kernel)
  2. halo exchange in z: the NG lowest and highest valid planes go to the neighbour
     below and above and land in its ghost planes (interior slab faces only)
  3. CFL timestep of the slab, then the minimum over all ranks
  4. hydro advance of the slab's boxes (one fused region) and the update.

With the fused step tail (the default) step 4 is pcg_plan_advance, whose update pass
also forms the slab's CFL minimum of the new state, and step 3 reduces that minimum
over the ranks: no separate timestep pass, except on the first step and after the state
was replaced (load_state), where step 3 runs the CFL reduction of the slab first.

Steps 1+pack, unpack+3a and 4 are CUDA graphs; the exchange and the reduction are NCCL
point-to-point and all-reduce calls through torch.distributed (DistComm), or direct
device copies between slabs held by one process (LocalComm, used to check the
decomposition on one device). The global domain's physical boundaries (outflow in z for
the flame) stay with the first and last slab; a periodic z wraps around the ranks.
"""
from __future__ import annotations

import numpy as np

from . import abi, hydro

NG = abi.NGROW


def neighbours(nranks, rank, periodic_z):
    """(down, up) ranks of rank's slab, None at a physical boundary."""
    if nranks == 1:
        return None, None
    down = rank - 1 if rank > 0 else (nranks - 1 if periodic_z else None)
    up = rank + 1 if rank < nranks - 1 else (0 if periodic_z else None)
    return down, up


def halo_planes(state, ng=NG):
    """Views of a grown slab state (ncomp, nz+2ng, ny+2ng, nx+2ng): the planes it sends
    down/up and the ghost planes it receives from below/above."""
    nzl = state.shape[1] - 2 * ng
    return {"send_down": state[:, ng:2 * ng], "send_up": state[:, nzl:nzl + ng],
            "recv_down": state[:, 0:ng], "recv_up": state[:, nzl + ng:nzl + 2 * ng]}


class SlabStepper:
    """The device side of one rank's slab (see the module docstring)."""

    def __init__(self, slab, nranks, rank, precision=abi.PREC_MIXED, fuse=True, cfl=0.3, device=0, fused_tail=True):
        import torch

        self.torch = torch
        self.slab = slab
        self.dev = torch.device("cuda", device)
        self.ns = slab.nspec
        self.nv = abi.nvar(self.ns)
        self.cfl = float(cfl)
        hydro.init(device)
        hydro.set_eos(slab.eos)
        self.down, self.up = neighbours(nranks, rank, slab.periodic[2])
        self.state = abi.Fab(torch.from_numpy(np.ascontiguousarray(slab.state)).to(self.dev), slab.lo)
        nx = slab.domhi[0] - slab.domlo[0] + 1
        ny = slab.domhi[1] - slab.domlo[1] + 1
        nz = slab.k1 - slab.k0 + 1
        self.hsrc = abi.Fab(torch.zeros((self.nv, nz, ny, nx), dtype=torch.float64, device=self.dev),
                            (slab.domlo[0], slab.domlo[1], slab.k0))
        self.dt = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.fused_tail = bool(fused_tail)
        self.dt_next = torch.zeros(1, dtype=torch.float64, device=self.dev)  # slab CFL minimum of the new state
        self._primed = False
        self.prm = abi.make_params(slab.dx, 0.0, self.ns, slab.domlo, slab.domhi, slab.bclo, slab.bchi,
                                   precision_mode=precision)
        boxes = [hydro.make_box(lo, hi, self.state, self.hsrc, slab.dx, 0.0, slab.domlo, slab.domhi, slab.bclo,
                                slab.bchi) for lo, hi in slab.boxes]
        self.plan = hydro.Plan(self.prm, boxes, fuse=fuse)
        # the slab's own fill domain: its k-range, z periodic only when one rank holds a
        # periodic level (otherwise zero-gradient, overwritten by the exchange inside)
        self.fill_lo = (slab.domlo[0], slab.domlo[1], slab.k0)
        self.fill_hi = (slab.domhi[0], slab.domhi[1], slab.k1)
        self.fill_periodic = (slab.periodic[0], slab.periodic[1], slab.periodic[2] and nranks == 1)
        v = halo_planes(self.state.data)
        self.views = v
        self.sbuf = {k: torch.empty_like(v["send_" + k]) for k in ("down", "up")}
        self.rbuf = {k: torch.zeros_like(v["recv_" + k]) for k in ("down", "up")}
        self.ncells = slab.ncells()
        self.graphs = None

    # -- phases
    def fill(self):
        """Local part of the ghost fill (no exchange)."""
        hydro.fill_ghosts(self.state, self.fill_lo, self.fill_hi, self.fill_periodic, NG)

    def fill_and_pack(self):
        self.fill()
        if self.down is not None:
            self.sbuf["down"].copy_(self.views["send_down"])
        if self.up is not None:
            self.sbuf["up"].copy_(self.views["send_up"])

    def _unpack(self):
        if self.down is not None:
            self.views["recv_down"].copy_(self.rbuf["down"])
        if self.up is not None:
            self.views["recv_up"].copy_(self.rbuf["up"])

    def unpack_and_estdt(self):
        """Unpack the received ghost planes; the slab's CFL timestep into dt (its CFL
        reduction, or with the fused tail the minimum the previous advance formed)."""
        self._unpack()
        if self.fused_tail and self._primed:
            self.dt.copy_(self.dt_next)
        else:
            self.plan.estdt(self.cfl, self.dt)

    def advance(self):
        if self.fused_tail:
            self.plan.advance(self.cfl, self.dt, self.dt_next)
        else:
            self.plan.hydro(self.dt)
            self.plan.update(self.dt)

    def load_state(self, src, non_blocking=False):
        """Replace the slab's state; the next step takes a fresh CFL reduction."""
        self.state.data.copy_(src, non_blocking=non_blocking)
        self._primed = False

    def capture(self):
        """CUDA graphs of the local phases (the timestep phase twice: from the CFL
        reduction and, with the fused tail, from the previous advance's minimum). One
        eager pass warms the library first (its exchange-free unpack would leave stale
        ghost planes, so the state and dt are restored afterwards: capturing does not
        advance the slab)."""
        torch = self.torch
        saved, saved_dt, primed = self.state.data.clone(), self.dt.clone(), self._primed
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.fill_and_pack()
            self.unpack_and_estdt()
            self.advance()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        self.state.data.copy_(saved)
        self.dt.copy_(saved_dt)
        torch.cuda.synchronize(self.dev)
        del saved
        gs = {}
        for key, fn, prime in ((0, self.fill_and_pack, None), ("fresh", self.unpack_and_estdt, False),
                               ("primed", self.unpack_and_estdt, True), (2, self.advance, None)):
            if prime is not None:
                self._primed = prime
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                fn()
            gs[key] = g
        self._primed = primed
        self.graphs = gs

    def phase(self, i):
        if self.graphs:
            if i == 1:
                self.graphs["primed" if self.fused_tail and self._primed else "fresh"].replay()
            else:
                self.graphs[i].replay()
        else:
            (self.fill_and_pack, self.unpack_and_estdt, self.advance)[i]()
        if i == 2 and self.fused_tail:
            self._primed = True

    def close(self):
        self.graphs = None
        self.plan.close()


class DistComm:
    """Halo exchange and timestep minimum between ranks through torch.distributed
    (NCCL on GPUs, gloo on CPU tensors)."""

    def exchange(self, slabs):
        import torch.distributed as dist

        (s,) = slabs
        # every rank posts its sends (down, up) and receives (from up, from down) in the
        # same order, so that with two ranks on a periodic level (down == up) the two
        # messages between a pair still match one to one
        ops = []
        if s.down is not None:
            ops.append(dist.P2POp(dist.isend, s.sbuf["down"], s.down))
        if s.up is not None:
            ops.append(dist.P2POp(dist.isend, s.sbuf["up"], s.up))
        if s.up is not None:
            ops.append(dist.P2POp(dist.irecv, s.rbuf["up"], s.up))
        if s.down is not None:
            ops.append(dist.P2POp(dist.irecv, s.rbuf["down"], s.down))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def min_dt(self, slabs):
        import torch.distributed as dist

        (s,) = slabs
        dist.all_reduce(s.dt, op=dist.ReduceOp.MIN)


class LocalComm:
    """The same exchange and reduction between slabs held by one process."""

    def exchange(self, slabs):
        for s in slabs:
            if s.up is not None:
                u = slabs[s.up]
                u.rbuf["down"].copy_(s.sbuf["up"])
                s.rbuf["up"].copy_(u.sbuf["down"])

    def min_dt(self, slabs):
        import torch

        m = torch.stack([s.dt for s in slabs]).min(dim=0).values
        for s in slabs:
            s.dt.copy_(m)


def step(slabs, comm):
    """One level step over the given slabs (one per process with DistComm, all of them
    with LocalComm)."""
    for s in slabs:
        s.phase(0)
    comm.exchange(slabs)
    for s in slabs:
        s.phase(1)
    comm.min_dt(slabs)
    for s in slabs:
        s.phase(2)
