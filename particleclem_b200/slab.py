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

Overlapped form (``overlap=True``): the hydro advance of the slab's interior planes, whose
4-cell stencil stays clear of the ghost planes the exchange fills, runs while the halo is
in flight; only the NG-plane bands next to an exchanging slab face wait for it. A step is

  1. local ghost fill and packing of the send planes (a device kernel)
  2. the exchange posted (NCCL works on NCCL's stream, ordered after the packing)
  3. hydro source of the interior region                 (runs during the exchange)
  4. wait for the exchange; unpack (a device kernel); hydro source of the bands
  5. S_new with computeTemp over the whole slab, then its CFL minimum
  6. the minimum over ranks, which is the next step's timestep.

Every region's hydro source is independent of how the level is cut (each output depends
only on traced states of grow(region, 1), inside the grow(region, 4) stencil), so the
overlapped step equals the plain one (bit for bit in the FP64 forms).
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

    def __init__(self, slab, nranks, rank, precision=abi.PREC_MIXED, fuse=True, cfl=0.3, device=0, fused_tail=True,
                 overlap=False):
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
        # overlapped form: the interior region and the bands next to exchanging faces
        self.plan_int = self.plan_bnd = None
        int_z, bands = self.regions(slab.k0, slab.k1, self.down is not None, self.up is not None)
        self.overlap = bool(overlap) and int_z is not None and bool(bands)
        if self.overlap:
            lo0, hi0 = (slab.domlo[0], slab.domlo[1]), (slab.domhi[0], slab.domhi[1])

            def box(z):
                return hydro.make_box((*lo0, z[0]), (*hi0, z[1]), self.state, self.hsrc, slab.dx, 0.0, slab.domlo,
                                      slab.domhi, slab.bclo, slab.bchi)

            self.plan_int = hydro.Plan(self.prm, [box(int_z)], fuse=True)
            self.plan_bnd = hydro.Plan(self.prm, [box(b) for b in bands], fuse=False)

    @staticmethod
    def regions(k0, k1, has_down, has_up):
        """z-ranges of the overlapped form: the interior (None if empty) and the bands of NG
        planes next to the slab faces that receive ghost planes from a neighbour."""
        lo = k0 + (NG if has_down else 0)
        hi = k1 - (NG if has_up else 0)
        bands = ([(k0, k0 + NG - 1)] if has_down else []) + ([(k1 - NG + 1, k1)] if has_up else [])
        return ((lo, hi) if lo <= hi else None), bands

    # -- phases
    def fill(self):
        """Local part of the ghost fill (no exchange)."""
        hydro.fill_ghosts(self.state, self.fill_lo, self.fill_hi, self.fill_periodic, NG)

    def _planes(self, z0, z1):
        """The box of all x, y cells (ghosts included) of the planes z0..z1."""
        sl = self.slab
        return (sl.domlo[0] - NG, sl.domlo[1] - NG, z0), (sl.domhi[0] + NG, sl.domhi[1] + NG, z1)

    def fill_and_pack(self):
        """Local ghost fill, then the NG lowest / highest valid planes into the send
        buffers (one copy kernel each)."""
        self.fill()
        k0, k1 = self.slab.k0, self.slab.k1
        if self.down is not None:
            lo, hi = self._planes(k0, k0 + NG - 1)
            hydro.copy_cells(self.state, abi.Fab(self.sbuf["down"], lo), lo, hi)
        if self.up is not None:
            lo, hi = self._planes(k1 - NG + 1, k1)
            hydro.copy_cells(self.state, abi.Fab(self.sbuf["up"], lo), lo, hi)

    def _unpack(self):
        """The received planes into the ghost planes below / above the slab."""
        k0, k1 = self.slab.k0, self.slab.k1
        if self.down is not None:
            lo, hi = self._planes(k0 - NG, k0 - 1)
            hydro.copy_cells(abi.Fab(self.rbuf["down"], lo), self.state, lo, hi)
        if self.up is not None:
            lo, hi = self._planes(k1 + 1, k1 + NG)
            hydro.copy_cells(abi.Fab(self.rbuf["up"], lo), self.state, lo, hi)

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

    # -- overlapped form
    def begin_step(self):
        """The step's timestep: the previous step's minimum over ranks of the new state."""
        self.dt.copy_(self.dt_next)

    def hydro_interior(self):
        self.plan_int.hydro(self.dt)

    def unpack_and_hydro_bands(self):
        self._unpack()
        self.plan_bnd.hydro(self.dt)

    def update_and_estdt(self):
        """S_new with computeTemp over the slab, then its CFL minimum into dt_next."""
        self.plan.update(self.dt)
        self.plan.estdt(self.cfl, self.dt_next)

    def close(self):
        self.graphs = None
        self.plan.close()
        for p in (self.plan_int, self.plan_bnd):
            if p is not None:
                p.close()


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

    def exchange_start(self, slabs):
        """Post the exchange and return its works; with NCCL the transfer runs on NCCL's
        stream after the work already queued (the packing), so later kernels overlap it."""
        import torch.distributed as dist

        (s,) = slabs
        ops = []
        if s.down is not None:
            ops.append(dist.P2POp(dist.isend, s.sbuf["down"], s.down))
        if s.up is not None:
            ops.append(dist.P2POp(dist.isend, s.sbuf["up"], s.up))
        if s.up is not None:
            ops.append(dist.P2POp(dist.irecv, s.rbuf["up"], s.up))
        if s.down is not None:
            ops.append(dist.P2POp(dist.irecv, s.rbuf["down"], s.down))
        return dist.batch_isend_irecv(ops) if ops else []

    def exchange_wait(self, works, slabs):
        """Order later work after the exchange (NCCL: the current stream waits; gloo: the
        host waits)."""
        for r in works:
            r.wait()

    def min_dt(self, slabs, attr="dt"):
        import torch.distributed as dist

        (s,) = slabs
        dist.all_reduce(getattr(s, attr), op=dist.ReduceOp.MIN)


class LocalComm:
    """The same exchange and reduction between slabs held by one process."""

    def exchange(self, slabs):
        for s in slabs:
            if s.up is not None:
                u = slabs[s.up]
                u.rbuf["down"].copy_(s.sbuf["up"])
                s.rbuf["up"].copy_(u.sbuf["down"])

    def exchange_start(self, slabs):
        self.exchange(slabs)
        return []

    def exchange_wait(self, works, slabs):
        pass

    def min_dt(self, slabs, attr="dt"):
        import torch

        m = torch.stack([getattr(s, attr) for s in slabs]).min(dim=0).values
        for s in slabs:
            getattr(s, attr).copy_(m)


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


def step_overlap(slabs, comm):
    """One level step in the overlapped form (see the module docstring). The first step,
    and a step after load_state, first take the fresh CFL timestep of the exchanged slabs.
    Slabs too thin for an interior region (at most 2 NG planes between two exchanging
    faces) take the plain step."""
    if not all(s.overlap for s in slabs):
        return step(slabs, comm)
    for s in slabs:
        s.fill_and_pack()
    if not all(s._primed for s in slabs):
        comm.exchange(slabs)
        for s in slabs:
            s._unpack()
            s.plan.estdt(s.cfl, s.dt_next)
        comm.min_dt(slabs, "dt_next")
    for s in slabs:
        s.begin_step()
    works = comm.exchange_start(slabs)
    for s in slabs:
        s.hydro_interior()  # overlaps the halo exchange
    comm.exchange_wait(works, slabs)
    for s in slabs:
        s.unpack_and_hydro_bands()
    for s in slabs:
        s.update_and_estdt()
    comm.min_dt(slabs, "dt_next")
    for s in slabs:
        s._primed = True
