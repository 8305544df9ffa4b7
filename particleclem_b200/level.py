"""Device-resident single-level advance: the level loop around the hydro path.

One step is what PeleC's level advance does around construct_hydro_source for a
Godunov run without sources (Source/Advance.cpp:266-352): fill the ghost cells of the
state (FillPatch/FillBoundary, :307-309), take the CFL timestep of the level
(estTimeStep, Source/PeleC.cpp:829-960), build the hydro source of every box
(Source/Hydro.cpp:4-301), then S_new = S_old + dt * hydro_source and computeTemp
(Source/Advance.cpp:397-417, Source/PeleC.cpp:2289-2305). The state never leaves the
device, dt stays in device memory, and a step can be captured in a CUDA graph.
"""
from __future__ import annotations

import numpy as np

from . import abi, hydro

NG = abi.NGROW


class _nullctx:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class LevelStepper:
    def __init__(self, level, precision=abi.PREC_MIXED, fuse=True, cfl=0.3, ppm_type=1, plm_iorder=4,
                 use_flattening=True, difmag=0.1, device=0, fused_tail=True, use_hybrid_weno=False, weno_scheme=1):
        import torch

        self.torch = torch
        self.level = level
        self.cfl = float(cfl)
        self.ns = level.nspec
        self.nv = abi.nvar(self.ns)
        self.dev = torch.device("cuda", device)
        hydro.init(device)
        hydro.set_eos(level.eos)
        self.state = abi.Fab(torch.from_numpy(np.ascontiguousarray(level.state)).to(self.dev), level.fab.lo)
        n = [level.domhi[d] - level.domlo[d] + 1 for d in range(3)]
        self.hsrc = abi.Fab(torch.zeros((self.nv, n[2], n[1], n[0]), dtype=torch.float64, device=self.dev),
                            tuple(level.domlo))
        self.dt = torch.zeros(1, dtype=torch.float64, device=self.dev)
        # with the fused tail the step also produces the next step's timestep
        self.fused_tail = bool(fused_tail)
        self.dt_next = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self._primed = False
        self.prm = abi.make_params(level.dx, 0.0, self.ns, level.domlo, level.domhi, level.bclo, level.bchi,
                                   ppm_type=ppm_type, plm_iorder=plm_iorder, use_flattening=use_flattening,
                                   difmag=difmag, precision_mode=precision, use_hybrid_weno=use_hybrid_weno,
                                   weno_scheme=weno_scheme)
        self.boxes = [hydro.make_box(lo, hi, self.state, self.hsrc, level.dx, 0.0, level.domlo, level.domhi,
                                     level.bclo, level.bchi) for lo, hi in level.boxes]
        self.plan = hydro.Plan(self.prm, self.boxes, fuse=fuse)
        self.graph = None
        self.ncells = level.ncells()

    # one level step, enqueued on the current stream
    def fill(self, stream=None):
        L = self.level
        hydro.fill_ghosts(self.state, L.domlo, L.domhi, L.periodic, NG, stream)

    def load_state(self, src, non_blocking=False):
        """Replace the level state (ghost cells included) with ``src``. The next step then
        takes its timestep from a fresh CFL reduction of the new state."""
        self.state.data.copy_(src, non_blocking=non_blocking)
        self._primed = False

    def _valid_rows(self):
        # the valid (j, k) rows, whole: x ghost cells included, so that the rows of one
        # k-slice are one contiguous run (copies of short strided rows, host to device
        # above all, run far below the bus bandwidth)
        lo, hi = self.level.domlo, self.level.domhi
        return (lo[0] - NG, lo[1], lo[2]), (hi[0] + NG, hi[1], hi[2])

    def upload(self, host, stream=None):
        """Copy the valid rows of ``host`` (a pinned tensor of the state's shape) into the
        state; the step's ghost fill forms the ghost cells. The next step takes a fresh
        CFL timestep."""
        hydro.copy_cells(abi.Fab(host, self.state.lo), self.state, *self._valid_rows(), stream)
        self._primed = False

    def download(self, host, stream=None):
        """Copy the valid rows of the state into ``host`` (pinned, the state's shape): the
        valid cells, with the x ghost cells of those rows as the step's ghost fill left
        them; the other ghost cells of ``host`` are not written."""
        hydro.copy_cells(self.state, abi.Fab(host, self.state.lo), *self._valid_rows(), stream)

    @property
    def row_bytes(self):
        """Bytes :meth:`upload` and :meth:`download` move."""
        n = [self.level.domhi[d] - self.level.domlo[d] + 1 for d in range(3)]
        return self.nv * (n[0] + 2 * NG) * n[1] * n[2] * 8

    def step(self, stream=None, fresh_dt=False):
        """One level step; self.dt holds the step's timestep afterwards. With the fused
        tail the CFL minimum of the new state is formed by the update pass itself; the
        timestep comes from a separate reduction on the first step, after
        :meth:`load_state`, and on every step when ``fresh_dt`` is set (a step whose
        state is written from outside between steps, as in a captured graph that is
        replayed on new inputs)."""
        self.fill(stream)
        if not self.fused_tail:
            self.plan.estdt(self.cfl, self.dt, stream)
            self.plan.hydro(self.dt, stream)
            self.plan.update(self.dt, stream)
            return
        if fresh_dt or not self._primed:
            self.plan.estdt(self.cfl, self.dt_next, stream)
            self._primed = True
        torch = self.torch
        with torch.cuda.stream(stream) if stream is not None else _nullctx():
            self.dt.copy_(self.dt_next)
        self.plan.advance(self.cfl, self.dt, self.dt_next, stream)

    # ghost fill (one pass), hydro stages (6), fused consup/update/CFL minimum, final minimum
    launches_per_step = 1 + 6 + 1 + 1

    def capture(self, fresh_dt=False):
        """Capture one step as a CUDA graph (after one eager step that warms the library:
        EOS upload, lazy module loading). ``fresh_dt`` as in :meth:`step`."""
        torch = self.torch
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.step(fresh_dt=fresh_dt)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.step(fresh_dt=fresh_dt)
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()

    def host_state(self):
        self.torch.cuda.synchronize(self.dev)
        return self.state.data.cpu().numpy()

    def close(self):
        self.graph = None
        self.plan.close()


class HostPipeline:
    """Advance host-resident level states through the device, one level step each.

    Every submitted state goes host -> device (pinned memory), takes one graph-captured
    level step and comes back device -> host. ``depth`` device slots (a LevelStepper each)
    rotate so that uploads, steps and downloads of successive submissions run at the same
    time: uploads and downloads use separate copy streams (the two DMA directions are
    independent) and the steps share one compute stream. A slot is reused only after its
    previous result has left the device, so with the copies each longer than a step the
    pipeline needs three slots to keep both DMA directions busy. With ``valid_only`` (the
    default) only the valid rows cross the bus, each way (:meth:`LevelStepper.upload`,
    :meth:`LevelStepper.download`; the step's ghost fill forms the ghost cells);
    otherwise the whole state including ghost cells.
    """

    def __init__(self, level, depth=3, valid_only=True, **stepper_kw):
        import torch

        self.torch = torch
        self.valid_only = bool(valid_only)
        self.slots = [LevelStepper(level, **stepper_kw) for _ in range(depth)]
        for s in self.slots:
            s.capture(fresh_dt=True)  # every submission is a new state
        dev = self.slots[0].dev
        self.up, self.comp, self.down = (torch.cuda.Stream(device=dev) for _ in range(3))
        ev = lambda: [torch.cuda.Event() for _ in range(depth)]  # noqa: E731
        self.ev_in, self.ev_step, self.ev_out = ev(), ev(), ev()
        self.used = [False] * depth
        self.k = 0
        self.ncells = self.slots[0].ncells
        self.state_bytes = self.slots[0].state.data.numel() * 8
        # bytes that cross the bus per submission, host to device and device to host
        self.h2d_bytes = self.d2h_bytes = self.slots[0].row_bytes if self.valid_only else self.state_bytes

    def submit(self, host_in, host_out):
        """Enqueue one advance of ``host_in`` (pinned, the level's state shape) into
        ``host_out`` (pinned; must not be read before :meth:`synchronize`)."""
        torch = self.torch
        b = self.k % len(self.slots)
        slot = self.slots[b]
        if self.used[b]:
            self.up.wait_event(self.ev_out[b])  # the slot's previous result has left the device
        with torch.cuda.stream(self.up):
            if self.valid_only:
                slot.upload(host_in, self.up)
            else:
                slot.state.data.copy_(host_in, non_blocking=True)
            self.ev_in[b].record(self.up)
        self.comp.wait_event(self.ev_in[b])
        with torch.cuda.stream(self.comp):
            slot.replay()
            self.ev_step[b].record(self.comp)
        self.down.wait_event(self.ev_step[b])
        with torch.cuda.stream(self.down):
            if self.valid_only:
                slot.download(host_out, self.down)
            else:
                host_out.copy_(slot.state.data, non_blocking=True)
            self.ev_out[b].record(self.down)
        self.used[b] = True
        self.k += 1

    def synchronize(self):
        for s in (self.up, self.comp, self.down):
            s.synchronize()

    def close(self):
        self.synchronize()
        for s in self.slots:
            s.close()
