"""Batched advance of independent boxes of any sizes.

The box loop of PeleC::construct_hydro_source (Source/Hydro.cpp:70-288) runs the Godunov
advance box by box with temporaries allocated per box; here a list of uneven boxes, each
with its own grown state FAB resident on the device, is one plan: every stage is one
launch over all boxes (segments of the launch map to boxes), the CFL timestep is the
minimum over all boxes (estTimeStep, Source/PeleC.cpp:829-960) and the update
S_new = S_old + dt * hydro_source plus computeTemp (Source/Advance.cpp:397-417) follows,
so a step is a fixed number of launches whatever the number of boxes, and it can be
captured in a CUDA graph. With the fused step tail (the default) the update pass also
forms the CFL minimum of the new states for the next step, as in level.LevelStepper. The boxes share no ghost cells (independent patches, as the boxes of different
ensemble members or of different AMR levels).
"""
from __future__ import annotations

import numpy as np

from . import abi, hydro
from .level import _nullctx


class BoxBatch:
    def __init__(self, patches, eos, precision=abi.PREC_MIXED, cfl=0.3, ppm_type=1, plm_iorder=4,
                 use_flattening=True, difmag=0.1, device=0, fused_tail=True):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.ns = eos.nspec
        self.nv = abi.nvar(self.ns)
        self.cfl = float(cfl)
        hydro.init(device)
        hydro.set_eos(eos)
        self.patches = patches
        self.states, self.hsrc, boxes = [], [], []
        for p in patches:
            u = abi.Fab(torch.from_numpy(np.ascontiguousarray(p.fab.data)).to(self.dev), tuple(p.fab.lo))
            n = [p.hi[d] - p.lo[d] + 1 for d in range(3)]
            h = abi.Fab(torch.zeros((self.nv, n[2], n[1], n[0]), dtype=torch.float64, device=self.dev), tuple(p.lo))
            self.states.append(u)
            self.hsrc.append(h)
            boxes.append(hydro.make_box(p.lo, p.hi, u, h, p.dx, 0.0))
        self.prm = abi.make_params(patches[0].dx, 0.0, self.ns, (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0),
                                   ppm_type=ppm_type, plm_iorder=plm_iorder, use_flattening=use_flattening,
                                   difmag=difmag, precision_mode=precision)
        self.plan = hydro.Plan(self.prm, boxes, fuse=False)
        self.dt = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.fused_tail = bool(fused_tail)
        self.dt_next = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self._primed = False
        self.ncells = int(sum(p.ncells for p in patches))
        self.graph = None

    @property
    def launches_per_step(self):
        # hydro stages (6 with the fused tail, whose consup is the tail), then the fused
        # tail and the final minimum, or estdt (2) + 7 stages + update
        return 6 + 2 if self.fused_tail else 2 + 7 + 1

    def step(self, stream=None):
        """One step of every box with the batch's CFL timestep (self.dt afterwards)."""
        if not self.fused_tail:
            self.plan.estdt(self.cfl, self.dt, stream)
            self.plan.hydro(self.dt, stream)
            self.plan.update(self.dt, stream)
            return
        if not self._primed:
            self.plan.estdt(self.cfl, self.dt_next, stream)
            self._primed = True
        with self.torch.cuda.stream(stream) if stream is not None else _nullctx():
            self.dt.copy_(self.dt_next)
        self.plan.advance(self.cfl, self.dt, self.dt_next, stream)

    def capture(self):
        torch = self.torch
        s = torch.cuda.Stream(device=self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self.step()  # library warm-up outside the capture
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.step()
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()

    def box_edges(self):
        return [[p.hi[d] - p.lo[d] + 1 for d in range(3)] for p in self.patches]

    def close(self):
        self.graph = None
        self.plan.close()
