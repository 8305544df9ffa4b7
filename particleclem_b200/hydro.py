"""Python mirror of the reference operator surface for the Godunov hydro path.

Functions take FABs (:class:`particleclem_b200.abi.Fab`) whose ``data`` are CUDA
float64 tensors of shape (ncomp, nz, ny, nx) and call the native library through
the C ABI (include/pcg_hydro.h). Names and argument meaning follow the reference:

* :func:`ctoprim`       -- pc_ctoprim launch   (Source/Hydro.cpp:104-116)
* :func:`srctoprim`     -- pc_srctoprim launch (Source/Hydro.cpp:161-174, Source/Hydro.H:14-68)
* :func:`umdrv`         -- pc_umdrv            (Source/Hydro.H:910-935)
* :func:`umeth`         -- pc_umeth_3D alone   (Source/Godunov.H:1142-1162)
* :func:`hydro_box`     -- one construct_hydro_source box iteration (Source/Hydro.cpp:70-249)
* :func:`hydro_boxes`   -- the whole box loop in one set of launches
* :func:`estdt`         -- estTimeStep's hydro reduction (Source/PeleC.cpp:829-960)
* :func:`update_state`  -- construct_Snew + computeTemp
* :func:`fill_ghosts`   -- single-level FillBoundary
* :class:`Plan`         -- persistent, graph-capturable form of the above

Errors raise :class:`particleclem_b200.native.PcgError` carrying the PCG_E* code.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, native
from .thermo import GammaLaw

_current_eos = {}


def _stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def init(device: int = 0):
    native.call("pcg_init", int(device))


def species_counts():
    """The species counts the loaded library has kernels for (ascending)."""
    lib = native.load()
    n = lib.pcg_species_counts(None, 0)
    buf = (C.c_int32 * max(n, 1))()
    lib.pcg_species_counts(buf, n)
    return tuple(int(buf[k]) for k in range(n))


def set_eos(eos):
    """Upload an EOS table (GammaLaw or Nasa7Mixture) to the library."""
    if isinstance(eos, GammaLaw):
        native.call("pcg_set_eos_gamma", float(eos.gamma), float(eos.mw))
    else:
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (eos.mw, eos.tmid, eos.a_lo, eos.a_hi)]
        ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        native.call("pcg_set_eos_nasa7", int(eos.nspec), *ptrs)
    _current_eos[eos.nspec] = eos


def _a4p(fab):
    return C.byref(abi.array4(fab)) if fab is not None else None


def ctoprim(prm, lo, hi, u, q, qaux, stream=None):
    native.call("pcg_ctoprim", C.byref(prm), abi.ivec(lo), abi.ivec(hi), _a4p(u), _a4p(q), _a4p(qaux),
                _stream_ptr(stream))


def umdrv(prm, lo, hi, uin, uout, q, qaux, src_q, flx, area, vol, stream=None):
    """pc_umdrv: uout += hydro source of box [lo,hi]; flx[3] overwritten."""
    native.call("pcg_umdrv", C.byref(prm), abi.ivec(lo), abi.ivec(hi), _a4p(uin), _a4p(uout), _a4p(q), _a4p(qaux),
                _a4p(src_q), abi.array4_list(flx), abi.array4_list(area), _a4p(vol), _stream_ptr(stream))


def srctoprim(prm, lo, hi, q, qaux, src, srcq, stream=None):
    """pc_srctoprim over [lo,hi]: srcq (QVAR comps) from the conserved sources src."""
    native.call("pcg_srctoprim", C.byref(prm), abi.ivec(lo), abi.ivec(hi), _a4p(q), _a4p(qaux), _a4p(src),
                _a4p(srcq), _stream_ptr(stream))


def umeth(prm, lo, hi, q, qaux, src_q, flx, qec, area, pdivu, vol, stream=None):
    """pc_umeth_3D: the unadjusted final fluxes flx[3], the face states qec[3] (NGDNV
    components, GDRHO not written) and pdivu of box [lo,hi]."""
    native.call("pcg_umeth", C.byref(prm), abi.ivec(lo), abi.ivec(hi), _a4p(q), _a4p(qaux), _a4p(src_q),
                abi.array4_list(flx), abi.array4_list(qec), abi.array4_list(area), _a4p(pdivu), _a4p(vol),
                _stream_ptr(stream))


def hydro_box(prm, lo, hi, uin, uout, flx=None, stream=None):
    native.call("pcg_hydro_box", C.byref(prm), abi.ivec(lo), abi.ivec(hi), _a4p(uin), _a4p(uout),
                abi.array4_list(flx) if flx is not None else None, _stream_ptr(stream))


def make_box(lo, hi, uin, uout, dx, dt, domlo=None, domhi=None, bclo=(0, 0, 0), bchi=(0, 0, 0), flx=None):
    b = native.Box()
    big = 1 << 30
    b.lo[:] = list(lo)
    b.hi[:] = list(hi)
    b.domlo[:] = list(domlo) if domlo is not None else [-big] * 3
    b.domhi[:] = list(domhi) if domhi is not None else [big] * 3
    b.bclo[:] = list(bclo)
    b.bchi[:] = list(bchi)
    b.dx[:] = [float(v) for v in dx]
    b.dt = float(dt)
    b.uin = abi.array4(uin)
    if uout is not None:  # pcg_step_boxes stores no hydro source
        b.uout = abi.array4(uout)
    if flx is not None:
        for d in range(3):
            b.flx[d] = abi.array4(flx[d])
    b._keep = (uin, uout, flx)  # the descriptor holds raw pointers: keep the FABs alive with it
    return b


def box_array(boxes):
    arr = (native.Box * len(boxes))()
    for i, b in enumerate(boxes):
        arr[i] = b
    return arr


def hydro_boxes(prm, boxes, stream=None):
    arr = box_array(boxes)
    native.call("pcg_hydro_boxes", C.byref(prm), len(boxes), arr, _stream_ptr(stream))


def step_boxes(prm, boxes, cfl, dt, dt_next, fill_ghosts=True, stream=None):
    """One full step of independent patches (ghost fill, hydro, S_new with computeTemp in
    place, next CFL timestep per box). dt / dt_next: CUDA float64 tensors of len(boxes)
    (dt None: each box's own dt)."""
    arr = box_array(boxes)
    native.call("pcg_step_boxes", C.byref(prm), len(boxes), arr, int(bool(fill_ghosts)), float(cfl),
                C.c_void_p(dt.data_ptr()) if dt is not None else None, C.c_void_p(dt_next.data_ptr()),
                _stream_ptr(stream))


def trim_workspace(device, keep_bytes=0):
    """Return all but ``keep_bytes`` of the library's workspace pool of ``device`` to the driver."""
    native.call("pcg_trim_workspace", int(device), int(keep_bytes))


def reserve_workspace(device, nbytes):
    """Grow the library's workspace pool of ``device`` to hold at least ``nbytes``."""
    native.call("pcg_reserve_workspace", int(device), int(nbytes))


def workspace_bytes(prm, extents):
    """Device bytes hydro_boxes allocates for boxes given as (lo, hi) pairs (host only)."""
    n = len(extents)
    lo = (C.c_int32 * (3 * n))(*[int(v) for l, _ in extents for v in l])
    hi = (C.c_int32 * (3 * n))(*[int(v) for _, h in extents for v in h])
    out = C.c_int64()
    native.call("pcg_hydro_workspace", C.byref(prm), n, lo, hi, C.byref(out))
    return out.value


def estdt(nspec, boxes, cfl, dt_out, stream=None):
    """dt_out: a CUDA float64 tensor of one element."""
    arr = box_array(boxes)
    native.call("pcg_estdt", int(nspec), len(boxes), arr, float(cfl), C.c_void_p(dt_out.data_ptr()),
                _stream_ptr(stream))


def update_state(nspec, boxes, s_new, dt_dev=None, stream=None):
    arr = box_array(boxes)
    native.call("pcg_update_state", int(nspec), len(boxes), arr, abi.array4_list(s_new),
                C.c_void_p(dt_dev.data_ptr()) if dt_dev is not None else None, _stream_ptr(stream))


def fill_ghosts(state, domlo, domhi, periodic, ng=abi.NGROW, stream=None):
    native.call("pcg_fill_ghosts", _a4p(state), abi.ivec(domlo), abi.ivec(domhi),
                abi.ivec([int(bool(p)) for p in periodic]), int(ng), _stream_ptr(stream))


def copy_cells(src, dst, lo, hi, stream=None):
    """Copy the cells [lo, hi] of every component of FAB ``src`` into FAB ``dst`` (host
    or device tensors; pinned host memory for an asynchronous copy), on ``stream``."""
    native.call("pcg_copy_cells", _a4p(src), _a4p(dst), abi.ivec(lo), abi.ivec(hi), _stream_ptr(stream))


class Plan:
    """Persistent launch plan over a fixed box list (graph-capturable runs)."""

    def __init__(self, prm, boxes, fuse=False):
        self._boxes = box_array(boxes)  # keep the descriptors alive with the plan
        self.prm = prm
        h = C.c_void_p()
        native.call("pcg_plan_create", C.byref(prm), len(boxes), self._boxes, int(bool(fuse)), C.byref(h))
        self.h = h

    def hydro(self, dt_dev=None, stream=None):
        native.call("pcg_plan_hydro", self.h, C.c_void_p(dt_dev.data_ptr()) if dt_dev is not None else None,
                    _stream_ptr(stream))

    STAGES = ("ctoprim", "prep", "trace", "flux0", "flux1", "flux2", "consup")

    def stages(self, first, last, dt_dev=None, stream=None):
        native.call("pcg_plan_stages", self.h, int(first), int(last),
                    C.c_void_p(dt_dev.data_ptr()) if dt_dev is not None else None, _stream_ptr(stream))

    def estdt(self, cfl, dt_dev, stream=None):
        native.call("pcg_plan_estdt", self.h, float(cfl), C.c_void_p(dt_dev.data_ptr()), _stream_ptr(stream))

    def advance(self, cfl, dt_dev, dt_next, stream=None):
        """Hydro stages and the fused update with this step's dt_dev; dt_next receives
        the next step's CFL timestep (both one-element CUDA float64 tensors)."""
        native.call("pcg_plan_advance", self.h, float(cfl), C.c_void_p(dt_dev.data_ptr()),
                    C.c_void_p(dt_next.data_ptr()), _stream_ptr(stream))

    def update(self, dt_dev=None, stream=None):
        native.call("pcg_plan_update", self.h, C.c_void_p(dt_dev.data_ptr()) if dt_dev is not None else None,
                    _stream_ptr(stream))

    def info(self):
        ws = C.c_int64()
        nr = C.c_int32()
        blk = (C.c_int64 * 7)()
        native.call("pcg_plan_info", self.h, C.byref(ws), C.byref(nr), blk)
        return {"workspace_bytes": ws.value, "nregions": nr.value, "blocks": list(blk)}

    def close(self):
        if self.h:
            native.call("pcg_plan_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
