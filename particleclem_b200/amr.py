"""Coarse/fine levels: the flux register, reflux and average-down behind the C ABI.

The reference stores each box's area-weighted hydro fluxes in AMReX flux registers after
the hydro source (Source/Hydro.cpp:281-287 -> PeleC::update_flux_registers,
Source/PeleC.cpp:1343-1400: CrseAdd on the coarse level, FineAdd on every fine substep),
resets the register at the start of the coarse step (Source/Advance.cpp:30-31) and, after
the fine subcycles, corrects the coarse cells next to the fine region
(PeleC::reflux, Source/PeleC.cpp:1403-1414) before averaging the fine level down onto the
coarse cells it covers (PeleC::avgDown, Source/PeleC.cpp:1440, called at :1098). ``FluxRegister`` and ``average_down`` are those
steps on the device (include/pcg_hydro.h, pcg_fluxreg_* and pcg_average_down).
"""
from __future__ import annotations

import ctypes as C

from . import abi, native
from .hydro import _stream_ptr


def _ivecs(boxes):
    flat = [int(v) for b in boxes for v in b]
    return (C.c_int32 * max(len(flat), 1))(*flat)


class FluxRegister:
    """The register between a coarse level (domain crse_domlo..crse_domhi, periodic
    flags) and the fine boxes above it (fine index space, refinement ratio ``ratio``)."""

    def __init__(self, ncomp, crse_domlo, crse_domhi, periodic, ratio, fine_boxes):
        self.fine_boxes = [(tuple(lo), tuple(hi)) for lo, hi in fine_boxes]
        self.ncomp = int(ncomp)
        self.ratio = int(ratio)
        h = C.c_void_p()
        native.call("pcg_fluxreg_create", self.ncomp, abi.ivec(crse_domlo), abi.ivec(crse_domhi),
                    abi.ivec([int(bool(p)) for p in periodic]), self.ratio, len(self.fine_boxes),
                    _ivecs([lo for lo, _ in self.fine_boxes]), _ivecs([hi for _, hi in self.fine_boxes]), C.byref(h))
        self.h = h

    def info(self):
        nf, nc = C.c_int32(), C.c_int32()
        native.call("pcg_fluxreg_info", self.h, C.byref(nf), C.byref(nc))
        return {"faces": nf.value, "cells": nc.value}

    def reset(self, stream=None):
        native.call("pcg_fluxreg_reset", self.h, _stream_ptr(stream))

    def crse_add(self, lo, hi, flx, dt, stream=None):
        """flx: the coarse box's three area-weighted face FABs."""
        native.call("pcg_fluxreg_crse_add", self.h, abi.ivec(lo), abi.ivec(hi), abi.array4_list(flx), float(dt),
                    _stream_ptr(stream))

    def fine_add(self, lo, hi, flx, dt, stream=None):
        """flx: the fine box's three area-weighted face FABs of one fine substep of dt."""
        native.call("pcg_fluxreg_fine_add", self.h, abi.ivec(lo), abi.ivec(hi), abi.array4_list(flx), float(dt),
                    _stream_ptr(stream))

    def reflux(self, s_crse, vol, stream=None):
        """S += accumulated corrections / vol on the coarse cells next to the fine region."""
        native.call("pcg_fluxreg_reflux", self.h, C.byref(abi.array4(s_crse)), float(vol), _stream_ptr(stream))

    def close(self):
        if getattr(self, "h", None):
            native.call("pcg_fluxreg_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def average_down(fine, crse, fine_lo, fine_hi, ratio, ncomp, stream=None):
    """Coarse cells under the fine box [fine_lo, fine_hi] become the mean of their
    ratio^3 fine cells (components 0..ncomp-1)."""
    native.call("pcg_average_down", C.byref(abi.array4(fine)), C.byref(abi.array4(crse)), abi.ivec(fine_lo),
                abi.ivec(fine_hi), int(ratio), int(ncomp), _stream_ptr(stream))
