"""Loader and ctypes signatures of the native library (include/pcg_hydro.h).

There is no fallback: if the CUDA library cannot be loaded (or built in place on a
machine with nvcc), every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import threading

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "include", "pcg_hydro.h")

PCG_OK = 0
ERRORS = {-1: "PCG_EINVAL", -2: "PCG_ECUDA", -3: "PCG_ENOMEM", -4: "PCG_EUNSUPPORTED",
          -5: "PCG_ETIMEDOUT", -6: "PCG_EBUDGET", -7: "PCG_ENOEOS"}


class PcgError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} -> {ERRORS.get(code, code)}: {msg}")
        self.code = code


class Box(C.Structure):
    _fields_ = [
        ("lo", C.c_int32 * 3),
        ("hi", C.c_int32 * 3),
        ("domlo", C.c_int32 * 3),
        ("domhi", C.c_int32 * 3),
        ("bclo", C.c_int32 * 3),
        ("bchi", C.c_int32 * 3),
        ("dx", C.c_double * 3),
        ("dt", C.c_double),
        ("uin", abi.Array4),
        ("uout", abi.Array4),
        ("flx", abi.Array4 * 3),
    ]


_P = C.POINTER
_A4 = _P(abi.Array4)
_I3 = _P(C.c_int32)
_PRM = _P(abi.HydroParams)
_V = C.c_void_p

SIGNATURES = {
    "pcg_init": ([C.c_int], C.c_int),
    "pcg_last_error": ([], C.c_char_p),
    "pcg_set_eos_gamma": ([C.c_double, C.c_double], C.c_int),
    "pcg_set_eos_nasa7": ([C.c_int, _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(C.c_double)], C.c_int),
    "pcg_species_counts": ([_P(C.c_int32), C.c_int32], C.c_int),
    "pcg_fluxreg_create": ([C.c_int32, _I3, _I3, _I3, C.c_int32, C.c_int32, _I3, _I3, _P(_V)], C.c_int),
    "pcg_fluxreg_info": ([_V, _P(C.c_int32), _P(C.c_int32)], C.c_int),
    "pcg_fluxreg_reset": ([_V, _V], C.c_int),
    "pcg_fluxreg_crse_add": ([_V, _I3, _I3, _A4, C.c_double, _V], C.c_int),
    "pcg_fluxreg_fine_add": ([_V, _I3, _I3, _A4, C.c_double, _V], C.c_int),
    "pcg_fluxreg_reflux": ([_V, _A4, C.c_double, _V], C.c_int),
    "pcg_fluxreg_destroy": ([_V], C.c_int),
    "pcg_average_down": ([_A4, _A4, _I3, _I3, C.c_int32, C.c_int32, _V], C.c_int),
    "pcg_ctoprim": ([_PRM, _I3, _I3, _A4, _A4, _A4, _V], C.c_int),
    "pcg_umdrv": ([_PRM, _I3, _I3, _A4, _A4, _A4, _A4, _A4, _A4, _A4, _A4, _V], C.c_int),
    "pcg_srctoprim": ([_PRM, _I3, _I3, _A4, _A4, _A4, _A4, _V], C.c_int),
    "pcg_umeth": ([_PRM, _I3, _I3, _A4, _A4, _A4, _A4, _A4, _A4, _A4, _A4, _V], C.c_int),
    "pcg_hydro_box": ([_PRM, _I3, _I3, _A4, _A4, _A4, _V], C.c_int),
    "pcg_hydro_boxes": ([_PRM, C.c_int32, _P(Box), _V], C.c_int),
    "pcg_step_boxes": ([_PRM, C.c_int32, _P(Box), C.c_int32, C.c_double, _V, _V, _V], C.c_int),
    "pcg_hydro_workspace": ([_PRM, C.c_int32, _P(C.c_int32), _P(C.c_int32), _P(C.c_int64)], C.c_int),
    "pcg_trim_workspace": ([C.c_int32, C.c_int64], C.c_int),
    "pcg_reserve_workspace": ([C.c_int32, C.c_int64], C.c_int),
    "pcg_hydro_box_noalloc": ([_PRM, _I3, _I3, _A4, _A4, _A4, _V], C.c_int),
    "pcg_estdt": ([C.c_int32, C.c_int32, _P(Box), C.c_double, _V, _V], C.c_int),
    "pcg_update_state": ([C.c_int32, C.c_int32, _P(Box), _A4, _V, _V], C.c_int),
    "pcg_fill_ghosts": ([_A4, _I3, _I3, _I3, C.c_int32, _V], C.c_int),
    "pcg_copy_cells": ([_A4, _A4, _I3, _I3, _V], C.c_int),
    "pcg_plan_create": ([_PRM, C.c_int32, _P(Box), C.c_int32, _P(_V)], C.c_int),
    "pcg_plan_hydro": ([_V, _V, _V], C.c_int),
    "pcg_plan_stages": ([_V, C.c_int32, C.c_int32, _V, _V], C.c_int),
    "pcg_plan_estdt": ([_V, C.c_double, _V, _V], C.c_int),
    "pcg_plan_update": ([_V, _V, _V], C.c_int),
    "pcg_plan_advance": ([_V, C.c_double, _V, _V, _V], C.c_int),
    "pcg_plan_info": ([_V, _P(C.c_int64), _P(C.c_int32), _P(C.c_int64)], C.c_int),
    "pcg_plan_destroy": ([_V], C.c_int),
    "pcg_set_launch_variant": ([C.c_int32, C.c_int32, C.c_int32, C.c_int32], C.c_int),
    "pcg_get_launch_variant": ([C.c_int32, C.c_int32, C.c_int32], C.c_int),
}

_lib = None
_lock = threading.Lock()


def header_functions(path: str = HEADER):
    """Names of the functions declared in the public header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pcg_[a-z0-9_]+)\s*\(", text)))


def lib_path() -> str:
    """The library to load: PCG_LIB if set (an alternative build), else the in-tree
    build."""
    from .build import LIB
    return os.environ.get("PCG_LIB", LIB)


def load(build_if_missing: bool = True):
    """Load libpcg_hydro.so (building it in place if it is missing and nvcc exists)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = lib_path()
        if not os.path.exists(path):
            if not build_if_missing or "PCG_LIB" in os.environ:
                raise OSError(f"{path} is missing; run particleclem_b200/build.py")
            from .build import build
            build()
        lib = C.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


def call(name, *args):
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != PCG_OK:
        raise PcgError(name, rc, lib.pcg_last_error().decode())
    return rc
