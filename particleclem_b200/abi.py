"""ctypes mirror of the C-ABI in include/pcg_hydro.h, and a small FAB helper.

A FAB here is a block of memory laid out exactly like ``amrex::FArrayBox`` /
``amrex::Array4``: component-major, then k, j, i with i fastest, covering the index box
``[lo, hi]``. In numpy/torch that is a C-contiguous array of shape
``(ncomp, nz, ny, nx)``. :func:`array4` turns one into the ``pcg_array4`` descriptor
the library takes (the same addressing as ``amrex::Array4``:
``p[(i-b0) + (j-b1)*js + (k-b2)*ks + n*ns]``, ``end`` exclusive).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

# ------------------------------------------------------------------ constants
# Source/IndexDefines.H:6-89 (NUM_ADV = NUM_AUX = NUM_LIN = 0)
URHO, UMX, UMY, UMZ, UEDEN, UEINT, UTEMP, UFS = range(8)
QRHO, QU, QV, QW, QGAME, QPRES, QREINT, QTEMP, QFS = range(9)
QGAMC, QC, QCSML, QDPDR, QDPDE, QRSPEC = range(6)
NQAUX = 6
NGDNV = 6
NGROW = 4  # PeleC::numGrow() for regular geometry (Source/PeleC.H:922-950)

# Source/PeleC.H:49-57
BC_INTERIOR, BC_INFLOW, BC_OUTFLOW, BC_SYMMETRY, BC_SLIP_WALL, BC_NO_SLIP_WALL, BC_USER = range(7)

# precision_mode values of pcg_hydro_params
PREC_FP64 = 0  # plain FP64, reference operation order, no FMA contraction
PREC_FP64_FAST = 1  # FP64 with FMA contraction
PREC_MIXED = 2  # FP32 trace/Riemann/transverse, FP64 update, Newton and dt


def nvar(nspec: int) -> int:
    return 7 + nspec


def qvar(nspec: int) -> int:
    return 8 + nspec


class Array4(C.Structure):
    _fields_ = [
        ("p", C.c_void_p),
        ("jstride", C.c_int64),
        ("kstride", C.c_int64),
        ("nstride", C.c_int64),
        ("begin", C.c_int32 * 3),
        ("end", C.c_int32 * 3),
        ("ncomp", C.c_int32),
    ]


class HydroParams(C.Structure):
    _fields_ = [
        ("dx", C.c_double * 3),
        ("dt", C.c_double),
        ("difmag", C.c_double),
        ("ppm_type", C.c_int32),
        ("plm_iorder", C.c_int32),
        ("use_flattening", C.c_int32),
        ("use_hybrid_weno", C.c_int32),
        ("weno_scheme", C.c_int32),
        ("domlo", C.c_int32 * 3),
        ("domhi", C.c_int32 * 3),
        ("bclo", C.c_int32 * 3),
        ("bchi", C.c_int32 * 3),
        ("nspec", C.c_int32),
        ("precision_mode", C.c_int32),
    ]


def make_params(dx, dt, nspec, domlo, domhi, bclo, bchi, ppm_type=1, plm_iorder=4,
                use_flattening=True, difmag=0.1, precision_mode=PREC_FP64, use_hybrid_weno=False,
                weno_scheme=1) -> HydroParams:
    """Parameter block with PeleC's defaults (Source/Params/_cpp_parameters: difmag 0.1,
    plm_iorder 4, use_flattening true; hybrid WENO off, weno_scheme 1)."""
    p = HydroParams()
    p.dx[:] = [float(v) for v in dx]
    p.dt = float(dt)
    p.difmag = float(difmag)
    p.ppm_type = int(ppm_type)
    p.plm_iorder = int(plm_iorder)
    p.use_flattening = int(bool(use_flattening))
    p.use_hybrid_weno = int(bool(use_hybrid_weno))
    p.weno_scheme = int(weno_scheme)
    p.domlo[:] = [int(v) for v in domlo]
    p.domhi[:] = [int(v) for v in domhi]
    p.bclo[:] = [int(v) for v in bclo]
    p.bchi[:] = [int(v) for v in bchi]
    p.nspec = int(nspec)
    p.precision_mode = int(precision_mode)
    return p


@dataclass
class Fab:
    """A FAB: ``data`` of shape (ncomp, nz, ny, nx) covering cells [lo, hi]."""

    data: object  # numpy.ndarray or torch.Tensor, float64, C-contiguous
    lo: tuple

    @property
    def hi(self):
        nz, ny, nx = self.data.shape[1:]
        return (self.lo[0] + nx - 1, self.lo[1] + ny - 1, self.lo[2] + nz - 1)

    @property
    def ncomp(self):
        return self.data.shape[0]

    def view(self, lo, hi):
        """numpy/torch view of the sub-box [lo, hi] (all components)."""
        s = [slice(lo[d] - self.lo[d], hi[d] - self.lo[d] + 1) for d in range(3)]
        return self.data[:, s[2], s[1], s[0]]


def _ptr(data) -> int:
    if isinstance(data, np.ndarray):
        return data.ctypes.data
    return data.data_ptr()  # torch.Tensor


def array4(fab: Fab) -> Array4:
    d = fab.data
    if isinstance(d, np.ndarray):
        if not d.flags["C_CONTIGUOUS"]:
            raise ValueError("FAB data must be C-contiguous")
    elif not d.is_contiguous():
        raise ValueError("FAB data must be contiguous")
    nc, nz, ny, nx = d.shape
    a = Array4()
    a.p = _ptr(d)
    a.jstride = nx
    a.kstride = nx * ny
    a.nstride = nx * ny * nz
    a.begin[:] = list(fab.lo)
    a.end[:] = [fab.lo[0] + nx, fab.lo[1] + ny, fab.lo[2] + nz]
    a.ncomp = nc
    return a


def array4_list(fabs):
    arr = (Array4 * len(fabs))()
    for i, f in enumerate(fabs):
        arr[i] = array4(f)
    return arr


def ivec(v):
    return (C.c_int32 * 3)(*[int(x) for x in v])


def grow(lo, hi, n):
    return tuple(l - n for l in lo), tuple(h + n for h in hi)


def nodes(lo, hi, d):
    h = list(hi)
    h[d] += 1
    return tuple(lo), tuple(h)
