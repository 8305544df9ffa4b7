"""ctypes wrapper of the CPU oracles (TEST INFRASTRUCTURE ONLY).

Two libraries share one C interface:
* ``oracle/_build/liboracle.so`` -- the plain-C restatement (always buildable: gcc);
* ``oracle/_ref/libpcg_ref_ns{1,9}.so`` -- the reference's own Godunov/PPM sources
  compiled in place against the AMReX-API shim (built only where the reference
  checkout exists; the built files travel with the repository snapshot).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from particleclem_b200 import abi
from particleclem_b200.thermo import GammaLaw

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
ORACLE_FAST_SO = os.path.join(HERE, "_build", "liboracle_omp.so")
REF_DIR = os.path.join(HERE, "_ref")


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def ref_so(nspec: int, fast: bool = False) -> str:
    return os.path.join(REF_DIR, f"libpcg_ref_{'fast_' if fast else ''}ns{nspec}.so")


def ref_available(nspec: int, fast: bool = False) -> bool:
    return os.path.exists(ref_so(nspec, fast))


def uniform_geometry(lo, hi, dx):
    """area[3] (face FABs) and vol (cell FAB) of a uniform Cartesian box, as PeleC's
    geom.GetFaceArea / GetVolume give them (Source/PeleC.cpp:605-617)."""
    area = []
    for d in range(3):
        nlo, nhi = abi.nodes(lo, hi, d)
        shp = tuple(nhi[e] - nlo[e] + 1 for e in (2, 1, 0))
        a = dx[(d + 1) % 3] * dx[(d + 2) % 3]
        area.append(abi.Fab(np.full((1,) + shp, a), nlo))
    shp = tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
    vol = abi.Fab(np.full((1,) + shp, dx[0] * dx[1] * dx[2]), tuple(lo))
    return area, vol


class CpuHydro:
    """One oracle library: prefix 'orc' (restatement) or 'ref' (reference build)."""

    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            if prefix == "orc":
                build_oracle()
            else:
                raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.prefix = prefix
        L = self.lib
        P = C.POINTER
        A4 = P(abi.Array4)
        I3 = P(C.c_int32)
        self._f("set_eos_gamma", [C.c_double, C.c_double], C.c_int)
        self._f("set_eos_nasa7", [C.c_int, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double)], C.c_int)
        self._f("ctoprim", [I3, I3, A4, A4, A4], C.c_int)
        self._f("umdrv", [P(abi.HydroParams), I3, I3, A4, A4, A4, A4, A4, A4, A4, A4], C.c_int)
        self._f("hydro_box", [P(abi.HydroParams), I3, I3, A4, A4, A4, A4, A4], C.c_int)
        self._f("srctoprim", [I3, I3, A4, A4, A4, A4], C.c_int)
        self._f("umeth", [P(abi.HydroParams), I3, I3, A4, A4, A4, A4, A4, A4, A4, A4], C.c_int)
        self._f("estdt", [I3, I3, A4, P(C.c_double)], C.c_double)
        self._f("update_state", [I3, I3, A4, A4, C.c_double, A4], C.c_int)
        self.eos = None

    def _f(self, name, argtypes, restype):
        fn = getattr(self.lib, f"{self.prefix}_{name}")
        fn.argtypes = argtypes
        fn.restype = restype
        setattr(self, "_" + name, fn)

    def set_eos(self, eos):
        if isinstance(eos, GammaLaw):
            rc = self._set_eos_gamma(eos.gamma, eos.mw)
        else:
            d = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))
            mw, tm, lo, hi = (np.ascontiguousarray(x, dtype=np.float64) for x in (eos.mw, eos.tmid, eos.a_lo, eos.a_hi))
            rc = self._set_eos_nasa7(eos.nspec, d(mw), d(tm), d(lo), d(hi))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}: set_eos failed ({rc})")
        self.eos = eos

    def hydro_box(self, prm, lo, hi, uin: abi.Fab, area=None, vol=None):
        """construct_hydro_source for one box: returns (hydro_source FAB, [flx FABs])."""
        nv = abi.nvar(self.eos.nspec)
        shp = tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
        uout = abi.Fab(np.zeros((nv,) + shp), tuple(lo))
        flx = []
        for d in range(3):
            nlo, nhi = abi.nodes(lo, hi, d)
            flx.append(abi.Fab(np.zeros((nv,) + tuple(nhi[e] - nlo[e] + 1 for e in (2, 1, 0))), nlo))
        if area is None:
            area, vol = uniform_geometry(lo, hi, tuple(prm.dx))
        rc = self._hydro_box(C.byref(prm), abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(uin)),
                             C.byref(abi.array4(uout)), abi.array4_list(flx), abi.array4_list(area),
                             C.byref(abi.array4(vol)))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}_hydro_box returned {rc}")
        return uout, flx

    def ctoprim(self, lo, hi, u: abi.Fab):
        ns = self.eos.nspec
        shp = tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
        q = abi.Fab(np.zeros((abi.qvar(ns),) + shp), tuple(lo))
        qa = abi.Fab(np.zeros((abi.NQAUX,) + shp), tuple(lo))
        rc = self._ctoprim(abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(u)), C.byref(abi.array4(q)),
                           C.byref(abi.array4(qa)))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}_ctoprim returned {rc}")
        return q, qa

    def srctoprim(self, lo, hi, q: abi.Fab, qa: abi.Fab, src: abi.Fab):
        """pc_srctoprim over [lo, hi]: the primitive sources srcQ (QVAR components)."""
        shp = tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
        sq = abi.Fab(np.zeros((abi.qvar(self.eos.nspec),) + shp), tuple(lo))
        rc = self._srctoprim(abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(q)), C.byref(abi.array4(qa)),
                             C.byref(abi.array4(src)), C.byref(abi.array4(sq)))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}_srctoprim returned {rc}")
        return sq

    def umeth(self, prm, lo, hi, q: abi.Fab, qa: abi.Fab, srcq=None, area=None, vol=None):
        """pc_umeth_3D alone: returns (flx[3], qec[3], pdivu) on the faces / cells of the box;
        qec component GDRHO is left zero (the reference does not write it)."""
        nv = abi.nvar(self.eos.nspec)
        flx, qec = [], []
        for d in range(3):
            nlo, nhi = abi.nodes(lo, hi, d)
            shp = tuple(nhi[e] - nlo[e] + 1 for e in (2, 1, 0))
            flx.append(abi.Fab(np.zeros((nv,) + shp), nlo))
            qec.append(abi.Fab(np.zeros((abi.NGDNV,) + shp), nlo))
        shp = tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
        pdivu = abi.Fab(np.zeros((1,) + shp), tuple(lo))
        if area is None:
            area, vol = uniform_geometry(lo, hi, tuple(prm.dx))
        rc = self._umeth(C.byref(prm), abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(q)), C.byref(abi.array4(qa)),
                         C.byref(abi.array4(srcq)) if srcq is not None else None, abi.array4_list(flx),
                         abi.array4_list(qec), abi.array4_list(area), C.byref(abi.array4(pdivu)),
                         C.byref(abi.array4(vol)))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}_umeth returned {rc}")
        return flx, qec, pdivu

    def estdt(self, lo, hi, u: abi.Fab, dx):
        dxa = (C.c_double * 3)(*dx)
        return self._estdt(abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(u)), dxa)

    def update_state(self, lo, hi, s_old: abi.Fab, hsrc: abi.Fab, dt):
        s_new = abi.Fab(np.zeros_like(s_old.data), s_old.lo)
        rc = self._update_state(abi.ivec(lo), abi.ivec(hi), C.byref(abi.array4(s_old)), C.byref(abi.array4(hsrc)),
                                float(dt), C.byref(abi.array4(s_new)))
        if rc != 0:
            raise RuntimeError(f"{self.prefix}_update_state returned {rc}")
        return s_new


def oracle(fast: bool = False) -> CpuHydro:
    return CpuHydro(ORACLE_FAST_SO if fast else ORACLE_SO, "orc")


def reference(nspec: int, fast: bool = False) -> CpuHydro:
    return CpuHydro(ref_so(nspec, fast), "ref")


def rel_errors(got: np.ndarray, ref: np.ndarray, floor: float = 0.0):
    """Per-component relative L1 and Linf errors (components on axis 0):
    rel-L1 = sum|g-r| / sum|r|, rel-Linf = max|g-r| / max|r|; a component whose
    reference is identically zero is compared against ``floor`` instead."""
    g = got.reshape(got.shape[0], -1)
    r = ref.reshape(ref.shape[0], -1)
    d = np.abs(g - r)
    s1 = np.abs(r).sum(axis=1)
    sinf = np.abs(r).max(axis=1)
    l1 = d.sum(axis=1) / np.where(s1 > 0, s1, 1.0)
    linf = d.max(axis=1) / np.where(sinf > 0, sinf, 1.0)
    zero = sinf == 0
    if floor > 0:
        l1 = np.where(zero, d.max(axis=1) / floor, l1)
        linf = np.where(zero, d.max(axis=1) / floor, linf)
    return l1, linf
