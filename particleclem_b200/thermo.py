"""Thermodynamics tables for the hydro path's EOS.

Two EOS kinds are supported, matching the two PelePhysics EOS models the reference's
Godunov configurations use (PeleC selects them at build time with ``Eos_Model``):

* ``GammaLaw``: a single species with constant ratio of specific heats
  (``Exec/RegTests/Sod/GNUmakefile:30``).
* ``Fuego``-style ideal-gas mixture: per-species NASA-7 polynomials, two temperature
  ranges (``Exec/RegTests/PMF/GNUmakefile:31-33``).

The 9-species table shipped here (``data/h2air_standin_nasa7.dat``) is a STAND-IN made by
``data/make_standin_thermo.py`` because the real mechanism's coefficients are not
available; any table in the same format can replace it.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

RU = 8.31446261815324e7  # erg / (mol K), CGS as in Pele
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
STANDIN_TABLE = os.path.join(DATA_DIR, "h2air_standin_nasa7.dat")
H2AIR_SPECIES = ("H2", "O2", "H2O", "H", "O", "OH", "HO2", "H2O2", "N2")
AIR_MW = 28.97


@dataclass
class GammaLaw:
    gamma: float = 1.4
    mw: float = AIR_MW
    nspec: int = field(default=1, init=False)
    kind: int = field(default=0, init=False)


@dataclass
class Nasa7Mixture:
    names: tuple
    mw: np.ndarray  # [nspec]
    tmid: np.ndarray  # [nspec]
    a_lo: np.ndarray  # [nspec, 7]
    a_hi: np.ndarray  # [nspec, 7]
    kind: int = field(default=1, init=False)

    @property
    def nspec(self) -> int:
        return len(self.names)

    def index(self, name: str) -> int:
        return self.names.index(name)

    # numpy evaluations (vectorised, used by the state generators only)
    def _coef(self, T):
        T = np.asarray(T, dtype=np.float64)
        lo = T[..., None] < self.tmid
        return np.where(lo[..., None], self.a_lo, self.a_hi)  # [..., nspec, 7]

    def e_species(self, T):
        """Mass-specific internal energy of each species, erg/g, shape [..., nspec]."""
        a = self._coef(T)
        T = np.asarray(T, dtype=np.float64)[..., None]
        h_rt = a[..., 5] + T * (a[..., 0] + T * (a[..., 1] / 2 + T * (a[..., 2] / 3 + T * (a[..., 3] / 4 + T * a[..., 4] / 5))))
        return RU / self.mw * (h_rt - T)

    def cv_species(self, T):
        a = self._coef(T)
        T = np.asarray(T, dtype=np.float64)[..., None]
        cp_r = a[..., 0] + T * (a[..., 1] + T * (a[..., 2] + T * (a[..., 3] + T * a[..., 4])))
        return RU / self.mw * (cp_r - 1.0)


def load_nasa7(path: str = STANDIN_TABLE) -> Nasa7Mixture:
    lines = [ln for ln in open(path).read().splitlines() if ln.strip() and not ln.startswith("#")]
    if len(lines) % 3:
        raise ValueError(f"{path}: expected 3 lines per species")
    names, mw, tmid, lo, hi = [], [], [], [], []
    for s in range(len(lines) // 3):
        head = lines[3 * s].split()
        names.append(head[0])
        mw.append(float(head[1]))
        tmid.append(float(head[3]))
        lo.append([float(v) for v in lines[3 * s + 1].split()])
        hi.append([float(v) for v in lines[3 * s + 2].split()])
    return Nasa7Mixture(tuple(names), np.array(mw), np.array(tmid), np.array(lo), np.array(hi))


def standin_mixture(nspec: int, base: Nasa7Mixture = None) -> Nasa7Mixture:
    """A NASA-7 table of ``nspec`` species (2 or more) built from the 9-species stand-in,
    for exercising species counts other than 9 (mechanisms of 2, 3 or 21 species have
    those sizes). It is a synthetic table, not a real mechanism: up to
    9 species it is the first ``nspec - 1`` stand-in species plus N2; above 9, the nine
    plus species whose polynomials repeat the stand-in's (cycling through them) with the
    molecular weight scaled by 1 + 0.1 m for the m-th repeat, so that every species has
    distinct thermodynamics in mass units."""
    base = base or load_nasa7()
    if nspec < 2:
        raise ValueError("a mixture has 2 or more species")
    if nspec <= base.nspec:
        idx = list(range(nspec - 1)) + [base.nspec - 1]
        return Nasa7Mixture(tuple(base.names[k] for k in idx), base.mw[idx].copy(), base.tmid[idx].copy(),
                            base.a_lo[idx].copy(), base.a_hi[idx].copy())
    names, mw, tmid, lo, hi = list(base.names), list(base.mw), list(base.tmid), list(base.a_lo), list(base.a_hi)
    for m in range(nspec - base.nspec):
        k = m % base.nspec
        names.append(f"{base.names[k]}_x{m + 1}")
        mw.append(base.mw[k] * (1.0 + 0.1 * (m + 1)))
        tmid.append(base.tmid[k])
        lo.append(base.a_lo[k])
        hi.append(base.a_hi[k])
    return Nasa7Mixture(tuple(names), np.array(mw), np.array(tmid), np.array(lo), np.array(hi))

