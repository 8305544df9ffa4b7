"""CPU oracle of the coarse/fine calls (test infrastructure only: the tests compare the
device flux register, reflux and average-down against it; nothing in the product path
imports it).

The register is AMReX's (EBFluxRegister / YAFluxRegister on regular boxes), which the
reference calls through PeleC::update_flux_registers (Source/PeleC.cpp:1343-1400: CrseAdd,
FineAdd with area-weighted fluxes and the cell volume as dx) and PeleC::reflux
(Source/PeleC.cpp:1403-1414). AMReX is not in the reference checkout, so its published
algorithm (conservative refluxing, Berger & Colella, J. Comput. Phys. 82, 1989) is
restated here in plain Python loops with the operation order of the device kernels:

* one accumulator per coarse face on the coarse/fine boundary, for the coarse cell c
  outside the fine region; s = +1 where the face is c's low face, -1 where it is c's high
  face; faces on non-periodic domain boundaries and between two fine boxes have none;
* CrseAdd of a coarse box: acc -= s * (dt * F_c) for the register faces of its cells
  (AMReX: d -= dtdx fx(i) where the cell below is fine, d += dtdx fx(i+1) where the cell
  above is fine);
* FineAdd of a fine box: acc += s * (dt * sum of the ratio^2 fine faces), the sum taken
  with the second transverse direction outermost;
* Reflux: S_c += acc * (1 / vol) per register face of c, faces of a cell in creation
  order (cells in k, j, i order);
* average-down: coarse = (sum of the ratio^3 fine cells, i fastest) * (1 / ratio^3).

Parity against AMReX itself is unpinned (AMReX is absent); the conservation of a two-level
advance pins the algorithm (tests/test_gpu_fluxreg.py).
"""
from __future__ import annotations

import numpy as np


def _fdiv(a, b):
    return a // b  # Python's floor division, as the library's floordiv


def _at(fab, i, j, k, n):
    """Element (i, j, k, n) of a FAB (data [n][k][j][i], lo)."""
    lo = fab.lo
    return fab.data[n, k - lo[2], j - lo[1], i - lo[0]]


class FluxRegister:
    def __init__(self, ncomp, crse_domlo, crse_domhi, periodic, ratio, fine_boxes):
        self.ncomp, self.ratio = int(ncomp), int(ratio)
        self.fine_boxes = [(tuple(lo), tuple(hi)) for lo, hi in fine_boxes]
        dn = [crse_domhi[d] - crse_domlo[d] + 1 for d in range(3)]
        cb = []
        for lo, hi in self.fine_boxes:
            for d in range(3):
                assert lo[d] % ratio == 0 and (hi[d] + 1) % ratio == 0, "fine box not aligned"
            cb.append(([_fdiv(lo[d], ratio) for d in range(3)], [_fdiv(hi[d] + 1, ratio) - 1 for d in range(3)]))

        def covered(c):
            return any(all(l[d] <= c[d] <= h[d] for d in range(3)) for l, h in cb)

        entries = []
        for b, ((flo, fhi), (clo, chi)) in enumerate(zip(self.fine_boxes, cb)):
            for d in range(3):
                t1, t2 = (1, 2) if d == 0 else ((0, 2) if d == 1 else (0, 1))
                for side in (0, 1):
                    for v in range(clo[t2], chi[t2] + 1):
                        for u in range(clo[t1], chi[t1] + 1):
                            c = [0, 0, 0]
                            f = [0, 0, 0]
                            c[t1], c[t2] = u, v
                            c[d] = clo[d] - 1 if side == 0 else chi[d] + 1
                            f[t1], f[t2] = u * ratio, v * ratio
                            sgn = -1 if side == 0 else 1
                            fface = flo[d] if side == 0 else fhi[d] + 1
                            if c[d] < crse_domlo[d] or c[d] > crse_domhi[d]:
                                if not periodic[d]:
                                    continue
                                c[d] += dn[d] if c[d] < crse_domlo[d] else -dn[d]
                            if covered(c):
                                continue
                            entries.append({"c": tuple(c), "f": tuple(f), "dir": d, "sgn": sgn, "fbox": b,
                                            "fface": fface})
        entries.sort(key=lambda e: (e["c"][2], e["c"][1], e["c"][0]))  # stable: creation order within a cell
        self.entries = entries
        self.acc = np.zeros((len(entries), self.ncomp))

    def reset(self):
        self.acc[:] = 0.0

    def crse_add(self, lo, hi, flx, dt):
        for t, e in enumerate(self.entries):
            c = e["c"]
            if not all(lo[d] <= c[d] <= hi[d] for d in range(3)):
                continue
            q = list(c)
            if e["sgn"] < 0:
                q[e["dir"]] += 1
            F = flx[e["dir"]]
            for n in range(self.ncomp):
                self.acc[t, n] = self.acc[t, n] - float(e["sgn"]) * (dt * _at(F, q[0], q[1], q[2], n))

    def fine_add(self, lo, hi, flx, dt):
        box = self.fine_boxes.index((tuple(lo), tuple(hi)))
        r = self.ratio
        for t, e in enumerate(self.entries):
            if e["fbox"] != box:
                continue
            d = e["dir"]
            t1, t2 = (1, 2) if d == 0 else ((0, 2) if d == 1 else (0, 1))
            F = flx[d]
            for n in range(self.ncomp):
                s = 0.0
                for b in range(r):
                    for a in range(r):
                        q = [0, 0, 0]
                        q[d] = e["fface"]
                        q[t1] = e["f"][t1] + a
                        q[t2] = e["f"][t2] + b
                        s = s + _at(F, q[0], q[1], q[2], n)
                self.acc[t, n] = self.acc[t, n] + float(e["sgn"]) * (dt * s)

    def reflux(self, s_crse, vol):
        inv = 1.0 / vol
        lo = s_crse.lo
        t = 0
        while t < len(self.entries):
            c = self.entries[t]["c"]
            u = t
            while u < len(self.entries) and self.entries[u]["c"] == c:
                u += 1
            for n in range(self.ncomp):
                v = s_crse.data[n, c[2] - lo[2], c[1] - lo[1], c[0] - lo[0]]
                for b in range(t, u):
                    v = v + self.acc[b, n] * inv
                s_crse.data[n, c[2] - lo[2], c[1] - lo[1], c[0] - lo[0]] = v
            t = u


def average_down(fine, crse, fine_lo, fine_hi, ratio, ncomp):
    w = 1.0 / float(ratio * ratio * ratio)
    clo = [_fdiv(fine_lo[d], ratio) for d in range(3)]
    chi = [_fdiv(fine_hi[d] + 1, ratio) - 1 for d in range(3)]
    for k in range(clo[2], chi[2] + 1):
        for j in range(clo[1], chi[1] + 1):
            for i in range(clo[0], chi[0] + 1):
                for n in range(ncomp):
                    s = 0.0
                    for cc in range(ratio):
                        for b in range(ratio):
                            for a in range(ratio):
                                s = s + _at(fine, i * ratio + a, j * ratio + b, k * ratio + cc, n)
                    crse.data[n, k - crse.lo[2], j - crse.lo[1], i - crse.lo[0]] = s * w
