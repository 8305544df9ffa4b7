"""Roofline arithmetic for the hydro path.

Algorithmic bytes are the bytes a stage must move at least once: every input element
it reads and every output element it writes, each counted once per launch (no stencil
re-reads). For a region of valid edges (nx, ny, nz), NS species, compute-type size
``r`` (8 FP64, 4 mixed) and NT = 6 + NS, NF = 7 + NS, NVAR = 7 + NS, QVAR = 8 + NS:

* ctoprim: read NVAR doubles and write QVAR + 6 doubles per cell of grow(box, 4); the
           mixed form (r = 4) also writes the FP32 copy of NT primitives on grow(box, 3)
* prep:    read (5 + NS) q doubles per cell of grow(box, 4); write 2 r per cell of
           grow(box, 1) and one double per node of the box
* trace:   read (5 + NS) q doubles per cell of grow(box, 3) (PLM: 6 + NS); write
           2 NT r per cell of grow(box, 1) per direction
* flux0:   per direction, read 2 NT r and write NF r per face of
           faces_d(grow(box,1) shrunk by one along d)
* flux1:   per direction D, read the two D-states (2 NT r) per D-face and the two
           O-fluxes (NF r) per O-face of those regions, write NF r per face of
           both (D|O) flux arrays
* flux2:   per direction, read 2 NT r per face, the two corrected fluxes (NF r per face
           of their regions), NVAR doubles of u and one divu per face; write NVAR + 2
           values per face of the box (FP32 in the mixed form without flux export)
* consup:  read 3 (NVAR + 2) final-flux values per face, write NVAR doubles per cell

The path-level figure is B_alg = 8 NVAR [(nx+8)(ny+8)(nz+8) + nx ny nz]
bytes per box (read the grown state once, write the hydro source once).
"""
from __future__ import annotations

import json
import os
import re

FALLBACK_HBM_GBS = 6650.0  # earlier measurement on this pool, used only without MEASURED_PEAKS.json


def peaks(root):
    path = os.path.join(root, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": FALLBACK_HBM_GBS, "source": "fallback"}


def _cells(n, g):
    return (n[0] + 2 * g) * (n[1] + 2 * g) * (n[2] + 2 * g)


def _faces(n, d, grow_other):
    m = [n[e] + 2 * grow_other for e in range(3)]
    m[d] = n[d] + 1
    return m[0] * m[1] * m[2]


def stage_bytes(stage, n, ns, r, ppm=True):
    """Algorithmic bytes of one launch of a hydro stage over one region of edges n."""
    nt, nf, nv, nq = 6 + ns, 7 + ns, 7 + ns, 8 + ns
    ff = 4 if r == 4 else 8  # final-flux element size
    if stage == "ctoprim":
        return _cells(n, 4) * 8 * (nv + nq + 6) + (_cells(n, 3) * nt * 4 if r == 4 else 0)
    if stage == "prep":
        nodes = (n[0] + 1) * (n[1] + 1) * (n[2] + 1)
        return _cells(n, 4) * 8 * (5 + ns) + _cells(n, 1) * 2 * r + nodes * 8
    if stage == "trace":
        rd = (5 + ns) if ppm else (6 + ns)
        return _cells(n, 3) * 8 * rd + 3 * _cells(n, 1) * 2 * nt * r
    if stage == "flux0":
        return sum(_faces(n, d, 1) * (2 * nt + nf) * r for d in range(3))
    if stage == "flux1":
        tot = 0
        for d in range(3):
            tot += _faces(n, d, 1) * 2 * nt * r  # D-states
            for o in range(3):
                if o == d:
                    continue
                t = 3 - d - o
                m = [n[0], n[1], n[2]]
                m[d] += 1
                m[t] += 2
                tot += m[0] * m[1] * m[2] * nf * r  # written (D|O) fluxes
        tot += sum(_faces(n, o, 1) * nf * r for o in range(3)) * 2  # each O-flux feeds two pairs
        return tot
    if stage == "flux2":
        tot = 0
        for d in range(3):
            f = _faces(n, d, 0)
            tot += f * (2 * nt * r + 2 * nf * r + nv * 8 + 8 + (nv + 2) * ff)
        return tot
    if stage == "consup":
        return sum(_faces(n, d, 0) * (nv + 2) * ff for d in range(3)) + n[0] * n[1] * n[2] * nv * 8
    raise ValueError(stage)


def b_alg_box(n, ns):
    nv = 7 + ns
    return 8 * nv * ((n[0] + 8) * (n[1] + 8) * (n[2] + 8) + n[0] * n[1] * n[2])


def traffic_table(root):
    """DRAM bytes per launch per kernel from profiles/dram_traffic.md (rows
    '| kernel | form | bytes |'), or {} if absent."""
    path = os.path.join(root, "profiles", "dram_traffic.md")
    out = {}
    try:
        for ln in open(path):
            m = re.match(r"\|\s*(k_\w+)\s*\|\s*(\w+)\s*\|\s*([0-9.eE+]+)\s*\|", ln)
            if m:
                out[(m.group(1), m.group(2))] = float(m.group(3))
    except OSError:
        pass
    return out


def dominant_kernel_roofline(region_edges, ns, r, stage_names, stage_ms, pk, form, root):
    """Roofline of the slowest hydro stage of one step (CUDA-event time per launch)."""
    hyd = [(ms, nm) for nm, ms in zip(stage_names, stage_ms) if nm.startswith("hydro.")]
    ms, nm = max(hyd)
    st = nm.split(".", 1)[1]
    byts = stage_bytes(st, region_edges, ns, r)
    achieved = byts / (ms * 1e-3) / 1e9
    tr = traffic_table(root).get(("k_" + st, form))
    return {"bound": "hbm", "kernel": "k_" + st, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "traffic": tr, "algorithmic_bytes_per_launch": byts,
            "launch_ms": ms, "share_of_step": ms / sum(v for n, v in zip(stage_names, stage_ms) if n != "advance"),
            "peak_source": pk["source"]}


def path_roofline(box_edges_list, ns, ms_per_step, pk):
    byts = sum(b_alg_box(n, ns) for n in box_edges_list)
    achieved = byts / (ms_per_step * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "algorithmic_bytes_per_step": byts, "peak_source": pk["source"],
            "note": "B_alg = 8*NVAR*[(n+8)^3 + n^3] per box: the path is FP64/FP32-ALU bound, not HBM bound"}
