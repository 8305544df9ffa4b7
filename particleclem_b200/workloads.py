"""Seeded synthetic states for the hydro path's workloads.

There is no public dataset for this path; every input is generated here from fixed
seeds. Each generator returns conserved states laid out as PeleC ``State_Type`` FABs:
components ``URHO, UMX, UMY, UMZ, UEDEN, UEINT, UTEMP, UFS..UFS+nspec-1``
(``Source/IndexDefines.H:6-13``), with ``NGROW = 4`` ghost cells.

Workloads (sizes as named by the benchmark configurations):

* ``sod``: one 32^3 box, single-species gamma = 1.4 gas, planar Sod discontinuity along
  x (rho 1 / 0.125, p 1 / 0.1, u = 0) with a seeded +-1 % uniform density perturbation;
  dx = 1/32, periodic in y/z, outflow in x.
* ``flame``: 9-species H2/air (stand-in NASA-7 thermo) on a periodic-in-x/y,
  outflow-in-z level of edge ``n`` (128 for the production case), CGS units,
  p = 1 atm, T following a tanh flame front 300 K -> 2200 K along z (width 0.05 cm)
  with seeded +-2 % sinusoidal wrinkling in x/y, unburnt stoichiometric H2/air
  blending to H2O/N2 with small OH/H/O/HO2 peaks, u_z = 1000 cm/s with seeded
  +-100 cm/s noise per component.
* ``flame_boxes``: independent boxes (edges given) from the flame generator with a
  per-box random flame offset; ghost cells come from the generator itself.
* ``turbulence``: periodic cube, single-species gamma = 1.4, rho = 1 +- 1 % noise,
  p = 1/gamma, divergence-free random velocity with a k^-5/3 spectrum over
  k = 1..kmax scaled to turbulent Mach 0.3.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .thermo import RU, GammaLaw, Nasa7Mixture, load_nasa7

NG = abi.NGROW


@dataclass
class Level:
    """One AMR level: a domain-sized state with a NG-cell halo plus its box list."""

    eos: object
    dx: tuple
    domlo: tuple
    domhi: tuple
    bclo: tuple
    bchi: tuple
    state: np.ndarray  # (NVAR, NZ+2NG, NY+2NG, NX+2NG), covers grow(domain, NG)
    boxes: list = field(default_factory=list)  # list of (lo, hi)
    periodic: tuple = (False, False, False)

    @property
    def nspec(self):
        return self.eos.nspec

    @property
    def fab(self) -> abi.Fab:
        return abi.Fab(self.state, tuple(l - NG for l in self.domlo))

    def box_fab(self, lo, hi, ng=NG) -> abi.Fab:
        """Copy of the grown box [lo-ng, hi+ng] as its own FAB."""
        glo, ghi = abi.grow(lo, hi, ng)
        return abi.Fab(np.ascontiguousarray(self.fab.view(glo, ghi)), glo)

    def fill_ghosts(self):
        fill_ghosts(self.state, self.periodic)

    def ncells(self):
        return sum(int(np.prod([h - l + 1 for l, h in zip(lo, hi)])) for lo, hi in self.boxes)


def fill_ghosts(state: np.ndarray, periodic, ng: int = NG):
    """Single-level FillBoundary: periodic wrap where periodic, else zero-gradient
    (first-order extrapolation, the ``foextrap`` fill PeleC uses for outflow)."""
    for d in range(3):
        ax = 3 - d  # numpy axis of direction d
        n = state.shape[ax] - 2 * ng
        lo_g = [slice(None)] * 4
        hi_g = [slice(None)] * 4
        if periodic[d]:
            lo_g[ax] = slice(0, ng)
            src = [slice(None)] * 4
            src[ax] = slice(n, n + ng)
            state[tuple(lo_g)] = state[tuple(src)]
            hi_g[ax] = slice(n + ng, n + 2 * ng)
            src[ax] = slice(ng, 2 * ng)
            state[tuple(hi_g)] = state[tuple(src)]
        else:
            for g in range(ng):
                lo_g[ax] = slice(g, g + 1)
                src = [slice(None)] * 4
                src[ax] = slice(ng, ng + 1)
                state[tuple(lo_g)] = state[tuple(src)]
                hi_g[ax] = slice(n + ng + g, n + ng + g + 1)
                src[ax] = slice(n + ng - 1, n + ng)
                state[tuple(hi_g)] = state[tuple(src)]


def tile_boxes(n, box):
    """Split a domain of edges n (tuple) into boxes of edge box (tuple)."""
    out = []
    for k in range(0, n[2], box[2]):
        for j in range(0, n[1], box[1]):
            for i in range(0, n[0], box[0]):
                out.append(((i, j, k), (min(i + box[0], n[0]) - 1, min(j + box[1], n[1]) - 1,
                                        min(k + box[2], n[2]) - 1)))
    return out


# ------------------------------------------------------------------ EOS helpers (numpy)
def _rmix(eos, Y):
    if isinstance(eos, GammaLaw):
        return RU * Y[0] / eos.mw
    return RU * np.tensordot(Y, 1.0 / eos.mw, axes=([0], [0]))


def conserved_from_prim(eos, rho, u, v, w, p, Y):
    """Conserved FAB components from primitive fields (numpy arrays of equal shape;
    Y has a leading species axis)."""
    nspec = eos.nspec
    rmix = _rmix(eos, Y)
    T = p / (rho * rmix)
    if isinstance(eos, GammaLaw):
        e = p / ((eos.gamma - 1.0) * rho)
    else:
        es = eos.e_species(T)  # [..., nspec]
        e = np.einsum("s...,...s->...", Y, es)
    U = np.empty((7 + nspec,) + rho.shape)
    U[abi.URHO] = rho
    U[abi.UMX] = rho * u
    U[abi.UMY] = rho * v
    U[abi.UMZ] = rho * w
    U[abi.UEINT] = rho * e
    U[abi.UEDEN] = rho * e + 0.5 * rho * (u * u + v * v + w * w)
    U[abi.UTEMP] = T
    U[abi.UFS:] = rho[None] * Y
    return U


# ------------------------------------------------------------------ Sod (config 1)
def sod(n=32, seed=1, gamma=1.4) -> Level:
    eos = GammaLaw(gamma=gamma)
    N = n + 2 * NG
    dx = 1.0 / n
    x = (np.arange(N) - NG + 0.5) * dx
    X = np.broadcast_to(x[None, None, :], (N, N, N))
    rho = np.where(X < 0.5, 1.0, 0.125)
    p = np.where(X < 0.5, 1.0, 0.1)
    rng = np.random.default_rng(seed)
    pert = rng.uniform(-1.0, 1.0, size=(n, n, n))
    rho = rho.copy()
    rho[NG:-NG, NG:-NG, NG:-NG] *= 1.0 + 0.01 * pert
    z = np.zeros_like(rho)
    U = conserved_from_prim(eos, rho, z, z, z, p, np.ones((1,) + rho.shape))
    lev = Level(eos, (dx, dx, dx), (0, 0, 0), (n - 1, n - 1, n - 1),
                (abi.BC_OUTFLOW, abi.BC_INTERIOR, abi.BC_INTERIOR),
                (abi.BC_OUTFLOW, abi.BC_INTERIOR, abi.BC_INTERIOR),
                np.ascontiguousarray(U), [((0, 0, 0), (n - 1, n - 1, n - 1))], (False, True, True))
    lev.fill_ghosts()
    return lev


# ------------------------------------------------------------------ H2/air flame (configs 2, 3, 5)
P_ATM = 1013250.0
Y_UNBURNT = {"H2": 0.0285, "O2": 0.2264, "N2": 0.7451}
Y_BURNT = {"H2O": 0.2548, "N2": 0.7452}
RADICAL_PEAKS = {"OH": 5e-3, "H": 5e-4, "O": 1e-3, "HO2": 1e-4}
FLAME_DELTA = 0.05  # cm
FLAME_DX = 0.005  # cm (50 um): 10 cells across the front


def _flame_prims(eos: Nasa7Mixture, Xc, Yc, Zc, zf, rng_vel, L):
    """Primitive fields of the flame generator at cell centres (Xc, Yc, Zc)."""
    xi = (Zc - zf) / FLAME_DELTA
    T = 300.0 + 950.0 * (1.0 + np.tanh(xi))
    c = 0.5 * (1.0 + np.tanh(xi))
    Y = np.zeros((eos.nspec,) + Zc.shape)
    for nm, v in Y_UNBURNT.items():
        Y[eos.index(nm)] += (1.0 - c) * v
    for nm, v in Y_BURNT.items():
        Y[eos.index(nm)] += c * v
    g = np.exp(-xi * xi)
    for nm, v in RADICAL_PEAKS.items():
        Y[eos.index(nm)] += v * g
    iN2 = eos.index("N2")
    Y[iN2] = 1.0 - (Y.sum(axis=0) - Y[iN2])
    p = np.full(Zc.shape, P_ATM)
    rho = p / (_rmix(eos, Y) * T)
    u = rng_vel.uniform(-100.0, 100.0, size=Zc.shape)
    v = rng_vel.uniform(-100.0, 100.0, size=Zc.shape)
    w = 1000.0 + rng_vel.uniform(-100.0, 100.0, size=Zc.shape)
    return rho, u, v, w, p, Y


def flame(n=128, box=32, seed=2, eos=None) -> Level:
    """The production flame level: periodic x/y, outflow z, edge n, boxes of edge box."""
    eos = eos or load_nasa7()
    N = n + 2 * NG
    L = n * FLAME_DX
    rng = np.random.default_rng(seed)
    phx, phy = rng.uniform(0, 2 * np.pi, size=2)
    c = (np.arange(N) - NG + 0.5) * FLAME_DX
    Zc, Yc, Xc = np.meshgrid(c, c, c, indexing="ij")
    zf = 0.5 * L + 0.02 * L * np.sin(2 * np.pi * Xc / L + phx) * np.cos(2 * np.pi * Yc / L + phy)
    rho, u, v, w, p, Y = _flame_prims(eos, Xc, Yc, Zc, zf, rng, L)
    U = conserved_from_prim(eos, rho, u, v, w, p, Y)
    lev = Level(eos, (FLAME_DX,) * 3, (0, 0, 0), (n - 1,) * 3,
                (abi.BC_INTERIOR, abi.BC_INTERIOR, abi.BC_OUTFLOW),
                (abi.BC_INTERIOR, abi.BC_INTERIOR, abi.BC_OUTFLOW),
                np.ascontiguousarray(U), tile_boxes((n, n, n), (box, box, box)), (True, True, False))
    lev.fill_ghosts()
    return lev


@dataclass
class Slab:
    """The z-slab [k0, k1] of a level decomposed over ranks: the level's global domain
    and boundary conditions, the state on grow(slab, NG) and the boxes tiling the slab."""

    eos: object
    dx: tuple
    domlo: tuple  # global domain
    domhi: tuple
    bclo: tuple
    bchi: tuple
    periodic: tuple
    k0: int
    k1: int
    state: np.ndarray  # (NVAR, k1-k0+1+2NG, NY+2NG, NX+2NG)
    boxes: list = field(default_factory=list)

    @property
    def nspec(self):
        return self.eos.nspec

    @property
    def lo(self):
        return (self.domlo[0] - NG, self.domlo[1] - NG, self.k0 - NG)

    def ncells(self):
        return sum(int(np.prod([h - l + 1 for l, h in zip(lo, hi)])) for lo, hi in self.boxes)


def slab_range(nz, nranks, rank, box):
    """k-range of rank's slab: equal slabs, each a whole number of boxes."""
    if nz % nranks or (nz // nranks) % box:
        raise ValueError(f"{nz} cells in z do not split into {nranks} slabs of whole {box}-boxes")
    nzl = nz // nranks
    return rank * nzl, (rank + 1) * nzl - 1


def split_level(lev: Level, nranks, rank, box) -> Slab:
    """Rank's slab of an existing level (ghost cells included, as the level holds them)."""
    nz = lev.domhi[2] - lev.domlo[2] + 1
    k0, k1 = slab_range(nz, nranks, rank, box)
    k0 += lev.domlo[2]
    k1 += lev.domlo[2]
    st = lev.state[:, k0 - lev.domlo[2]:k1 - lev.domlo[2] + 1 + 2 * NG]
    boxes = [b for b in lev.boxes if b[0][2] >= k0 and b[1][2] <= k1]
    return Slab(lev.eos, lev.dx, lev.domlo, lev.domhi, lev.bclo, lev.bchi, lev.periodic, k0, k1,
                np.ascontiguousarray(st), boxes)


def flame_slab(n=128, nz=256, nranks=2, rank=0, box=32, seed=2, eos=None) -> Slab:
    """Rank's slab of the flame level of edges (n, n, nz): periodic x/y, outflow z, the
    front wrinkled around z = nz*dx/2; the velocity noise is drawn per rank."""
    eos = eos or load_nasa7()
    k0, k1 = slab_range(nz, nranks, rank, box)
    L = n * FLAME_DX
    Lz = nz * FLAME_DX
    phx, phy = np.random.default_rng(seed).uniform(0, 2 * np.pi, size=2)
    rng = np.random.default_rng(seed * 7919 + rank)
    c = (np.arange(n + 2 * NG) - NG + 0.5) * FLAME_DX
    cz = (np.arange(k0 - NG, k1 + NG + 1) + 0.5) * FLAME_DX
    Zc, Yc, Xc = np.meshgrid(cz, c, c, indexing="ij")
    zf = 0.5 * Lz + 0.02 * L * np.sin(2 * np.pi * Xc / L + phx) * np.cos(2 * np.pi * Yc / L + phy)
    rho, u, v, w, p, Y = _flame_prims(eos, Xc, Yc, Zc, zf, rng, L)
    U = conserved_from_prim(eos, rho, u, v, w, p, Y)
    boxes = [((b[0][0], b[0][1], b[0][2] + k0), (b[1][0], b[1][1], b[1][2] + k0))
             for b in tile_boxes((n, n, k1 - k0 + 1), (box, box, box))]
    return Slab(eos, (FLAME_DX,) * 3, (0, 0, 0), (n - 1, n - 1, nz - 1),
                (abi.BC_INTERIOR, abi.BC_INTERIOR, abi.BC_OUTFLOW), (abi.BC_INTERIOR, abi.BC_INTERIOR, abi.BC_OUTFLOW),
                (True, True, False), k0, k1, np.ascontiguousarray(U), boxes)


@dataclass
class Patch:
    """An independent box: its own grown state FAB, no physical boundaries."""

    lo: tuple
    hi: tuple
    fab: abi.Fab  # conserved state on grow([lo,hi], NG)
    dx: tuple = (FLAME_DX,) * 3

    @property
    def ncells(self):
        return int(np.prod([h - l + 1 for l, h in zip(self.lo, self.hi)]))


def flame_patch(edges, seed, eos=None) -> Patch:
    """One independent flame box of the given edges with a random front offset."""
    eos = eos or load_nasa7()
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(e) for e in edges)
    lo = (0, 0, 0)
    hi = (nx - 1, ny - 1, nz - 1)
    xs = (np.arange(nx + 2 * NG) - NG + 0.5) * FLAME_DX
    ys = (np.arange(ny + 2 * NG) - NG + 0.5) * FLAME_DX
    zs = (np.arange(nz + 2 * NG) - NG + 0.5) * FLAME_DX
    Zc, Yc, Xc = np.meshgrid(zs, ys, xs, indexing="ij")
    Lz = nz * FLAME_DX
    off = rng.uniform(-0.5, 0.5) * Lz
    phx, phy = rng.uniform(0, 2 * np.pi, size=2)
    Lw = 32 * FLAME_DX
    zf = 0.5 * Lz + off + 0.02 * Lw * np.sin(2 * np.pi * Xc / Lw + phx) * np.cos(2 * np.pi * Yc / Lw + phy)
    rho, u, v, w, p, Y = _flame_prims(eos, Xc, Yc, Zc, zf, rng, Lz)
    U = conserved_from_prim(eos, rho, u, v, w, p, Y)
    return Patch(lo, hi, abi.Fab(np.ascontiguousarray(U), (-NG, -NG, -NG)))


def log_uniform_edges(nbox, seed, lo=8, hi=64):
    """Box edges drawn log-uniform in [lo, hi] per axis (anisotropic)."""
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=(nbox, 3)))).astype(int)


def _flame_patch_job(spec):
    edges, seed, eos = spec
    return flame_patch(edges, seed, eos)


def flame_patches(specs, eos=None, workers=None):
    """flame_patch for every (edges, seed) of ``specs``, in order. Many patches are
    generated in parallel by a pool of worker processes started with "spawn" (no CUDA
    state is inherited), each patch from its own seed, so the result is the same as the
    serial one."""
    eos = eos or load_nasa7()
    workers = min(16, os.cpu_count() or 1) if workers is None else int(workers)
    if workers <= 1 or len(specs) < 16:
        return [flame_patch(e, sd, eos) for e, sd in specs]
    import multiprocessing
    from concurrent.futures import ProcessPoolExecutor

    with ProcessPoolExecutor(max_workers=workers, mp_context=multiprocessing.get_context("spawn")) as ex:
        return list(ex.map(_flame_patch_job, [(tuple(int(x) for x in e), int(sd), eos) for e, sd in specs],
                           chunksize=max(1, len(specs) // (4 * workers))))


def flame_boxes(nbox=512, seed=3, eos=None, lo=8, hi=64):
    edges = log_uniform_edges(nbox, seed, lo, hi)
    return flame_patches([(e, seed * 100003 + b) for b, e in enumerate(edges)], eos)


def serving_patches(nruns=16, per_run=32, seed=5, eos=None, edges=(16, 24, 32, 48, 64)):
    """Requests of an ensemble of ``nruns`` runs: each run submits ``per_run`` flame
    boxes whose edges are drawn uniformly from ``edges`` per axis (run-seeded), each
    with its own front offset. Returned in submission order (runs interleaved) with
    the run of each."""
    rngs = [np.random.default_rng(seed * 1000 + r) for r in range(nruns)]
    specs, runs = [], []
    for k in range(per_run):
        for r in range(nruns):
            e = rngs[r].choice(np.asarray(edges), size=3)
            specs.append((e, seed * 100003 + r * 1009 + k))
            runs.append(r)
    return flame_patches(specs, eos), runs


# ------------------------------------------------------------------ turbulence (config 4)
def turbulence(n=256, box=64, seed=4, kmax=32, mach=0.3, gamma=1.4) -> Level:
    eos = GammaLaw(gamma=gamma)
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n, d=1.0 / n)
    # wavenumber components broadcast over (kz, ky, kx) instead of full meshgrid copies
    KZ, KY, KX = k[:, None, None], k[None, :, None], k[None, None, :]
    K = np.sqrt(KX * KX + KY * KY + KZ * KZ)
    shell = (K >= 0.5) & (K <= kmax + 0.5)
    amp = np.zeros_like(K)
    # E(k) ~ k^-5/3 spread over the shell area 4 pi k^2: |u_k| ~ k^(-11/6)
    amp[shell] = K[shell] ** (-11.0 / 6.0)
    uh = []
    for _ in range(3):
        ph = rng.uniform(0, 2 * np.pi, size=K.shape)
        # exp(i ph) as cos + i sin: the same values, several times faster than complex exp
        uh.append(amp * (np.cos(ph) + 1j * np.sin(ph)))
    Ksafe = np.where(K == 0, 1.0, K)
    kdotu = (KX * uh[0] + KY * uh[1] + KZ * uh[2]) / (Ksafe ** 2)
    uh = [uh[0] - KX * kdotu, uh[1] - KY * kdotu, uh[2] - KZ * kdotu]  # solenoidal projection
    vel = [np.real(np.fft.ifftn(c)) for c in uh]
    urms = np.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2) / 3.0)
    c0 = 1.0  # rho = 1, p = 1/gamma
    vel = [v * (mach * c0 / urms) for v in vel]
    rho = 1.0 * (1.0 + 0.01 * rng.standard_normal((n, n, n)))
    p = np.full((n, n, n), 1.0 / gamma)
    U = conserved_from_prim(eos, rho, vel[0], vel[1], vel[2], p, np.ones((1, n, n, n)))
    N = n + 2 * NG
    state = np.zeros((U.shape[0], N, N, N))
    state[:, NG:-NG, NG:-NG, NG:-NG] = U
    lev = Level(eos, (1.0 / n,) * 3, (0, 0, 0), (n - 1,) * 3, (abi.BC_INTERIOR,) * 3, (abi.BC_INTERIOR,) * 3,
                state, tile_boxes((n, n, n), (box, box, box)), (True, True, True))
    lev.fill_ghosts()
    return lev


# ------------------------------------------------------------------ generic random states (tests)
def _smooth_noise(rng, shape, passes=2):
    a = rng.standard_normal(shape)
    for _ in range(passes):
        for ax in range(3):
            a = 0.25 * np.roll(a, 1, axis=ax) + 0.5 * a + 0.25 * np.roll(a, -1, axis=ax)
    return a / (np.abs(a).max() + 1e-300)


def random_patch(edges, seed, eos=None, shock=True) -> Patch:
    """A box with smooth random primitive fields plus (optionally) a pressure jump, so
    every limiter, flattening and Riemann branch is exercised. Gamma law (nspec 1,
    O(1) units) or the NASA-7 mixture (nspec 9, CGS) depending on ``eos``."""
    eos = eos or GammaLaw()
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(e) for e in edges)
    shp = (nz + 2 * NG, ny + 2 * NG, nx + 2 * NG)
    jump = np.zeros(shp)
    if shock:
        X = np.arange(shp[2])[None, None, :] + 0.7 * np.arange(shp[1])[None, :, None] \
            + 0.3 * np.arange(shp[0])[:, None, None]
        jump = (X > 0.5 * X.max()).astype(float)
    if isinstance(eos, GammaLaw):
        rho = 1.0 + 0.3 * _smooth_noise(rng, shp) - 0.5 * jump
        p = 1.0 + 0.3 * _smooth_noise(rng, shp) - 0.7 * jump
        vel = [0.5 * _smooth_noise(rng, shp) for _ in range(3)]
        Y = np.ones((1,) + shp)
    else:
        T = 1200.0 + 600.0 * _smooth_noise(rng, shp) + 500.0 * jump
        Y = rng.uniform(0.2, 1.0, size=(eos.nspec,) + shp)
        Y = Y / Y.sum(axis=0, keepdims=True)
        p = P_ATM * (1.0 + 0.2 * _smooth_noise(rng, shp) - 0.4 * jump)
        rho = p / (_rmix(eos, Y) * T)
        vel = [2.0e4 * _smooth_noise(rng, shp) for _ in range(3)]
    U = conserved_from_prim(eos, rho, vel[0], vel[1], vel[2], p, Y)
    dx = (1.0 / 32,) * 3 if isinstance(eos, GammaLaw) else (FLAME_DX,) * 3
    return Patch((0, 0, 0), (nx - 1, ny - 1, nz - 1), abi.Fab(np.ascontiguousarray(U), (-NG, -NG, -NG)), dx)
