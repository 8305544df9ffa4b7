"""Shared helpers of the test suite: oracle access, host<->device FAB copies, and the
parity metrics of the hot path (per-component relative L1 / Linf)."""
import numpy as np

import pyoracle
from particleclem_b200 import abi, thermo, workloads as wl

FP64_TOL = 1e-12  # plain FP64 forms vs the FP64 oracle (rel L1 and Linf per component)
MIXED_TOL = 1e-6  # mixed form vs the FP64 oracle (rel L1 per component of S_new)

_ORACLE = None
_EOS9 = None


def oracle():
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = pyoracle.oracle()
    return _ORACLE


def eos9():
    global _EOS9
    if _EOS9 is None:
        _EOS9 = thermo.load_nasa7()
    return _EOS9


def to_gpu(fab):
    import torch

    return abi.Fab(torch.from_numpy(np.ascontiguousarray(fab.data)).cuda(), tuple(fab.lo))


def gpu_zeros(ncomp, lo, hi):
    import torch

    shp = (ncomp,) + tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
    return abi.Fab(torch.zeros(shp, dtype=torch.float64, device="cuda"), tuple(lo))


def np_zeros(ncomp, lo, hi):
    shp = (ncomp,) + tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0))
    return abi.Fab(np.zeros(shp), tuple(lo))


def to_cpu(fab):
    import torch

    torch.cuda.synchronize()
    return fab.data.cpu().numpy()


def params_for(patch_or_level, dt, ppm_type=1, plm_iorder=4, prec=abi.PREC_FP64, nspec=None):
    if isinstance(patch_or_level, wl.Level):
        L = patch_or_level
        return abi.make_params(L.dx, dt, L.nspec, L.domlo, L.domhi, L.bclo, L.bchi, ppm_type=ppm_type,
                               plm_iorder=plm_iorder, precision_mode=prec)
    big = 1 << 30
    return abi.make_params(patch_or_level.dx, dt, nspec, (-big,) * 3, (big,) * 3, (0, 0, 0), (0, 0, 0),
                           ppm_type=ppm_type, plm_iorder=plm_iorder, precision_mode=prec)


def group_scales(ref, nspec):
    """Per-component normalisers: sum|r| and max|r| of the component's physical group
    (mass: rho and the species densities; momentum: the three components as a vector;
    energy: rho E and rho e; temperature alone). Near-zero components of a vector (for
    example the transverse momentum source of a planar Sod problem) are measured against
    the group's scale instead of inflating round-off into large relative errors."""
    nv = ref.shape[0]
    r = np.abs(ref.reshape(nv, -1))
    s1, sinf = r.sum(axis=1), r.max(axis=1)
    groups = [[abi.URHO] + list(range(abi.UFS, abi.UFS + nspec)), [abi.UMX, abi.UMY, abi.UMZ],
              [abi.UEDEN, abi.UEINT], [abi.UTEMP]]
    g1, ginf = np.ones(nv), np.ones(nv)
    for g in groups:
        g = [c for c in g if c < nv]
        a, b = s1[g].max(), sinf[g].max()
        g1[g] = a if a > 0 else 1.0
        ginf[g] = b if b > 0 else 1.0
    return g1, ginf


def rel_errors(got, ref, nspec=None):
    """Per-component relative L1 and Linf of conserved-variable arrays (components on
    axis 0), normalised by the component's group scale (see group_scales)."""
    nv = ref.shape[0]
    nspec = nv - 7 if nspec is None else nspec
    d = np.abs(got.reshape(nv, -1) - ref.reshape(nv, -1))
    g1, ginf = group_scales(ref, nspec)
    return d.sum(axis=1) / g1, d.max(axis=1) / ginf


def rel_err(got, ref):
    """(max over components of rel L1, max over components of rel Linf)."""
    l1, linf = rel_errors(got, ref)
    return float(l1.max()), float(linf.max())


def random_sources(fab, seed, scale=2.0):
    """A source FAB for the state ``fab`` (NVAR components on the same cells): each
    component a smooth random field of amplitude ``scale`` times the component's typical
    magnitude per unit time, so that hdt * srcQ perturbs the traced states by a fraction
    of a percent at CFL-limited timesteps. The role of PeleC's sources_for_hydro
    (Source/Hydro.cpp:29-46) in a run with reactions or diffusion."""
    rng = np.random.default_rng(seed)
    u = fab.data
    out = np.empty_like(u)
    for n in range(u.shape[0]):
        mag = np.abs(u[n]).mean() + 1e-30
        out[n] = scale * mag * wl._smooth_noise(rng, u.shape[1:])
    return abi.Fab(out, tuple(fab.lo))
