"""Generate the stand-in NASA-7 thermo table for the 9-species H2/O2/N2 mixture.

The hydro path evaluates the mixture EOS through NASA-7 polynomials (two temperature
ranges split at T_mid = 1000 K), exactly like a Fuego-generated mechanism would. The
coefficient table of the real hydrogen mechanism is not available here, so this script
builds a clearly labelled STAND-IN table from a simple, documented physical model:

  cp/R(T) = 5/2 (translation) + rot (1 linear, 3/2 nonlinear, 0 atoms)
            + sum over vibrational modes of the Einstein function E(theta_i / T),
  E(x) = x^2 e^x / (e^x - 1)^2,

with rounded characteristic vibrational temperatures theta_i chosen per molecule
(listed below). Each range is least-squares fitted by the quartic cp/R = a0 + a1 T +
a2 T^2 + a3 T^3 + a4 T^4 on [300, 1000] K and [1000, 3500] K. The enthalpy constant a5
is set so that h(298.15 K) equals the species' standard enthalpy of formation (public
thermochemical values, rounded), with the high-range a5 matched for continuity of h at
T_mid. a6 (entropy) is not used by the hydro path and is written as 0.

Molecular weights use the standard atomic weights H = 1.008, O = 15.999, N = 14.007.

The output file has one header line and then, per species, one line
  name  W  Tlow  Tmid  Thigh
followed by the seven low-range and the seven high-range coefficients. Any table in the
same format (for example the real mechanism's) can be dropped in instead.

Usage: python make_standin_thermo.py [out_path]
"""
import sys
import numpy as np

# name, atoms (H, O, N), linear?, vibrational temperatures [K], h_f(298.15) [kJ/mol]
SPECIES = [
    ("H2", (2, 0, 0), True, [6330.0], 0.0),
    ("O2", (0, 2, 0), True, [2270.0], 0.0),
    ("H2O", (2, 1, 0), False, [5260.0, 2290.0, 5400.0], -241.83),
    ("H", (1, 0, 0), None, [], 218.0),
    ("O", (0, 1, 0), None, [], 249.18),
    ("OH", (1, 1, 0), True, [5380.0], 37.3),
    ("HO2", (1, 2, 0), False, [5100.0, 2000.0, 1580.0], 12.0),
    ("H2O2", (2, 2, 0), False, [5400.0, 2000.0, 1270.0, 500.0, 5400.0, 1830.0], -135.9),
    ("N2", (0, 0, 2), True, [3390.0], 0.0),
]
ATOMIC_W = (1.008, 15.999, 14.007)
R_KJ = 8.31446261815324e-3  # kJ/(mol K)
T_LOW, T_MID, T_HIGH = 300.0, 1000.0, 3500.0


def cp_over_r(T, linear, thetas):
    cp = np.full_like(T, 2.5)
    if linear is None:
        return cp
    cp += 1.0 if linear else 1.5
    for th in thetas:
        x = th / T
        ex = np.exp(x)
        cp += x * x * ex / (ex - 1.0) ** 2
    return cp


def fit_range(t0, t1, linear, thetas):
    # Fit in x = T / 1000 (well conditioned), then rescale to powers of T.
    T = np.linspace(t0, t1, 400)
    A = np.vander(T / 1000.0, 5, increasing=True)
    coef, *_ = np.linalg.lstsq(A, cp_over_r(T, linear, thetas), rcond=None)
    return coef / 1000.0 ** np.arange(5)


def h_over_r_poly(a, T):
    """h/R minus the constant a5: a0 T + a1 T^2/2 + a2 T^3/3 + a3 T^4/4 + a4 T^5/5."""
    return sum(a[i] * T ** (i + 1) / (i + 1) for i in range(5))


def build():
    rows = []
    for name, atoms, linear, thetas, hf in SPECIES:
        w = sum(n * aw for n, aw in zip(atoms, ATOMIC_W))
        lo = fit_range(T_LOW, T_MID, linear, thetas)
        hi = fit_range(T_MID, T_HIGH, linear, thetas)
        a5_lo = hf / R_KJ - h_over_r_poly(lo, 298.15)
        a5_hi = a5_lo + h_over_r_poly(lo, T_MID) - h_over_r_poly(hi, T_MID)
        rows.append((name, w, list(lo) + [a5_lo, 0.0], list(hi) + [a5_hi, 0.0]))
    return rows


def write(path):
    rows = build()
    with open(path, "w") as f:
        f.write("# STAND-IN NASA-7 table (not the real mechanism): made by make_standin_thermo.py\n")
        for name, w, lo, hi in rows:
            f.write(f"{name} {w!r} {T_LOW!r} {T_MID!r} {T_HIGH!r}\n")
            f.write(" ".join(repr(float(v)) for v in lo) + "\n")
            f.write(" ".join(repr(float(v)) for v in hi) + "\n")


if __name__ == "__main__":
    write(sys.argv[1] if len(sys.argv) > 1 else "h2air_standin_nasa7.dat")
