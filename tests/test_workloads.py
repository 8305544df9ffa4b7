"""Synthetic workload generators: shapes, admissible states and ghost filling."""
import numpy as np

from particleclem_b200 import abi, workloads as wl


def test_flame_level_shapes_and_mass_fractions():
    lev = wl.flame(n=16, box=8)
    assert lev.state.shape == (16, 24, 24, 24)
    assert len(lev.boxes) == 8 and lev.ncells() == 16 ** 3
    rho = lev.state[abi.URHO]
    Y = lev.state[abi.UFS:] / rho
    assert (rho > 0).all() and (Y >= 0).all()
    np.testing.assert_allclose(Y.sum(axis=0), 1.0, rtol=1e-12)
    T = lev.state[abi.UTEMP]
    assert 299.0 < T.min() and T.max() < 2201.0


def test_periodic_ghosts_wrap():
    lev = wl.turbulence(n=8, box=8, seed=1, kmax=2)
    s = lev.state
    g = abi.NGROW
    np.testing.assert_array_equal(s[:, :, :, :g], s[:, :, :, 8:8 + g])
    np.testing.assert_array_equal(s[:, :g], s[:, 8:8 + g])


def test_log_uniform_box_edges_in_range():
    e = wl.log_uniform_edges(512, 3)
    assert e.shape == (512, 3) and e.min() >= 8 and e.max() <= 64


def test_turbulence_velocity_is_solenoidal_and_scaled():
    lev = wl.turbulence(n=16, box=16, seed=4, kmax=4)
    g = abi.NGROW
    u = lev.state[abi.UMX:abi.UMZ + 1, g:-g, g:-g, g:-g] / lev.state[abi.URHO, g:-g, g:-g, g:-g]
    urms = np.sqrt((u ** 2).mean(axis=(1, 2, 3)).mean())
    assert 0.2 < urms < 0.45
