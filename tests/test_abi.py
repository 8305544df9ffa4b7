"""The C-ABI library: it loads and exports every function include/pcg_hydro.h
declares, and rejects bad arguments with PCG_E* codes before touching a device."""
import ctypes as C

import pytest

from particleclem_b200 import abi, native


def test_header_declares_the_operator_surface():
    fns = native.header_functions()
    for f in ("pcg_ctoprim", "pcg_umdrv", "pcg_hydro_box", "pcg_hydro_boxes", "pcg_estdt", "pcg_update_state",
              "pcg_fill_ghosts", "pcg_plan_create", "pcg_last_error"):
        assert f in fns


def test_library_exports_every_declared_function():
    lib = native.load()
    missing = [f for f in native.header_functions() if not hasattr(lib, f)]
    assert not missing, missing
    assert set(native.header_functions()) <= set(native.SIGNATURES), "python binding lags the header"


def _rc(name, *args):
    lib = native.load()
    return getattr(lib, name)(*args)


def test_argument_errors_are_codes_not_aborts():
    assert _rc("pcg_hydro_box", None, None, None, None, None, None, None) == -1  # PCG_EINVAL
    assert "params" in native.load().pcg_last_error().decode()
    assert _rc("pcg_set_eos_gamma", 0.5, 28.97) == -1
    prm = abi.make_params((1, 1, 1), 0.1, 1, (0, 0, 0), (7, 7, 7), (0, 0, 0), (0, 0, 0), ppm_type=3)
    assert _rc("pcg_hydro_box", C.byref(prm), abi.ivec((0, 0, 0)), abi.ivec((7, 7, 7)), None, None, None, None) == -1
    assert "ppm_type" in native.load().pcg_last_error().decode()
    prm = abi.make_params((1, 1, 1), 0.1, 1, (0, 0, 0), (7, 7, 7), (0, 0, 0), (0, 0, 0), ppm_type=0)
    prm.use_hybrid_weno = 1  # WENO edge values exist for the PPM trace only (Source/PeleC.cpp:384-386)
    assert _rc("pcg_hydro_box", C.byref(prm), abi.ivec((0, 0, 0)), abi.ivec((7, 7, 7)), None, None, None, None) == -1
    prm = abi.make_params((1, 1, 1), 0.1, 5, (0, 0, 0), (7, 7, 7), (0, 0, 0), (0, 0, 0))
    assert _rc("pcg_hydro_box", C.byref(prm), abi.ivec((0, 0, 0)), abi.ivec((7, 7, 7)), None, None, None, None) == -4
    assert _rc("pcg_plan_destroy", None) == 0


@pytest.mark.parametrize("bc", [-1, 7])
def test_unknown_boundary_types_are_rejected(bc):
    """Boundary codes outside PeleC's PCPhysBCType (Source/PeleC.H:49-57) fail with
    PCG_EINVAL before any device work; inflow and user_bc are accepted (low-order faces)."""
    import numpy as np

    prm = abi.make_params((1, 1, 1), 0.1, 1, (0, 0, 0), (7, 7, 7), (bc, 0, 0), (0, 0, 0))
    u = abi.Fab(np.zeros((8, 16, 16, 16)), (-4, -4, -4))
    o = abi.Fab(np.zeros((8, 8, 8, 8)), (0, 0, 0))
    rc = _rc("pcg_hydro_box", C.byref(prm), abi.ivec((0, 0, 0)), abi.ivec((7, 7, 7)), C.byref(abi.array4(u)),
             C.byref(abi.array4(o)), None, None)
    assert rc == -1


def test_copy_cells_argument_errors():
    """pcg_copy_cells rejects, before any device work, arrays that do not cover the box,
    differing component counts and an empty box (PCG_EINVAL)."""
    import numpy as np

    a = abi.Fab(np.zeros((3, 6, 6, 6)), (0, 0, 0))
    b = abi.Fab(np.zeros((2, 6, 6, 6)), (0, 0, 0))
    c = abi.Fab(np.zeros((3, 4, 4, 4)), (1, 1, 1))

    def rc(src, dst, lo, hi):
        return _rc("pcg_copy_cells", C.byref(abi.array4(src)), C.byref(abi.array4(dst)), abi.ivec(lo), abi.ivec(hi),
                   None)

    assert rc(a, b, (0, 0, 0), (5, 5, 5)) == -1
    assert "component counts" in native.load().pcg_last_error().decode()
    assert rc(a, c, (0, 0, 0), (3, 3, 3)) == -1
    assert "dst must cover" in native.load().pcg_last_error().decode()
    assert rc(a, a, (2, 2, 2), (1, 5, 5)) == -1


def test_workspace_pool_argument_errors():
    """pcg_reserve_workspace and pcg_trim_workspace reject bad devices and sizes with
    PCG_EINVAL before any device work; reserving nothing is a no-op."""
    assert _rc("pcg_reserve_workspace", -1, 0) == -1
    assert _rc("pcg_reserve_workspace", 0, -5) == -1
    assert _rc("pcg_reserve_workspace", 0, 0) == 0
    assert _rc("pcg_trim_workspace", -1, 0) == -1
    assert _rc("pcg_trim_workspace", 0, -1) == -1


def test_tiled_trace_variants_only_for_the_mixed_trace():
    """Launch variants 3-5 (the TMA-staged tiled trace) exist for the mixed form's trace
    only; every other (form, stage) takes 0-2."""
    from particleclem_b200 import autotune

    saved = autotune.get_variant(abi.PREC_MIXED, 9, autotune.TRACE_STAGE)
    try:
        assert _rc("pcg_set_launch_variant", abi.PREC_MIXED, 9, autotune.TRACE_STAGE, 5) == 0
        assert autotune.get_variant(abi.PREC_MIXED, 9, autotune.TRACE_STAGE) == 5
        assert _rc("pcg_set_launch_variant", abi.PREC_MIXED, 9, autotune.TRACE_STAGE, 6) == -1
        assert _rc("pcg_set_launch_variant", abi.PREC_FP64, 9, autotune.TRACE_STAGE, 3) == -1
        assert _rc("pcg_set_launch_variant", abi.PREC_MIXED, 9, 3, 3) == -1  # flux0
    finally:
        autotune.set_variant(abi.PREC_MIXED, 9, autotune.TRACE_STAGE, saved)
    assert autotune.describe(abi.PREC_MIXED, autotune.TRACE_STAGE, 4).startswith("TMA-staged tiles")


def test_species_counts_of_the_build():
    """pcg_species_counts lists the species counts the library was compiled for (the
    build's PCG_NSPEC list); a mixture table or a call for any other count is refused with
    PCG_EUNSUPPORTED before any device work, and a one-species NASA-7 table with
    PCG_EINVAL (one species is the gamma law)."""
    import numpy as np

    from particleclem_b200 import build, hydro

    counts = hydro.species_counts()
    assert counts == build.species_counts()
    assert 1 in counts and 9 in counts
    missing = next(n for n in range(2, 64) if n not in counts)
    tab = [np.ones(7 * missing) for _ in range(4)]
    ptrs = [t.ctypes.data_as(C.POINTER(C.c_double)) for t in tab]
    assert _rc("pcg_set_eos_nasa7", missing, *ptrs) == -4
    assert str(missing) in native.load().pcg_last_error().decode()
    assert _rc("pcg_set_eos_nasa7", 1, *ptrs) == -1
    prm = abi.make_params((1, 1, 1), 0.1, missing, (0, 0, 0), (7, 7, 7), (0, 0, 0), (0, 0, 0))
    assert _rc("pcg_hydro_box", C.byref(prm), abi.ivec((0, 0, 0)), abi.ivec((7, 7, 7)), None, None, None, None) == -4


def test_species_build_options(monkeypatch):
    """PCG_NSPEC parsing of the build: sorted unique counts, the EOS bank sized to the
    largest (even, at least 16), one strict/fast/mixed unit per count plus the host units;
    bad lists are refused."""
    from particleclem_b200 import build

    monkeypatch.setenv("PCG_NSPEC", "9, 1,53,9")
    assert build.species_counts() == (1, 9, 53)
    assert build.max_species((1, 9, 53)) == 54
    assert build.max_species((1, 2, 9)) == 16
    tags = [u[0] for u in build.units((1, 9, 53))]
    assert tags[:3] == ["strict_ns53", "fast_ns53", "mixed_ns53"]  # largest units start first
    assert sorted(tags) == sorted([f"{k}_ns{n}" for n in (1, 9, 53) for k in ("strict", "fast", "mixed")]
                                  + ["host", "fluxreg"])
    assert all("-DPCG_MAXNS=54" in u[2] for u in build.units((1, 9, 53)) if u[0] != "fluxreg")
    monkeypatch.setenv("PCG_NSPEC", "0,9")
    with pytest.raises(ValueError):
        build.species_counts()
    monkeypatch.delenv("PCG_NSPEC")
    assert build.species_counts() == build.DEFAULT_NSPEC
