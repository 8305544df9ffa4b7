"""GPU test of the z-slab decomposition: a level cut into slabs (held by one process,
exchanged by device copies) advances exactly like the undecomposed level in the plain
FP64 form, for the flame (outflow z) and periodic turbulence; graph replay of the slab
phases equals their eager run."""
import numpy as np
import pytest

from particleclem_b200 import abi, workloads as wl
from particleclem_b200.level import LevelStepper
from particleclem_b200.slab import LocalComm, SlabStepper, step

pytestmark = pytest.mark.gpu
NG = abi.NGROW


def _global_valid(st):
    return st.host_state()[:, NG:-NG, NG:-NG, NG:-NG]


def _slabs_valid(slabs):
    return np.concatenate([s.state.data.cpu().numpy()[:, NG:-NG, NG:-NG, NG:-NG] for s in slabs], axis=1)


@pytest.mark.parametrize("name,nranks", [("flame", 2), ("turbulence", 2), ("turbulence", 4)])
def test_slabs_equal_whole_level_fp64(name, nranks):
    lev = wl.flame(n=16, box=8) if name == "flame" else wl.turbulence(n=32, box=8, kmax=4)
    ref = LevelStepper(lev, precision=abi.PREC_FP64, fuse=False)
    slabs = [SlabStepper(wl.split_level(lev, nranks, r, 8), nranks, r, precision=abi.PREC_FP64, fuse=False)
             for r in range(nranks)]
    comm = LocalComm()
    for _ in range(3):
        ref.step()
        step(slabs, comm)
        assert all(float(s.dt.item()) == float(ref.dt.item()) for s in slabs)
    np.testing.assert_array_equal(_slabs_valid(slabs), _global_valid(ref))
    ref.close()
    for s in slabs:
        s.close()


def test_slab_graphs_equal_eager_mixed():
    lev = wl.flame(n=16, box=8)
    a = [SlabStepper(wl.split_level(lev, 2, r, 8), 2, r, precision=abi.PREC_MIXED) for r in range(2)]
    b = [SlabStepper(wl.split_level(lev, 2, r, 8), 2, r, precision=abi.PREC_MIXED) for r in range(2)]
    comm = LocalComm()
    for s in a:
        s.capture()  # leaves the slab's state as it was
    for _ in range(2):
        step(a, comm)
        step(b, comm)
    np.testing.assert_array_equal(_slabs_valid(a), _slabs_valid(b))
    for s in a + b:
        s.close()


@pytest.mark.parametrize("captured", [False, True])
def test_slab_fused_tail_equals_separate_passes_fp64(captured):
    """The fused step tail (the update pass forms each slab's CFL minimum, reduced over
    the slabs before the next step) against the separate CFL, hydro and update passes,
    bit for bit in the plain FP64 form; then a state loaded mid-run restarts from a fresh
    CFL reduction in both."""
    lev = wl.flame(n=16, box=8)
    a = [SlabStepper(wl.split_level(lev, 2, r, 8), 2, r, precision=abi.PREC_FP64) for r in range(2)]
    b = [SlabStepper(wl.split_level(lev, 2, r, 8), 2, r, precision=abi.PREC_FP64, fused_tail=False)
         for r in range(2)]
    if captured:
        for s in a:
            s.capture()
    comm = LocalComm()
    for _ in range(3):
        step(a, comm)
        step(b, comm)
        assert float(a[0].dt.item()) == float(b[0].dt.item())
    np.testing.assert_array_equal(_slabs_valid(a), _slabs_valid(b))
    fresh = [s.state.data.clone() for s in b]
    for s, f in zip(a, fresh):
        s.load_state(f)
    for _ in range(2):
        step(a, comm)
        step(b, comm)
        assert float(a[0].dt.item()) == float(b[0].dt.item())
    np.testing.assert_array_equal(_slabs_valid(a), _slabs_valid(b))
    for s in a + b:
        s.close()


@pytest.mark.parametrize("name", ["flame", "turbulence"])
def test_overlapped_slab_steps_equal_plain_fp64(name):
    """The overlapped form (interior advanced while the halo is exchanged, then the bands
    next to exchanging faces) equals the plain slab step bit for bit in the FP64 form; the
    halo planes are packed and unpacked by the library's copy kernel."""
    from particleclem_b200.slab import step_overlap

    lev = wl.flame(n=16, box=8) if name == "flame" else wl.turbulence(n=32, box=8, kmax=4)
    mk = lambda ov: [SlabStepper(wl.split_level(lev, 2, r, 8), 2, r, precision=abi.PREC_FP64, fuse=True,  # noqa
                                 overlap=ov) for r in range(2)]
    plain, over = mk(False), mk(True)
    assert all(s.overlap for s in over)
    comm = LocalComm()
    for _ in range(3):
        step(plain, comm)
        step_overlap(over, comm)
        assert all(float(a.dt.item()) == float(b.dt.item()) for a, b in zip(plain, over))
    np.testing.assert_array_equal(_slabs_valid(over), _slabs_valid(plain))
    for s in plain + over:
        s.close()
