"""Failure paths of the CUDA path, driven from the host without faulting,
trapping or hanging the GPU.

  * a non-finite position pushed through dmdgpu_set_state -> DMDGPU_ERR_NAN;
  * a pair list that overflows its capacity -> DMDGPU_ERR_CAPACITY (the
    builders write nothing past the capacity);
  * a list-build grid barrier that can never complete: each bounded wait gives
    up (20 ms here), the kernel returns, the call reports DMDGPU_ERR_GPU, later
    calls on that context refuse to issue work, and the GPU context stays
    usable for a new engine;
  * checkpoints with a wrong magic word, an unknown version, or truncated data
    are refused with DMDGPU_ERR_MISMATCH (the reference reads them blindly,
    src/sim/checkpoint.cpp:40-47).
"""
import struct

import numpy as np
import pytest

from dmd_b200 import workloads as W

pytestmark = pytest.mark.gpu

ERR_NAN, ERR_MISMATCH, ERR_GPU, ERR_CAPACITY = 1, 3, 5, 9


def _engine(cfg, precision="mixed", profile="phys"):
    from dmd_b200.core import Engine
    return Engine(cfg, precision=precision, profile=profile)


def _water(n_mol=200, seed=4):
    box = (n_mol / 33.43) ** (1 / 3)
    return W.water_box(n_mol=n_mol, box=box, seed=seed, spacing=box / round(box / 0.1045)).config()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_nan_position_reported(precision):
    from dmd_b200.core import DmdGpuError
    eng = _engine(_water(), precision)
    eng.run_n(3)
    pos = eng.positions
    pos[17, 1] = np.nan
    eng.set_positions(pos)
    with pytest.raises(DmdGpuError) as ei:
        eng.run_n(1)
    assert ei.value.code == ERR_NAN, str(ei.value)


def test_list_capacity_overflow_reported():
    from dmd_b200.core import DmdGpuError
    eng = _engine(_water())
    eng.run_n(2)
    eng.test_inject("list_capacity")
    with pytest.raises(DmdGpuError) as ei:
        eng.run_n(1)
    assert ei.value.code == ERR_CAPACITY, str(ei.value)
    assert np.all(np.isfinite(eng.positions))


def test_barrier_timeout_reported_and_context_usable():
    from dmd_b200.core import DmdGpuError
    cfg = _water()
    eng = _engine(cfg)
    eng.run_n(2)
    eng.test_inject("barrier_timeout")
    with pytest.raises(DmdGpuError) as ei:
        eng.run_n(1)
    assert ei.value.code == ERR_GPU and "timed out" in str(ei.value)
    # the table is refused from now on, without issuing work
    with pytest.raises(DmdGpuError) as ei2:
        eng.run_n(1)
    assert ei2.value.code == ERR_GPU
    assert np.all(np.isfinite(eng.positions))  # state can still be read
    eng.close()
    # the GPU context is intact: a new engine runs and matches a clean run
    a, b = _engine(cfg), _engine(cfg)
    a.run_n(5)
    b.run_n(5)
    assert np.array_equal(a.positions, b.positions)


def test_corrupt_checkpoints_refused(tmp_path):
    from dmd_b200.core import DmdGpuError
    cfg = W.argon_fcc(n_cells=3, a=0.575, T=90.0, seed=2).config()
    eng = _engine(cfg, "fp64", "ref")
    eng.run_n(4)
    good = tmp_path / "good.bin"
    eng.save_checkpoint(str(good))
    raw = good.read_bytes()
    cases = {
        "magic": struct.pack("<I", 0xDEADBEEF) + raw[4:],
        "version": raw[:4] + struct.pack("<I", 7) + raw[8:],
        "truncated": raw[: len(raw) // 2],
    }
    for name, blob in cases.items():
        p = tmp_path / f"{name}.bin"
        p.write_bytes(blob)
        fresh = _engine(cfg, "fp64", "ref")
        with pytest.raises(DmdGpuError) as ei:
            fresh.load_checkpoint(str(p))
        assert ei.value.code == ERR_MISMATCH, (name, str(ei.value))
    fresh = _engine(cfg, "fp64", "ref")
    fresh.load_checkpoint(str(good))
    assert fresh.current_step == 4
