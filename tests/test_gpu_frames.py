"""Trajectory frames exported while the run continues (dmdgpu_set_frame_writer):
the frame writing of the reference's run loop (EngineWrapper::run_n,
python/dmd/core.cpp:29-44; H5MDWriter::write_frame,
src/trajectory/h5md_writer.cpp:191) with a stub writer in place of HDF5.

Each frame must hold exactly the state a plain run reaches at that step
(positions, velocities with the pending thermostat scale, box, time), frames
must arrive once each in step order across calls, and exporting must change no
bit of the trajectory.
"""
import threading

import numpy as np
import pytest

from dmd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _water(n_mol=300, seed=5):
    box = (n_mol / 33.43) ** (1 / 3)
    c = W.water_box(n_mol=n_mol, box=box, seed=seed, spacing=box / round(box / 0.1045)).config()
    c.thermostat.type = "nose-hoover"
    c.barostat.type = "berendsen"  # the box moves, so the frame's box is checked too
    c.barostat.tau = 0.5
    return c


class StubWriter:
    """Stands in for H5MDWriter: keeps a copy of every frame it is handed."""

    def __init__(self):
        self.frames = []
        self.threads = set()

    def __call__(self, frame):
        self.threads.add(threading.get_ident())
        self.frames.append(frame)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_frames_match_plain_run(precision):
    from dmd_b200.core import Engine
    cfg = _water()
    w = StubWriter()
    eng = Engine(cfg, precision=precision, profile="phys")
    eng.set_frame_writer(5, w)
    for n in (3, 9, 11):  # 23 steps in calls that do not line up with the interval
        eng.run_n(n)
    eng.flush_frames()
    assert [f["step"] for f in w.frames] == [5, 10, 15, 20]
    plain = Engine(cfg, precision=precision, profile="phys")
    for f in w.frames:
        plain.run_n(f["step"] - plain.current_step)
        s = plain.scalars()
        assert np.array_equal(f["positions"], plain.positions), f["step"]
        assert np.array_equal(f["velocities"], plain.velocities), f["step"]
        assert f["box"] == s.box and f["time"] == s.time, f["step"]
    plain.run_n(23 - plain.current_step)
    # exporting frames changed nothing
    assert np.array_equal(eng.positions, plain.positions)
    assert np.array_equal(eng.velocities, plain.velocities)
    assert eng.potential_energy == plain.potential_energy


def test_frames_off_and_many_in_flight():
    """Interval 1 over more steps than staging slots (the run waits for the
    writer only when it falls that far behind); then export turned off."""
    from dmd_b200.core import Engine
    cfg = _water(n_mol=200, seed=8)
    w = StubWriter()
    eng = Engine(cfg, precision="mixed", profile="phys")
    eng.set_frame_writer(1, w)
    eng.run_n(17)
    eng.flush_frames()
    assert [f["step"] for f in w.frames] == list(range(1, 18))
    eng.set_frame_writer(0)
    eng.run_n(4)
    eng.flush_frames()
    assert len(w.frames) == 17
    assert all(np.all(np.isfinite(f["positions"])) for f in w.frames)
