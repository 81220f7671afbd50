"""Batched replicas and continuous serving (C ABI batch API via dmd_b200.batch).

A slot's result must be the same alone and in the mix.  The batch shares kernel
launches, not arithmetic (fixed-point force sums, per-replica reductions in a
fixed order), so results are compared bit for bit.  Admitting or releasing a
job rebuilds the device table: every running replica carries its state over,
its pair list is rebuilt in the frame of its last build (same slots, tile
centres and chunks) and its forces are evaluated again at the same positions,
so a job is bit for bit the same as the same job run alone without any
rebuilds.
"""
import numpy as np
import pytest

from dmd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _mix():
    """Uneven LJ fluids, decane melts and four water boxes with different PME
    meshes (K = 20, 24, 23, 21: odd K^3 mesh sizes next to each other)."""
    cfgs = [W.lj_fluid(600, 0.65, 1.2, 11).config(), W.lj_fluid(1500, 0.80, 0.9, 12).config(),
            W.lj_fluid(2600, 0.72, 1.4, 13).config(), W.decane_melt(12, 14).config(),
            W.decane_melt(20, 15).config()]
    for n_mol, seed in ((300, 16), (500, 17), (450, 18), (360, 19)):
        box = (n_mol / 33.43) ** (1 / 3)
        cfgs.append(W.water_box(n_mol=n_mol, box=box, seed=seed,
                                spacing=box / round(box / 0.1045)).config())
    return cfgs


def _alone(cfg, steps, precision):
    from dmd_b200.core import Engine
    e = Engine(cfg, precision=precision, profile="phys")
    e.run_n(steps)
    return e.positions, e.velocities, e.potential_energy


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_matches_alone(precision):
    from dmd_b200.batch import Batch
    cfgs = _mix()
    steps = 30
    b = Batch(precision=precision, profile="phys")
    slots = [b.admit(c, steps) for c in cfgs]
    b.step(steps)
    assert sorted(b.poll()) == sorted(slots)
    for s, c in zip(slots, cfgs):
        p, v, pe = _alone(c, steps, precision)
        assert np.array_equal(b.positions(s), p), (s, "positions")
        assert np.array_equal(b.velocities(s), v), (s, "velocities")
        assert b.scalars(s).potential_energy == pe
        assert b.scalars(s).step == steps


def test_serving_admit_and_release_midway():
    """Continuous batching: B arrives while A runs, C after A is released; every
    result equals the same job run alone."""
    from dmd_b200.batch import Batch
    cfgs = _mix()
    a_cfg, b_cfg, c_cfg = cfgs[1], cfgs[5], cfgs[3]
    b = Batch(precision="mixed", profile="phys")
    a = b.admit(a_cfg, 25)
    b.step(10)
    s_b = b.admit(b_cfg, 20)          # repack while A is mid-run (A at step 10)
    b.step(15)                        # A done at 25, B at 15
    assert b.poll() == [a]
    pa, va, pe_a = b.positions(a), b.velocities(a), b.scalars(a).potential_energy
    b.release(a)
    s_c = b.admit(c_cfg, 12)          # C takes the freed slot id and memory (B at step 15)
    assert s_c == a
    b.step(12)                        # B done at 20 (stops there), C at 12
    assert sorted(b.poll()) == sorted([s_b, s_c])
    # B (Nose-Hoover water) reaches its target while C keeps stepping: its last
    # pending thermostat scale must survive the steps it sits out
    for cfg, n, got, vel, pe in (
            (a_cfg, 25, pa, va, pe_a),
            (b_cfg, 20, b.positions(s_b), b.velocities(s_b), b.scalars(s_b).potential_energy),
            (c_cfg, 12, b.positions(s_c), b.velocities(s_c), b.scalars(s_c).potential_energy)):
        p, v, pe_alone = _alone(cfg, n, "mixed")
        assert got.shape == p.shape
        assert np.array_equal(got, p), (n, np.abs(got - p).max())
        assert np.array_equal(vel, v), (n, np.abs(vel - v).max())
        assert pe == pe_alone
    assert b.active == 0


def test_budget_admission():
    from dmd_b200.batch import Batch, BudgetExceeded
    cfgs = _mix()
    need = Batch.footprint(cfgs[2], precision="mixed", profile="phys")
    b = Batch(budget_bytes=int(need * 1.5), precision="mixed", profile="phys")
    b.admit(cfgs[2], 5)
    with pytest.raises(BudgetExceeded):
        b.admit(cfgs[2], 5)
    assert b.used_bytes <= b.budget_bytes


def test_serve_stream_results_equal_alone():
    """The request loop: jobs arriving over time (virtual clock in steps) are
    admitted while others run; each result equals the same job run alone, bit
    for bit."""
    from dmd_b200.serve import job_mix, run_alone, serve
    jobs = job_mix(6, rate=0.05, seed=7, scale=0.02)
    out = serve(jobs, precision="mixed", profile="phys", chunk=10, virtual=True)
    assert out["jobs"] == 6
    assert out["job_latency"]["p99"] >= out["job_latency"]["p50"] > 0
    assert any(j.repacks for j in jobs)       # the mix did overlap
    for j in jobs:
        assert j.result["step"] == j.n_steps
        p, v, pe = run_alone(j, "mixed", "phys")
        assert np.array_equal(j.result["positions"], p), (j.jid, np.abs(j.result["positions"] - p).max())
        assert np.array_equal(j.result["velocities"], v), (j.jid, np.abs(j.result["velocities"] - v).max())
        assert j.result["potential_energy"] == pe, j.jid
