"""GPU dynamics parity: thermostats, barostats and trajectories through the C ABI
against the FP64 CPU oracle (whose REF engine is pinned bit for bit to the
reference's compiled SimulationEngine step), plus single-point parity at the
full size of the 30k-atom water box and NVE energy drift against the
reference's own engine.

Tolerances:
  fp64 path: positions within 1e-9 of the box edge, velocities 1e-9 relative RMS
             (argon; the water trajectories follow the existing 1e-8 / 1e-7);
  mixed path: argon 2e-5 (as the REF argon trajectory test); PHYS water 1e-6 nm
             in positions and 2e-5 relative RMS in velocities after 10 steps of
             0.5 fs (a 1e-6 relative force error moves an H atom by ~1e-8 nm
             and its velocity by ~3e-6 relative over that time).
"""
import numpy as np
import pytest

from dmd_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _engine(cfg, precision, profile, **kw):
    from dmd_b200.core import Engine
    return Engine(cfg, precision=precision, profile=profile, **kw)


def _water(n_mol=300, seed=9):
    box = (n_mol / 33.43) ** (1 / 3)
    return W.water_box(n_mol=n_mol, box=box, seed=seed, spacing=box / round(box / 0.1045)).config()


ARGON_TOL = {"fp64": 1e-9, "mixed": 2e-5}


def _follow(oe, eng, cfg, tol, rounds=4, steps=6):
    for k in range(rounds):
        oe.step(steps)
        eng.run_n(steps)
        L = oe.scalars()["box"]
        assert abs(eng.scalars().box - L) <= tol * L, (k, eng.scalars().box, L)
        assert np.abs(eng.positions - oe.get(0)).max() / L < tol, (k, np.abs(eng.positions - oe.get(0)).max())
        assert rel_rms(eng.velocities, oe.get(1)) < tol, (k, rel_rms(eng.velocities, oe.get(1)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("profile", ["ref", "phys"])
def test_andersen_thermostat_trajectory(oracle, profile, precision):
    """AndersenThermostat::apply (src/thermostat/andersen.cpp:14-32).  REF: the
    reference's own stream (mt19937_64 seeded per call, uniform then three
    normals per collision) drawn on the host, so the collided atoms and their
    new velocities are the reference's exactly; PHYS: counter-based Philox per
    (atom, call), the same draws as the oracle's restatement."""
    cfg = W.argon_fcc(n_cells=4, a=0.575, T=120.0, seed=7).config()
    cfg.thermostat.type = "andersen"
    cfg.thermostat.temperature = 100.0
    cfg.thermostat.frequency = 5.0  # collision probability 0.01 per atom per step
    oe = oracle.engine(cfg, profile)
    eng = _engine(cfg, precision, profile)
    v0 = eng.velocities.copy()
    _follow(oe, eng, cfg, ARGON_TOL[precision])
    # collisions happened: some atoms' velocities were redrawn
    assert oe.scalars()["andersen_calls"] == 24
    assert not np.allclose(eng.velocities, v0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_berendsen_barostat_ref(oracle, precision):
    """BerendsenBarostat::apply (src/barostat/berendsen_barostat.cpp:14-66) in the
    REF profile: mu = 1 - (dt/tau) (beta / 0.0602214086) (P0[bar] -
    P[kJ mol^-1 nm^-3]), the reference's unit mix, then positions and box scaled
    by mu^(1/3), with the second force evaluation the reference does after
    scaling."""
    cfg = W.argon_fcc(n_cells=4, a=0.575, T=120.0, seed=5).config()
    cfg.thermostat.type = "berendsen"
    cfg.thermostat.temperature = 100.0
    cfg.barostat.type = "berendsen"
    cfg.barostat.pressure = 100.0
    cfg.barostat.tau = 0.5
    oe = oracle.engine(cfg, "ref")
    eng = _engine(cfg, precision, "ref")
    _follow(oe, eng, cfg, ARGON_TOL[precision])
    assert oe.scalars()["box"] != cfg.box_size  # the box did move


@pytest.mark.parametrize("thermo,baro", [("nose-hoover", "none"), ("berendsen", "none"),
                                         ("berendsen", "berendsen")])
def test_water_trajectory_phys_mixed(oracle, thermo, baro):
    """Mixed precision PHYS water with SPME under each thermostat and the
    barostat follows the FP64 oracle (the FP64 path is held to 1e-8 in
    test_gpu_parity.py)."""
    cfg = _water(300, seed=9)
    cfg.thermostat.type = thermo
    cfg.barostat.type = baro
    cfg.barostat.tau = 0.5
    oe = oracle.engine(cfg, "phys")
    eng = _engine(cfg, "mixed", "phys")
    for k in range(2):
        oe.step(5)
        eng.run_n(5)
        assert np.abs(eng.positions - oe.get(0)).max() < 1e-6, k
        assert rel_rms(eng.velocities, oe.get(1)) < 2e-5, (k, rel_rms(eng.velocities, oe.get(1)))
        s, so = eng.scalars(), oe.scalars()
        assert abs(s.box - so["box"]) <= 1e-9 * so["box"], k
        assert abs(s.zeta - so["zeta"]) <= 1e-4 * abs(so["zeta"]) + 1e-6, (k, s.zeta, so["zeta"])


WATER30K = (10_000, 6.69)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("profile", ["phys", "ref"])
def test_single_point_water30k(oracle, profile, precision):
    """The 30k-atom water box at full size (64^3 SPME mesh, rc 1.0 nm): total
    forces and energy against the FP64 oracle on identical inputs."""
    n_mol, box = WATER30K
    cfg = W.water_box(n_mol=n_mol, box=box, seed=7, spacing=box / 64).config()
    F_o, e_o = oracle.forces(cfg, profile)
    eng = _engine(cfg, precision, profile)
    F, e = eng.compute_forces()
    tol = {"fp64": 1e-9, "mixed": 1e-5}[precision]
    assert rel_rms(F, F_o) < tol, rel_rms(F, F_o)
    tot = sum(e.values())
    assert abs(tot - e_o["total"]) <= tol * abs(e_o["total"]), (tot, e_o["total"])


def _nve_drift(energies):
    """max_t |E(t) - E(t1)| / |E(t1)| (tests/integration/test_argon_nve.cpp:150-171),
    t1 the first step: both engines evaluate their initial forces inside it."""
    e = np.asarray(energies, dtype=np.float64)
    return float(np.max(np.abs(e - e[0])) / abs(e[0]))


def _gpu_energies(cfg, precision, profile, steps):
    eng = _engine(cfg, precision, profile)
    out = []
    m = np.asarray(cfg.masses)
    for _ in range(steps):
        eng.run_n(1)
        v = eng.velocities
        ke = 0.5 * float(np.sum(m[:, None] * v * v))
        out.append(ke + eng.potential_energy)
    return out


def _ref_energies(ref, cfg, steps):
    re_ = ref.engine(cfg)
    m = np.asarray(cfg.masses)
    out = []
    for _ in range(steps):
        re_.step(1)
        v = re_.get(1)
        out.append(0.5 * float(np.sum(m[:, None] * v * v)) + re_.scalars()["pe"])
    return out


def test_nve_drift_no_worse_than_reference(ref):
    """NVE argon (dt 2 fs, 1.0 nm cutoff, Maxwell-Boltzmann start): the energy
    drift of the mixed-precision PHYS path (the product configuration) and of
    the FP64 path is no worse than that of the reference's own engine
    (compiled from its sources) on the same inputs."""
    cfg = W.argon_fcc(n_cells=4, a=0.575, T=120.0, seed=3).config()
    cfg.thermostat.type = "none"
    steps = 600
    d_ref = _nve_drift(_ref_energies(ref, cfg, steps))
    d_mixed = _nve_drift(_gpu_energies(cfg, "mixed", "phys", steps))
    d_fp64 = _nve_drift(_gpu_energies(cfg, "fp64", "phys", steps))
    assert d_mixed <= d_ref, (d_mixed, d_ref)
    assert d_fp64 <= d_ref, (d_fp64, d_ref)


def test_single_point_water750k(oracle):
    """The 750k-atom water box at full size (192^3 SPME mesh, Berendsen NPT
    configuration), mixed precision, PHYS: total forces and energy against the
    FP64 oracle on identical inputs (1e-5)."""
    cfg = W.water_box(n_mol=250_000, box=19.56, seed=7, spacing=0.1019, thermostat="berendsen",
                      barostat="berendsen").config()
    F_o, e_o = oracle.forces(cfg, "phys")
    eng = _engine(cfg, "mixed", "phys")
    F, e = eng.compute_forces()
    assert rel_rms(F, F_o) < 1e-5, rel_rms(F, F_o)
    tot = sum(e.values())
    assert abs(tot - e_o["total"]) <= 1e-5 * abs(e_o["total"]), (tot, e_o["total"])
