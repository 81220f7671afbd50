"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Tolerances (relative RMS force error = |F - F_oracle|_2 / |F_oracle|_2 over 3N
components, energy error = |E - E_oracle| / |E_oracle|):
  fp64  path: 1e-9 force, 1e-9 energy (fixed-point accumulation at 2^-32)
  mixed path: 1e-5 force, 1e-5 energy (the stated target)
Pair lists must be identical as sorted integer (i<j) pair sets.
"""
import math

import numpy as np
import pytest

from dmd_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "mixed": 1e-5}


def rel_rms(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _engine(cfg, precision, profile, **kw):
    from dmd_b200.core import Engine
    return Engine(cfg, precision=precision, profile=profile, **kw)


def _argon(nc=5):
    return W.argon_fcc(n_cells=nc, a=0.575).config()


def _water(n_mol=1000, seed=3):
    box = (n_mol / 33.43) ** (1 / 3)
    return W.water_box(n_mol=n_mol, box=box, seed=seed, spacing=box / round(box / 0.1045)).config()


def _decane(n=30, seed=5, impropers=False):
    return W.decane_melt(n, seed, impropers=impropers).config()


def _jitter(cfg, s=0.01, seed=0):
    rng = np.random.default_rng(seed)
    n = len(cfg.masses)
    cfg.pos_x = cfg.pos_x + rng.normal(0, s, n)
    cfg.pos_y = cfg.pos_y + rng.normal(0, s, n)
    cfg.pos_z = cfg.pos_z + rng.normal(0, s, n)
    return cfg


SYSTEMS = {"argon": lambda: _jitter(_argon()), "water": lambda: _water(),
           "decane": lambda: _jitter(_decane(impropers=True), 0.005)}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("profile", ["ref", "phys"])
@pytest.mark.parametrize("system", ["argon", "water", "decane"])
def test_single_point_forces(oracle, system, profile, precision):
    cfg = SYSTEMS[system]()
    F_o, e_o = oracle.forces(cfg, profile)
    eng = _engine(cfg, precision, profile)
    F, e = eng.compute_forces()
    tol = TOL[precision]
    assert rel_rms(F, F_o) < tol, (system, profile, precision, rel_rms(F, F_o))
    tot = sum(e.values())
    assert abs(tot - e_o["total"]) <= tol * max(abs(e_o["total"]), 1.0) * 10, (tot, e_o["total"])


COMPONENTS = [(0, "lj"), (1, "bond"), (2, "angle"), (3, "dihedral"), (4, "creal"), (5, "pme"),
              (6, "excl"), (7, "improper")]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("profile", ["ref", "phys"])
def test_components_water_decane(oracle, profile, precision):
    for cfg in (_jitter(_water(600), 0.01), _jitter(_decane(20, impropers=True), 0.005)):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
        eng = _engine(cfg, precision, profile)
        for comp, name in COMPONENTS:
            f_o, e_o, _ = oracle.component(cfg, profile, comp)
            f, e = eng.component_compute(comp, pos, cfg.box_size)
            if np.linalg.norm(f_o) == 0 and e_o == 0:
                assert np.abs(f).max() < 1e-6 and abs(e) < 1e-6, name
                continue
            # fp64: the 2^-32 fixed-point step dominates for the small PME forces
            tol = TOL[precision] * ((30 if precision == "fp64" else 3) if name == "pme" else 1)
            assert rel_rms(f, f_o) < tol, (name, profile, precision, rel_rms(f, f_o))
            assert abs(e - e_o) <= tol * max(abs(e_o), 1.0) * 10, (name, e, e_o)


@pytest.mark.parametrize("profile", ["ref", "phys"])
@pytest.mark.parametrize("system", ["argon", "water", "decane"])
def test_pair_set_identical(oracle, system, profile):
    cfg = SYSTEMS[system]()
    eng = _engine(cfg, "mixed", profile, skin=0.1)
    eng.compute_forces()
    pi, pj = eng.pair_list()
    pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
    if profile == "ref":
        oi, oj = oracle.pairs(pos, cfg.box_size, cfg.lj_cutoff)
    else:
        rc = cfg.lj_cutoff
        if np.any(cfg.charges != 0):
            rc = max(rc, cfg.coulomb_cutoff)
        oi, oj = oracle.pairs(pos, cfg.box_size, rc + 0.1)
        ex = set(zip(np.minimum(cfg.excl_i, cfg.excl_j), np.maximum(cfg.excl_i, cfg.excl_j)))
        keep = np.array([(a, b) not in ex for a, b in zip(oi, oj)], bool)
        oi, oj = oi[keep], oj[keep]
    assert len(pi) == len(oi)
    assert np.array_equal(pi, oi) and np.array_equal(pj, oj)


# (molecules, box): 938 tiles (plain-scan list build) and 2063 tiles (cell ranges)
BIG_WATER = {"30k": (10_000, 6.69), "66k": (22_000, 8.70)}


def _big_water(size, shift_images):
    n_mol, box = BIG_WATER[size]
    cfg = W.water_box(n_mol=n_mol, box=box, seed=9, spacing=box / round(box / 0.1045)).config()
    if shift_images:
        # atoms scattered over periodic images (unwrapped coordinates)
        rng = np.random.default_rng(4)
        n = len(cfg.masses)
        L = cfg.box_size
        cfg.pos_x = cfg.pos_x + L * rng.integers(-1, 3, n)
        cfg.pos_y = cfg.pos_y + L * rng.integers(-2, 2, n)
        cfg.pos_z = cfg.pos_z + L * rng.integers(-1, 2, n)
    return cfg


@pytest.mark.parametrize("profile", ["ref", "phys"])
@pytest.mark.parametrize("shift_images", [False, True])
@pytest.mark.parametrize("size", ["30k", "66k"])
def test_pair_set_identical_large_box(oracle, size, profile, shift_images):
    """Boxes several cutoffs wide, below and above the tile count at which the
    list build takes its candidates from the sort grid's nearby columns and
    slabs: the pair set must still be the full O(N^2) minimum-image set."""
    cfg = _big_water(size, shift_images)
    eng = _engine(cfg, "mixed", profile, skin=0.1)
    eng.compute_forces()
    pi, pj = eng.pair_list()
    pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
    rc = cfg.lj_cutoff
    if profile == "phys":
        rc = max(rc, cfg.coulomb_cutoff) + 0.1
    oi, oj = oracle.pairs(pos, cfg.box_size, rc)
    if profile == "phys":
        n = len(cfg.masses)
        ei = np.asarray(cfg.excl_i, np.int64)
        ej = np.asarray(cfg.excl_j, np.int64)
        ex = np.minimum(ei, ej) * n + np.maximum(ei, ej)
        keep = ~np.isin(oi.astype(np.int64) * n + oj, ex)
        oi, oj = oi[keep], oj[keep]
    assert len(pi) == len(oi)
    assert np.array_equal(pi, oi) and np.array_equal(pj, oj)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_argon_trajectory_ref(oracle, precision):
    """REF profile argon NVE (the reference's LJ is correct): positions/velocities
    follow the FP64 oracle step by step, list cadence and counter included."""
    cfg = W.argon_fcc(n_cells=4, a=0.575, T=120.0, seed=5).config()
    oe = oracle.engine(cfg, "ref")
    eng = _engine(cfg, precision, "ref")
    tol = {"fp64": 1e-9, "mixed": 2e-5}[precision]
    for k in range(4):
        oe.step(6)
        eng.run_n(6)
        for which, name in ((0, "positions"), (1, "velocities")):
            g = eng.positions if which == 0 else eng.velocities
            o = oe.get(which)
            if which == 0:
                err = np.abs(g - o).max() / cfg.box_size
            else:
                err = rel_rms(g, o)
            assert err < tol, (k, name, err)
        s = eng.scalars()
        assert s.lj_step_since_rebuild == oe.scalars()["lj_counter"]
        assert abs(s.potential_energy - oe.scalars()["pe"]) < 1e-6 * abs(oe.scalars()["pe"]) * (100 if precision == "mixed" else 1)


@pytest.mark.parametrize("thermo,baro", [("nose-hoover", "none"), ("berendsen", "none"),
                                         ("berendsen", "berendsen")])
def test_water_trajectory_phys(oracle, thermo, baro):
    cfg = _water(300, seed=9)
    cfg.thermostat.type = thermo
    cfg.barostat.type = baro
    cfg.barostat.tau = 0.5
    oe = oracle.engine(cfg, "phys")
    eng = _engine(cfg, "fp64", "phys")
    oe.step(10)
    eng.run_n(10)
    assert np.abs(eng.positions - oe.get(0)).max() < 1e-8
    assert rel_rms(eng.velocities, oe.get(1)) < 1e-7
    s, so = eng.scalars(), oe.scalars()
    assert abs(s.box - so["box"]) < 1e-12 * so["box"] + 1e-14
    assert abs(s.zeta - so["zeta"]) <= 1e-7 * abs(so["zeta"]) + 1e-12


def test_run_to_run_bitwise():
    cfg = _water(500, seed=2)
    a = _engine(cfg, "mixed", "phys")
    b = _engine(cfg, "mixed", "phys")
    a.run_n(25)
    b.run_n(25)
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.velocities, b.velocities)
    assert a.potential_energy == b.potential_energy


def test_run_to_run_bitwise_cell_list_build():
    """A box large enough for the cell-range list build: its chunks, and with
    them the trajectory through several list rebuilds, repeat bit for bit."""
    cfg = _big_water("66k", False)
    a = _engine(cfg, "mixed", "phys")
    b = _engine(cfg, "mixed", "phys")
    a.run_n(40)
    b.run_n(40)
    assert a.scalars().list_builds > 1
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.velocities, b.velocities)
    assert a.potential_energy == b.potential_energy


def test_checkpoint_restart_bitwise(tmp_path):
    """tests/integration/test_checkpoint_restart.cpp: N steps == N/2 + save/load + N/2."""
    cfg = W.argon_fcc(n_cells=2, a=0.575, T=85.0, seed=4).config()
    cfg.lj_cutoff = 0.5
    full = _engine(cfg, "fp64", "ref")
    full.run_n(200)
    half = _engine(cfg, "fp64", "ref")
    half.run_n(100)
    p = str(tmp_path / "ck.bin")
    half.save_checkpoint(p)
    fresh = _engine(cfg, "fp64", "ref")
    fresh.load_checkpoint(p)
    assert fresh.current_step == 100
    fresh.run_n(100)
    assert fresh.current_step == 200
    assert np.array_equal(full.positions, fresh.positions)
    assert np.array_equal(full.velocities, fresh.velocities)


def _rigid_water(n_mol=100, tol=1e-8):
    """Rigid 3-site water: O-H1, O-H2 and H1-H2 distance constraints."""
    c = W.water_box(n_mol=n_mol, box=(n_mol / 33.4) ** (1 / 3), seed=3, spacing=0.1).config()
    mol = np.arange(n_mol) * 3
    r0, th = 0.09572, math.radians(104.52)
    c.constraint_type = "shake"
    c.constraint_tolerance = tol
    c.constraint_i = np.stack([mol, mol, mol + 1], 1).reshape(-1).astype(np.int32)
    c.constraint_j = np.stack([mol + 1, mol + 2, mol + 2], 1).reshape(-1).astype(np.int32)
    c.constraint_dist = np.tile([r0, r0, 2 * r0 * math.sin(th / 2)], n_mol)
    c.thermostat.type = "berendsen"
    c.dt = 0.001
    return c


@pytest.mark.parametrize("profile", ["ref", "phys"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_water_shake_rattle_trajectory(oracle, precision, profile):
    """Rigid water: SHAKE after the drift and RATTLE after the second half kick
    on the GPU (one thread per molecule) follow the FP64 oracle, whose REF
    engine is pinned bit for bit to the reference's Constraints (PHYS also
    gives SHAKE's displacement to the half-step velocities)."""
    c = _rigid_water()
    oe = oracle.engine(c, profile)
    eng = _engine(c, precision, profile)
    # positions (over the box edge) and velocities (relative RMS) against the
    # oracle.  The box (1.44 nm) is narrower than twice the list cutoff, so
    # the pair kernels take the minimum image of every pair at every
    # evaluation, as the oracle does.
    tol_x, tol_v = {"fp64": (1e-8, 1e-8), "mixed": (1e-4, 1e-4)}[precision]
    ci, cj, d0 = np.asarray(c.constraint_i), np.asarray(c.constraint_j), np.asarray(c.constraint_dist)
    L = c.box_size
    for k in range(3):
        oe.step(4)
        eng.run_n(4)
        x, v = eng.positions, eng.velocities
        assert np.abs(x - oe.get(0)).max() / L < tol_x, k
        assert rel_rms(v, oe.get(1)) < tol_v, k
        d = x[cj] - x[ci]
        d -= np.round(d / L) * L
        assert np.abs((d ** 2).sum(1) - d0 ** 2).max() < 1e-7, k
        # RATTLE: no relative velocity along the constraints
        assert np.abs((d * (v[cj] - v[ci])).sum(1)).max() < 1e-6, k


def test_constraints_rejected_with_andersen_thermostat():
    c = _rigid_water(n_mol=20)
    c.thermostat.type = "andersen"
    with pytest.raises(Exception, match="Andersen thermostat"):
        _engine(c, "fp64", "ref")


def _argon_andersen_npt(nc=4, seed=5):
    cfg = W.argon_fcc(n_cells=nc, a=0.575, T=120.0, seed=seed).config()
    cfg.thermostat.type = "berendsen"
    cfg.thermostat.temperature = 100.0
    cfg.barostat.type = "andersen"
    cfg.barostat.pressure = 300.0
    cfg.barostat.tau = 0.5
    return cfg


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_argon_andersen_barostat_ref(oracle, precision):
    """REF NPT with the Andersen barostat: positions, velocities and the box
    follow the FP64 oracle, whose restatement is pinned bit for bit to the
    reference's AndersenBarostat."""
    cfg = _argon_andersen_npt()
    oe = oracle.engine(cfg, "ref")
    eng = _engine(cfg, precision, "ref")
    tol = {"fp64": 1e-9, "mixed": 2e-5}[precision]
    for k in range(4):
        oe.step(6)
        eng.run_n(6)
        L = oe.scalars()["box"]
        assert abs(eng.scalars().box - L) <= tol * L, (k, eng.scalars().box, L)
        assert np.abs(eng.positions - oe.get(0)).max() / L < tol, k
        assert rel_rms(eng.velocities, oe.get(1)) < tol, k
    assert oe.scalars()["box"] != cfg.box_size


def test_andersen_barostat_phys_rejected():
    cfg = _argon_andersen_npt(nc=2)
    with pytest.raises(Exception, match="Andersen barostat"):
        _engine(cfg, "fp64", "phys")


def test_checkpoint_restart_bitwise_andersen_barostat(tmp_path):
    """The piston velocity travels in the checkpoint: N steps == N/2 + save/load + N/2."""
    cfg = _argon_andersen_npt(nc=3, seed=8)
    full = _engine(cfg, "fp64", "ref")
    full.run_n(40)
    half = _engine(cfg, "fp64", "ref")
    half.run_n(20)
    p = str(tmp_path / "ck.bin")
    half.save_checkpoint(p)
    fresh = _engine(cfg, "fp64", "ref")
    fresh.load_checkpoint(p)
    fresh.run_n(20)
    assert np.array_equal(full.positions, fresh.positions)
    assert np.array_equal(full.velocities, fresh.velocities)
    assert full.scalars().box == fresh.scalars().box


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_restart_bitwise_phys_npt(tmp_path, precision):
    """PHYS NPT: N steps == N/2 + save/load + N/2, bit for bit.  The trailer
    carries the barostat scale chosen at the end of the saved step (applied with
    the next drift) and the frame of the last list build, which the restart
    rebuilds the list in, so the mixed path's FP32 tile frame is the same too."""
    cfg = _water(300, seed=3)
    cfg.thermostat.type = "berendsen"
    cfg.barostat.type = "berendsen"
    cfg.barostat.tau = 0.5
    full = _engine(cfg, precision, "phys")
    full.run_n(30)
    half = _engine(cfg, precision, "phys")
    half.run_n(15)
    p = str(tmp_path / "ck_npt.bin")
    half.save_checkpoint(p)
    fresh = _engine(cfg, precision, "phys")
    fresh.load_checkpoint(p)
    fresh.run_n(15)
    assert fresh.current_step == 30
    assert fresh.box_size == full.box_size
    assert np.array_equal(full.positions, fresh.positions)
    assert np.array_equal(full.velocities, fresh.velocities)
    assert fresh.potential_energy == full.potential_energy


def test_repack_is_invisible():
    """A table rebuild (what admission / release does to running replicas)
    rebuilds each list in the frame of its last build: the trajectory continues
    bit for bit."""
    cfg = _water(400, seed=6)
    a = _engine(cfg, "mixed", "phys")
    a.run_n(24)
    b = _engine(cfg, "mixed", "phys")
    b.run_n(9)
    b.repack()
    b.run_n(8)
    b.repack()
    b.run_n(7)
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.velocities, b.velocities)
    assert a.potential_energy == b.potential_energy


@pytest.mark.parametrize("system", ["argon", "water", "decane"])
def test_cluster_form(oracle, system):
    """The 8-atom i-cluster pair form (nb_form="cluster8"): its rows hold the
    same pair set as the chunk list (pair_list checks them pair for pair),
    forces follow the FP64 oracle within the mixed tolerance, and runs repeat
    bit for bit."""
    cfg = SYSTEMS[system]()
    eng = _engine(cfg, "mixed", "phys", nb_form="cluster8")
    F, e = eng.compute_forces()
    pi, _ = eng.pair_list()  # raises if the cluster rows and the chunks disagree
    assert len(pi) > 0
    F_o, e_o = oracle.forces(cfg, "phys")
    assert rel_rms(F, F_o) < TOL["mixed"], rel_rms(F, F_o)
    a = _engine(cfg, "mixed", "phys", nb_form="cluster8")
    b = _engine(cfg, "mixed", "phys", nb_form="cluster8")
    a.run_n(20)
    b.run_n(20)
    assert np.array_equal(a.positions, b.positions)
    assert a.potential_energy == b.potential_energy


@pytest.mark.parametrize("form", ["chunk32", "cluster8"])
def test_narrow_box_minimum_image(oracle, form):
    """A box narrower than twice the list cutoff (100 flexible waters, 1.44 nm
    against 2 x 1.1 nm): the nearest image of a listed pair changes between
    list builds, so the mixed path runs these replicas through the
    minimum-image pair kernel and follows the oracle, which takes the minimum
    image at every evaluation.  A wide box runs without it; a barostat (which
    may shrink the box) turns it on."""
    c = W.water_box(n_mol=100, box=(100 / 33.4) ** (1 / 3), seed=3, spacing=0.1).config()
    c.thermostat.type = "berendsen"
    c.dt = 0.001
    oe = oracle.engine(c, "phys")
    eng = _engine(c, "mixed", "phys", nb_form=form)
    L = c.box_size
    for k in range(3):
        oe.step(4)
        eng.run_n(4)
        assert np.abs(eng.positions - oe.get(0)).max() / L < 1e-6, k
        assert rel_rms(eng.velocities, oe.get(1)) < 1e-4, k
    info = eng.launch_info()
    assert info["packed"] and info["min_image_kernel"], info
    wide = _engine(_water(1000), "mixed", "phys", nb_form=form)
    wide.run_n(2)
    assert not wide.launch_info()["min_image_kernel"]
    c2 = _water(1000)
    c2.barostat.type = "berendsen"
    c2.barostat.tau = 0.5
    npt = _engine(c2, "mixed", "phys", nb_form=form)
    F, _ = npt.compute_forces()  # at the starting configuration, as the oracle's
    assert npt.launch_info()["min_image_kernel"]
    F_o, _ = oracle.forces(c2, "phys")
    assert rel_rms(F, F_o) < TOL["mixed"]


def test_launch_info_reports_tuned_shape():
    """The launch configuration query after a run: the default chunk form, a
    blocks-per-SM count inside the tuner's candidates, and the captured step's
    kernel count equal to what a timed step reports."""
    eng = _engine(_water(1000), "mixed", "phys")
    eng.run_n(40)
    info = eng.launch_info()
    assert info["packed"] and info["nb_form"] == "chunk32"
    assert info["nb_blocks_per_sm"] in (1, 2, 3)
    assert info["n_replicas"] == 1 and info["n_atoms"] == 3000
    t = eng.step_timed(5, 0)
    assert info["launches_per_step"] > 0
    assert t["kernel_launches"] >= 5 * info["launches_per_step"] - 5
