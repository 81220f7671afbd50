"""Pin the CPU oracle before trusting it.

* Known-answer tests of the reference's own unit tests (values restated from
  tests/unit/force/*.cpp and tests/unit/core/test_cell.cpp).
* Bit-for-bit agreement of the oracle's ref profile with the reference's own
  classes compiled from source (oracle/_ref), component by component and for
  whole trajectories.
* The self-written FFT against numpy.fft; phys forces against finite
  differences of their energies; phys SPME against a direct Ewald sum.
"""
import math

import numpy as np
import pytest

from dmd_b200 import workloads as W
from dmd_b200.core import SimulationConfig

KE = 138.935456


# ---- known-answer tests from the reference's unit tests -------------------
def test_bspline_kat(oracle):
    # tests/unit/force/test_coulomb_pme.cpp:9-22
    assert abs(oracle.theta4(0.0) - 2.0 / 3.0) < 1e-12
    assert abs(oracle.theta4(1.0) - 1.0 / 6.0) < 1e-12
    assert abs(oracle.theta4(2.0)) < 1e-12
    assert abs(oracle.theta4(0.5) - (4.0 - 6.0 * 0.25 + 3.0 * 0.125) / 6.0) < 1e-12
    assert abs(oracle.theta4(0.3) - oracle.theta4(-0.3)) < 1e-12
    assert abs(oracle.dtheta4(0.0)) < 1e-12
    assert abs(oracle.dtheta4(0.5) + oracle.dtheta4(-0.5)) < 1e-12
    assert abs(oracle.dtheta4(1.0) + 0.5) < 1e-12
    assert abs(oracle.dtheta4(-1.0) - 0.5) < 1e-12


def test_self_energy_kat(oracle):
    # tests/unit/force/test_coulomb_pme.cpp:26-41
    a = 3.5
    assert abs(oracle.self_energy(a, [1.0]) - (-KE * a / math.sqrt(math.pi))) < 1e-10
    q = [1.0, -1.0, 0.5, -0.5]
    assert abs(oracle.self_energy(a, q) - (-KE * a / math.sqrt(math.pi) * 2.5)) < 1e-10


def test_min_image_kat(oracle):
    # tests/unit/core/test_cell.cpp:10-18
    out = oracle.min_image(2.0, [1.8, 0.3, -0.4])
    assert np.allclose(out, [-0.2, 0.3, -0.4], atol=1e-12)


def _cfg(pos, box, **kw):
    c = SimulationConfig()
    pos = np.asarray(pos, dtype=float)
    n = len(pos)
    c.box_size = box
    c.pos_x, c.pos_y, c.pos_z = pos[:, 0], pos[:, 1], pos[:, 2]
    c.mass = np.ones(n)
    c.charges = kw.pop("charges", np.zeros(n))
    c.atom_types = np.zeros(n, np.int32)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def test_bond_kat(oracle):
    # tests/unit/force/test_harmonic_bond.cpp:30-54 and :56-76
    c = _cfg([[0, 0, 0], [1.5, 0, 0]], 10.0, bond_i=[0], bond_j=[1], bond_k=[100.0], bond_r0=[1.0])
    f, e, _ = oracle.component(c, "ref", 1)
    assert abs(e - 0.5 * 100 * 0.25) < 1e-12
    assert abs(f[0, 0] - 50.0) < 1e-12 and abs(f[1, 0] + 50.0) < 1e-12
    c = _cfg([[0, 0, 0], [1.0, 0, 0], [2.8, 0, 0]], 20.0, bond_i=[0, 1], bond_j=[1, 2],
             bond_k=[100.0, 200.0], bond_r0=[1.0, 1.5])
    _, e, _ = oracle.component(c, "ref", 1)
    assert abs(e - 9.0) < 1e-10


def test_lj_kat(oracle):
    # tests/unit/force/test_lennard_jones.cpp:7-61
    c = _cfg([[0, 0, 0], [0.3, 0, 0]], 10.0, lj_sigma=[0.3], lj_epsilon=[0.5], lj_cutoff=2.0, use_lj=True)
    _, e, _ = oracle.component(c, "ref", 0)
    assert abs(e) < 1e-12
    c = _cfg([[0, 0, 0], [0.2, 0, 0]], 10.0, lj_sigma=[0.2649], lj_epsilon=[0.5], lj_cutoff=2.0, use_lj=True)
    f, e, _ = oracle.component(c, "ref", 0)
    assert e > 0 and f[0, 0] < 0 and f[1, 0] > 0


def test_dihedral_kat(oracle):
    # tests/unit/force/test_periodic_dihedral.cpp:7-108
    base = dict(dihedral_i=[0], dihedral_j=[1], dihedral_k=[2], dihedral_l=[3])
    c = _cfg([[0, 0, 0], [1, 0, 0], [2, 0, 0], [3, 0, 1]], 20.0, dihedral_periodicity=[1],
             dihedral_k_phi=[10.0], dihedral_phi0=[math.pi], **base)
    _, e, _ = oracle.component(c, "ref", 3)
    assert abs(e) < 1e-10
    c = _cfg([[0, 0, 0], [1, 0, 0], [1, 1, 0], [1, 1, 1]], 20.0, dihedral_periodicity=[2],
             dihedral_k_phi=[3.0], dihedral_phi0=[math.pi / 3], **base)
    _, e, _ = oracle.component(c, "ref", 3)
    assert abs(e - 3.0 * (1.0 + math.cos(2.0 * math.pi / 2.0 - math.pi / 3.0))) < 1e-10
    c = _cfg([[0, 0, 0], [1, 0, 0], [1.2, 0.5, 0], [1.5, 0.8, 0.5]], 20.0, dihedral_periodicity=[3],
             dihedral_k_phi=[5.0], dihedral_phi0=[0.0], **base)
    for prof in ("ref", "phys"):
        f, _, _ = oracle.component(c, prof, 3)
        assert np.abs(f.sum(0)).max() < 1e-12


def test_angle_kat(oracle):
    # tests/unit/force/test_harmonic_angle.cpp:7-74
    base = dict(angle_i=[0], angle_j=[1], angle_k=[2], angle_k_theta=[100.0])
    c = _cfg([[0, 0, 0], [0, 1, 0], [1, 1, 0]], 10.0, angle_theta0=[math.pi / 2], **base)
    _, e, _ = oracle.component(c, "ref", 2)
    assert abs(e) < 1e-12
    c = _cfg([[0, 0, 0], [0, 1, 0], [1, 1, 1]], 10.0, angle_theta0=[math.pi / 3], **base)
    f, e, _ = oracle.component(c, "ref", 2)
    assert e > 0 and np.abs(f.sum(0)).max() < 1e-12


# ---- oracle (ref profile) == reference classes, bit for bit ---------------
def _small_water(n_mol=300, seed=3):
    w = W.water_box(n_mol=n_mol, box=(n_mol / 33.4) ** (1 / 3), seed=seed, spacing=0.1)
    return w.config()


def test_pairs_equal_reference(oracle, ref):
    c = W.argon_fcc(n_cells=5, a=0.575).config()
    rng = np.random.default_rng(1)
    pos = np.stack([c.pos_x, c.pos_y, c.pos_z], 1) + rng.normal(0, 0.02, (len(c.masses), 3))
    _, _, (ri, rj) = ref.lj(c, pos=pos)
    oi, oj = oracle.pairs(pos, c.box_size, c.lj_cutoff)
    assert np.array_equal(ri, oi) and np.array_equal(rj, oj)


@pytest.mark.parametrize("which", ["argon", "water", "decane"])
def test_components_bitwise_vs_reference(oracle, ref, which):
    if which == "argon":
        c = W.argon_fcc(n_cells=5, a=0.575).config()
    elif which == "water":
        c = _small_water()
    else:
        c = W.decane_melt(20, 5, impropers=True).config()
    rng = np.random.default_rng(2)
    pos = np.stack([c.pos_x, c.pos_y, c.pos_z], 1) + rng.normal(0, 0.005, (len(c.masses), 3))
    fr, er, _ = ref.lj(c, pos=pos)
    fo, eo, _ = oracle.component(c, "ref", 0, pos=pos)
    assert np.array_equal(fr, fo) and er == eo
    if len(c.bond_i):
        fr, er = ref.bond(c, pos=pos)
        fo, eo, _ = oracle.component(c, "ref", 1, pos=pos)
        assert np.array_equal(fr, fo) and er == eo
    if len(c.angle_i):
        fr, er = ref.angle(c, pos=pos)
        fo, eo, _ = oracle.component(c, "ref", 2, pos=pos)
        assert np.array_equal(fr, fo) and er == eo
    if len(c.dihedral_i):
        fr, er = ref.dihedral(c, pos=pos)
        fo, eo, _ = oracle.component(c, "ref", 3, pos=pos)
        assert np.array_equal(fr, fo) and er == eo
    if len(c.improper_i):
        fr, er = ref.improper(c, pos=pos)
        fo, eo, _ = oracle.component(c, "ref", 7, pos=pos)
        assert np.array_equal(fr, fo) and er == eo
    if len(c.excl_i):
        fr, er = ref.exclusion(c, pos=pos)
        fo, eo, _ = oracle.component(c, "ref", 6, pos=pos)
        assert np.array_equal(fr, fo) and er == eo


@pytest.mark.parametrize("thermo,baro", [("none", "none"), ("berendsen", "none"),
                                         ("nose-hoover", "none"), ("andersen", "none"),
                                         ("berendsen", "berendsen")])
def test_trajectory_bitwise_vs_reference(oracle, ref, thermo, baro):
    c = W.argon_fcc(n_cells=3, a=0.575, T=120.0, seed=11).config()
    c.lj_cutoff = 0.8
    c.thermostat.type = thermo
    c.thermostat.temperature = 100.0
    c.thermostat.frequency = 5.0
    c.barostat.type = baro
    c.barostat.pressure = 100.0
    re_ = ref.engine(c)
    oe = oracle.engine(c, "ref")
    for _ in range(3):
        re_.step(7)
        oe.step(7)
        for w in (0, 1, 2):
            assert np.array_equal(re_.get(w), oe.get(w)), (thermo, baro, w)
        rs, os_ = re_.scalars(), oe.scalars()
        assert rs["pe"] == os_["pe"] and rs["box"] == os_["box"]
        assert rs["lj_counter"] == os_["lj_counter"] and rs["zeta"] == os_["zeta"]


def test_trajectory_water_cutoff_bitwise(oracle, ref):
    c = _small_water(n_mol=100)
    c.coulomb_type = "cutoff"
    c.thermostat.type = "nose-hoover"
    re_ = ref.engine(c)
    oe = oracle.engine(c, "ref")
    re_.step(5)
    oe.step(5)
    for w in (0, 1, 2):
        assert np.array_equal(re_.get(w), oe.get(w))


@pytest.mark.parametrize("n_mol,box,spacing", [(100, 1.45, 0.1), (216, 1.87, 0.12), (60, 1.24, 0.11)])
def test_pme_bitwise_vs_reference(oracle, ref, n_mol, box, spacing):
    """CoulombPME::compute (the reference's own source, compiled against the
    FFTW-API shim) against the oracle's REF restatement: identical bits, on
    even and odd meshes (K = 14, 16, 11)."""
    c = W.water_box(n_mol=n_mol, box=box, seed=n_mol, spacing=spacing,
                    thermostat="nose-hoover", dt=0.0005).config()
    rng = np.random.default_rng(n_mol)
    pos = np.stack([c.pos_x, c.pos_y, c.pos_z], 1) + rng.normal(0, 0.01, (len(c.masses), 3))
    fr, er = ref.pme(c, pos=pos)
    fo, eo, _ = oracle.component(c, "ref", 5, pos=pos)
    assert np.array_equal(fr, fo) and er == eo


def test_trajectory_water_pme_bitwise(oracle, ref):
    """Whole engine with the pme branch of build_force_engine (direct + PME +
    exclusion) against the oracle engine, REF profile."""
    c = _small_water(n_mol=100)
    c.coulomb_type = "pme"
    c.thermostat.type = "nose-hoover"
    re_ = ref.engine(c)
    oe = oracle.engine(c, "ref")
    for _ in range(2):
        re_.step(3)
        oe.step(3)
        for w in (0, 1, 2):
            assert np.array_equal(re_.get(w), oe.get(w))
        assert re_.scalars()["pe"] == oe.scalars()["pe"]


# ---- FFT ---------------------------------------------------------------------
@pytest.mark.parametrize("K", [8, 12, 15, 16, 20])
def test_fft_vs_numpy(oracle, K):
    rng = np.random.default_rng(K)
    a = rng.normal(size=(K, K, K))
    ours = oracle.rfft3(a)
    ref = np.fft.rfftn(a)
    assert np.abs(ours - ref).max() < 1e-11 * np.abs(ref).max()


# ---- phys profile: forces are gradients of the energy ------------------------
def _fd_check(oracle, c, comp, n_check=6, h=1e-6, tol=2e-6, seed=0):
    rng = np.random.default_rng(seed)
    pos = np.stack([c.pos_x, c.pos_y, c.pos_z], 1)
    f, _, _ = oracle.component(c, "phys", comp, pos=pos)
    atoms = rng.choice(len(pos), size=min(n_check, len(pos)), replace=False)
    for a in atoms:
        for d in range(3):
            p1 = pos.copy()
            p1[a, d] += h
            p2 = pos.copy()
            p2[a, d] -= h
            e1 = oracle.component(c, "phys", comp, pos=p1)[1]
            e2 = oracle.component(c, "phys", comp, pos=p2)[1]
            fd = -(e1 - e2) / (2 * h)
            assert abs(fd - f[a, d]) <= tol * max(1.0, abs(fd)), (comp, a, d, fd, f[a, d])


def test_phys_fd_bonded(oracle):
    c = W.decane_melt(4, 9, impropers=True).config()
    rng = np.random.default_rng(5)
    c.pos_x = c.pos_x + rng.normal(0, 0.01, len(c.pos_x))
    c.pos_y = c.pos_y + rng.normal(0, 0.01, len(c.pos_x))
    for comp in (1, 2, 3, 7):
        _fd_check(oracle, c, comp, n_check=10, tol=5e-6)


def test_phys_fd_nonbonded(oracle):
    c = _small_water(n_mol=60, seed=4)
    for comp in (0, 4, 6):
        _fd_check(oracle, c, comp, n_check=5, tol=5e-6)


def test_phys_fd_pme(oracle):
    c = _small_water(n_mol=40, seed=6)
    c.pme_grid_spacing = c.box_size / 16
    _fd_check(oracle, c, 5, n_check=4, h=1e-5, tol=2e-5)


def _direct_ewald_recip(pos, q, L, alpha, kmax):
    """Reciprocal-space Ewald energy by explicit k sums (reference for SPME)."""
    m = np.arange(-kmax, kmax + 1)
    M = np.stack(np.meshgrid(m, m, m, indexing="ij"), -1).reshape(-1, 3)
    M = M[np.any(M != 0, axis=1)]
    k = 2 * np.pi * M / L
    k2 = (k ** 2).sum(1)
    S = (q[None, :] * np.exp(1j * (k @ pos.T))).sum(1)
    V = L ** 3
    return 0.5 * (4 * np.pi * KE / V * np.exp(-k2 / (4 * alpha ** 2)) / k2 * np.abs(S) ** 2).sum()


def test_phys_pme_vs_direct_ewald(oracle):
    c = _small_water(n_mol=30, seed=8)
    c.pme_grid_spacing = c.box_size / 32
    pos = np.stack([c.pos_x, c.pos_y, c.pos_z], 1)
    _, e, _ = oracle.component(c, "phys", 5)
    e_self = -KE * c.ewald_coeff / math.sqrt(math.pi) * (c.charges ** 2).sum()
    e_dir = _direct_ewald_recip(pos, c.charges, c.box_size, c.ewald_coeff, 14)
    assert abs((e - e_self) - e_dir) < 2e-4 * abs(e_dir)


def test_philox_known_answer(oracle):
    # Philox4x32-10 test vector from the Random123 distribution (counter 0, key 0)
    assert oracle.philox([0, 0, 0, 0], 0) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]


# ---- distance constraints: SHAKE / RATTLE (src/integrate/constraints.cpp) ----
def test_shake_rattle_kat(oracle):
    # tests/unit/integrate/test_constraints.cpp:11-92 (box 100 nm: no wrapping)
    m2, m3 = np.ones(2), np.ones(3)
    p, _ = oracle.shake(np.array([[0.0, 0.0, 0.0], [1.1, 0.1, 0.05]]), m2, [0], [1], [1.0], 100.0)
    assert abs(np.linalg.norm(p[1] - p[0]) - 1.0) < 1e-6
    p, _ = oracle.shake(np.array([[0.0, 0.0, 0.0], [1.05, 0.1, 0.0], [2.1, -0.1, 0.0]]), m3,
                        [0, 1], [1, 2], [1.0, 1.0], 100.0)
    assert abs(np.linalg.norm(p[1] - p[0]) - 1.0) < 1e-6
    assert abs(np.linalg.norm(p[2] - p[1]) - 1.0) < 1e-6
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    v, _ = oracle.rattle(pos, np.array([[0.1, 0.0, 0.0], [0.3, 0.0, 0.0]]), m2, [0], [1], 100.0)
    assert abs((pos[1, 0] - pos[0, 0]) * (v[1, 0] - v[0, 0])) < 1e-8


def _constrained_water(n_mol, seed, jitter):
    """Rigid-water constraints (O-H1, O-H2, H1-H2) on a perturbed water box
    shifted so that molecules straddle the periodic boundary."""
    w = W.water_box(n_mol=n_mol, box=(n_mol / 33.43) ** (1 / 3), seed=seed, spacing=0.1)
    rng = np.random.default_rng(seed)
    L = w.box
    pos = w.pos + rng.normal(0.0, jitter, w.pos.shape) + 0.5 * L
    mol = np.arange(n_mol) * 3
    ci = np.stack([mol, mol, mol + 1], 1).reshape(-1).astype(np.int32)
    cj = np.stack([mol + 1, mol + 2, mol + 2], 1).reshape(-1).astype(np.int32)
    r0, th = 0.09572, math.radians(104.52)
    dist = np.tile([r0, r0, 2 * r0 * math.sin(th / 2)], n_mol)
    vel = rng.normal(0.0, 0.5, pos.shape)
    return pos, vel, w.mass, ci, cj, dist, L


@pytest.mark.parametrize("jitter,tol", [(0.002, 1e-8), (0.01, 1e-10)])
def test_shake_rattle_bitwise_vs_reference(oracle, ref, jitter, tol):
    pos, vel, m, ci, cj, dist, L = _constrained_water(300, 11, jitter)
    p_o, sweeps = oracle.shake(pos, m, ci, cj, dist, L, tol)
    p_r = ref.shake(pos, m, ci, cj, dist, L, tol)
    assert sweeps > 1
    assert np.array_equal(p_o, p_r)
    v_o, _ = oracle.rattle(p_o, vel, m, ci, cj, L, tol)
    v_r = ref.rattle(p_r, vel, m, ci, cj, dist, L, tol)
    assert np.array_equal(v_o, v_r)
    # converged: bond lengths and relative velocities along the bonds
    d = p_o[cj] - p_o[ci]
    d -= np.round(d / L) * L
    r2 = (d ** 2).sum(1)
    assert np.abs(r2 - dist ** 2).max() < 10 * tol
    assert np.abs((d * (v_o[cj] - v_o[ci])).sum(1)).max() < 10 * tol


def _rigid(c, tol):
    """Rigid-water constraints (O-H1, O-H2, H1-H2) on a water config."""
    n_mol = len(c.masses) // 3
    mol = np.arange(n_mol) * 3
    r0, th = 0.09572, math.radians(104.52)
    c.constraint_type = "shake"
    c.constraint_tolerance = tol
    c.constraint_i = np.stack([mol, mol, mol + 1], 1).reshape(-1).astype(np.int32)
    c.constraint_j = np.stack([mol + 1, mol + 2, mol + 2], 1).reshape(-1).astype(np.int32)
    c.constraint_dist = np.tile([r0, r0, 2 * r0 * math.sin(th / 2)], n_mol)
    return c


def test_trajectory_shake_bitwise_vs_reference(oracle, ref):
    """SimulationEngine::step with constraints (SHAKE after the drift, RATTLE
    after the second half kick): the oracle engine's REF profile against the
    reference's own classes, bit for bit."""
    c = _rigid(_small_water(n_mol=100), 1e-8)
    c.coulomb_type = "cutoff"
    c.thermostat.type = "berendsen"
    c.dt = 0.001
    re_ = ref.engine(c)
    oe = oracle.engine(c, "ref")
    for _ in range(3):
        re_.step(4)
        oe.step(4)
        for w in (0, 1, 2):
            assert np.array_equal(re_.get(w), oe.get(w)), w
        assert re_.scalars()["pe"] == oe.scalars()["pe"]


def test_phys_shake_keeps_constraints(oracle):
    """PHYS profile: after every step the constrained distances hold to the
    tolerance and the relative velocities along them vanish (RATTLE)."""
    tol = 1e-10
    c = _rigid(_small_water(n_mol=100), tol)
    c.coulomb_type = "cutoff"
    c.dt = 0.002
    oe = oracle.engine(c, "phys")
    ci, cj, d0 = np.asarray(c.constraint_i), np.asarray(c.constraint_j), np.asarray(c.constraint_dist)
    L = c.box_size
    for _ in range(5):
        oe.step(2)
        x, v = oe.get(0), oe.get(1)
        d = x[cj] - x[ci]
        d -= np.round(d / L) * L
        assert np.abs((d ** 2).sum(1) - d0 ** 2).max() < 10 * tol
        assert np.abs((d * (v[cj] - v[ci])).sum(1)).max() < 10 * tol


@pytest.mark.parametrize("pressure", [1.0, 300.0])
def test_trajectory_andersen_barostat_bitwise_vs_reference(oracle, ref, pressure):
    """AndersenBarostat (piston velocity, exp(eps_dot dt) scaling of positions
    and box) in the engine step: the oracle's REF restatement against the
    reference's own class, bit for bit, box included."""
    c = W.argon_fcc(n_cells=3, a=0.575, T=120.0, seed=11).config()
    c.lj_cutoff = 0.8
    c.thermostat.type = "berendsen"
    c.thermostat.temperature = 100.0
    c.barostat.type = "andersen"
    c.barostat.pressure = pressure
    c.barostat.tau = 0.5
    re_ = ref.engine(c)
    oe = oracle.engine(c, "ref")
    box0 = c.box_size
    for _ in range(3):
        re_.step(7)
        oe.step(7)
        for w in (0, 1, 2):
            assert np.array_equal(re_.get(w), oe.get(w)), w
        rs, os_ = re_.scalars(), oe.scalars()
        assert rs["box"] == os_["box"] and rs["pe"] == os_["pe"]
    assert oe.scalars()["box"] != box0


def test_rigid_water_workload_round_trip_and_oracle(oracle):
    """water_box(rigid=True) in the reference's input format: system.json
    constraints + config.json "shake" read back by load_inputs give the same
    constraints as the direct config; the oracle keeps them through steps."""
    from dmd_b200.inputs import load_inputs
    w = W.water_box(n_mol=64, box=(64 / 33.4) ** (1 / 3), seed=2, spacing=0.1, rigid=True,
                    dt=0.002, thermostat="berendsen")
    c = w.config()
    sysj, cfgj = w.to_json()
    b = load_inputs(sysj, cfgj)
    assert c.constraint_type == b.constraint_type == "shake"
    assert c.constraint_tolerance == b.constraint_tolerance == 1e-8
    for k in ("constraint_i", "constraint_j", "constraint_dist"):
        assert np.array_equal(np.asarray(getattr(c, k)), np.asarray(getattr(b, k))), k
    ci, cj, d0 = np.asarray(c.constraint_i), np.asarray(c.constraint_j), np.asarray(c.constraint_dist)
    oe = oracle.engine(c, "phys")
    oe.step(10)
    x = oe.get(0)
    d = x[cj] - x[ci]
    d -= np.round(d / c.box_size) * c.box_size
    assert np.abs((d ** 2).sum(1) - d0 ** 2).max() < 1e-7
