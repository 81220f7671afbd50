"""Seeded synthetic systems with the shapes of the benchmark configurations.

No public dataset is involved: every system is generated from a seed.  Each
generator returns a :class:`Workload` holding numpy arrays; ``.config()``
gives a SimulationConfig directly, ``.to_json()`` gives the reference's
``system.json`` / ``config.json`` dictionaries for the drop-in path.

  argon_fcc       LJ argon on an FCC lattice (4,000 atoms, 5.75 nm box)
  water_box       flexible 3-site water, jittered lattice, random orientations
                  (30,000 atoms in 6.69 nm; 750,000 atoms in 19.56 nm)
  lj_fluid        LJ fluid at reduced density / temperature (batch replicas)
  decane_melt     united-atom n-decane melt, chains grown as random walks
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .core import SimulationConfig
from .inputs import apply_config

KB = 0.008314462618
AR_SIGMA, AR_EPS, AR_MASS = 0.3405, 0.996, 39.948


@dataclass
class Workload:
    name: str
    box: float
    pos: np.ndarray                      # (N, 3)
    mass: np.ndarray
    charge: np.ndarray
    type_names: list
    lj_pairs: list                       # [(type_i, type_j, sigma, epsilon)]
    run: dict
    electrostatics: dict
    thermostat: dict
    barostat: dict
    lj_cutoff: float
    bonds: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    bond_k: np.ndarray = field(default_factory=lambda: np.zeros(0))
    bond_r0: np.ndarray = field(default_factory=lambda: np.zeros(0))
    angles: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    angle_k: np.ndarray = field(default_factory=lambda: np.zeros(0))
    angle_t0: np.ndarray = field(default_factory=lambda: np.zeros(0))
    dihedrals: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    dih_k: np.ndarray = field(default_factory=lambda: np.zeros(0))
    dih_n: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    dih_phi0: np.ndarray = field(default_factory=lambda: np.zeros(0))
    impropers: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    imp_k: np.ndarray = field(default_factory=lambda: np.zeros(0))
    imp_phi0: np.ndarray = field(default_factory=lambda: np.zeros(0))
    exclusions: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    constraints: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    constraint_dist: np.ndarray = field(default_factory=lambda: np.zeros(0))
    constraint_tol: float = 1e-6

    @property
    def n_atoms(self) -> int:
        return len(self.mass)

    def config_json(self) -> dict:
        return {
            "run": dict(self.run),
            "output": {"trajectory_path": "trajectory.h5", "nstxout": 0, "nstvout": 0,
                       "nstenergy": 0, "energy_path": "energy.h5", "checkpoint_interval": 0,
                       "checkpoint_path": "checkpoint.bin"},
            "lj": {"cutoff": float(self.lj_cutoff)},
            "electrostatics": dict(self.electrostatics),
            "thermostat": dict(self.thermostat),
            "barostat": dict(self.barostat),
            "constraints": {"type": "shake" if len(self.constraints) else "none",
                            "tolerance": float(self.constraint_tol)},
        }

    def to_json(self) -> tuple[dict, dict]:
        """(system.json, config.json) in the reference's input format."""
        ff = {"lennard_jones": {"cutoff": float(self.lj_cutoff), "pairs": [
            {"type_i": a, "type_j": b, "sigma": float(s), "epsilon": float(e)}
            for a, b, s, e in self.lj_pairs]}}
        if len(self.bonds):
            ff["bonds"] = [{"i": int(i), "j": int(j), "k": float(k), "r0": float(r)}
                           for (i, j), k, r in zip(self.bonds, self.bond_k, self.bond_r0)]
        if len(self.angles):
            ff["angles"] = [{"i": int(i), "j": int(j), "k": int(k), "k_theta": float(kt),
                             "theta0": float(t0)}
                            for (i, j, k), kt, t0 in zip(self.angles, self.angle_k, self.angle_t0)]
        if len(self.dihedrals):
            ff["dihedrals"] = [{"i": int(i), "j": int(j), "k": int(k), "l": int(l),
                                "k_phi": float(kp), "periodicity": int(n), "phi0": float(p0)}
                               for (i, j, k, l), kp, n, p0 in
                               zip(self.dihedrals, self.dih_k, self.dih_n, self.dih_phi0)]
        if len(self.impropers):
            ff["impropers"] = [{"i": int(i), "j": int(j), "k": int(k), "l": int(l), "k_phi": float(kp),
                                "phi0": float(p0)}
                               for (i, j, k, l), kp, p0 in zip(self.impropers, self.imp_k, self.imp_phi0)]
        if len(self.constraints):
            ff["constraints"] = [{"i": int(i), "j": int(j), "distance": float(dd)}
                                 for (i, j), dd in zip(self.constraints, self.constraint_dist)]
        system = {
            "cell": {"box_size": float(self.box), "positions": self.pos.tolist()},
            "atoms": {"mass": self.mass.tolist(), "charge": self.charge.tolist(),
                      "type": list(self.type_names)},
            "force_field": ff,
            "exclusions": self.exclusions.tolist(),
        }
        return system, self.config_json()

    def config(self) -> SimulationConfig:
        """SimulationConfig equal to load_inputs(*self.to_json())."""
        cfg = SimulationConfig()
        n = self.n_atoms
        cfg.box_size = float(self.box)
        cfg.pos_x, cfg.pos_y, cfg.pos_z = (self.pos[:, k].copy() for k in range(3))
        cfg.mass = self.mass
        cfg.charges = self.charge
        names = sorted(set(self.type_names))
        idx = {nm: i for i, nm in enumerate(names)}
        tn = np.asarray(self.type_names)
        types = np.zeros(n, np.int32)
        for nm, i in idx.items():
            types[tn == nm] = i
        cfg.atom_types = types
        nt = len(names)
        sig = np.full((nt, nt), 1.0)
        eps = np.zeros((nt, nt))
        for a, b, s, e in self.lj_pairs:
            sig[idx[a], idx[b]] = sig[idx[b], idx[a]] = s
            eps[idx[a], idx[b]] = eps[idx[b], idx[a]] = e
        cfg.use_lj = True
        cfg.lj_sigma, cfg.lj_epsilon = sig.ravel(), eps.ravel()
        if len(self.bonds):
            cfg.bond_i, cfg.bond_j = self.bonds[:, 0], self.bonds[:, 1]
            cfg.bond_k, cfg.bond_r0 = self.bond_k, self.bond_r0
        if len(self.angles):
            cfg.angle_i, cfg.angle_j, cfg.angle_k = self.angles[:, 0], self.angles[:, 1], self.angles[:, 2]
            cfg.angle_k_theta, cfg.angle_theta0 = self.angle_k, self.angle_t0
        if len(self.dihedrals):
            d = self.dihedrals
            cfg.dihedral_i, cfg.dihedral_j, cfg.dihedral_k, cfg.dihedral_l = d[:, 0], d[:, 1], d[:, 2], d[:, 3]
            cfg.dihedral_k_phi, cfg.dihedral_periodicity, cfg.dihedral_phi0 = self.dih_k, self.dih_n, self.dih_phi0
        if len(self.impropers):
            m = self.impropers
            cfg.improper_i, cfg.improper_j, cfg.improper_k, cfg.improper_l = m[:, 0], m[:, 1], m[:, 2], m[:, 3]
            cfg.improper_k_phi, cfg.improper_phi0 = self.imp_k, self.imp_phi0
        cfg.excl_i = self.exclusions[:, 0].tolist() if len(self.exclusions) else []
        cfg.excl_j = self.exclusions[:, 1].tolist() if len(self.exclusions) else []
        if len(self.constraints):
            cfg.constraint_i = self.constraints[:, 0].tolist()
            cfg.constraint_j = self.constraints[:, 1].tolist()
            cfg.constraint_dist = self.constraint_dist.tolist()
        apply_config(cfg, self.config_json())
        return cfg


def _run(dt, n_steps, T, seed, gen_vel=True):
    return {"dt": float(dt), "n_steps": int(n_steps), "init_temperature": float(T),
            "gen_vel": bool(gen_vel), "seed": int(seed)}


def _thermo(kind="none", T=300.0, tau=0.1, freq=10.0):
    return {"type": kind, "temperature": float(T), "tau": float(tau), "frequency": float(freq)}


def _baro(kind="none", P=1.0, tau=1.0, beta=4.5e-5):
    return {"type": kind, "pressure": float(P), "tau": float(tau), "compressibility": float(beta)}


def _elec(kind="cutoff", rc=1.0, spacing=0.12, alpha=3.12, order=4):
    return {"coulomb_type": kind, "cutoff": float(rc), "pme_order": int(order),
            "pme_grid_spacing": float(spacing), "ewald_coeff": float(alpha)}


def argon_fcc(n_cells: int = 10, a: float = 0.575, T: float = 120.0, seed: int = 2024,
              n_steps: int = 1000, rc: float = 1.0, dt: float = 0.002) -> Workload:
    """FCC argon (4 atoms per cell, lattice constant a); velocities generated by the
    engine at T with the seed (gen_vel)."""
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(n_cells)
    cells = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = ((cells[:, None, :] + base[None]) * a).reshape(-1, 3)
    n = len(pos)
    return Workload(
        name=f"argon_fcc_{n}", box=n_cells * a, pos=pos, mass=np.full(n, AR_MASS),
        charge=np.zeros(n), type_names=["Ar"] * n, lj_pairs=[("Ar", "Ar", AR_SIGMA, AR_EPS)],
        run=_run(dt, n_steps, T, seed), electrostatics=_elec("cutoff", rc),
        thermostat=_thermo(), barostat=_baro(), lj_cutoff=rc)


def _rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


WATER = dict(q_o=-0.8476, q_h=0.4238, m_o=15.9994, m_h=1.008, r0=0.1, theta0_deg=109.47,
             k_b=345000.0, k_a=383.0, sig_o=0.3166, eps_o=0.650)


def water_box(n_mol: int = 10_000, box: float = 6.69, seed: int = 7, spacing: float = 0.1045,
              thermostat: str = "nose-hoover", barostat: str = "none", n_steps: int = 1000,
              dt: float = 0.0005, T: float = 300.0, jitter: float = 0.1,
              rigid: bool = False, constraint_tol: float = 1e-8) -> Workload:
    """3-site water on a jittered cubic lattice with random orientations (O, H1,
    H2 per molecule; 1-2 and 1-3 exclusions).  Flexible by default; rigid=True
    adds SHAKE/RATTLE distance constraints O-H1, O-H2 and H1-H2 at the model's
    bond length and angle (the bond and angle terms stay in the force field)."""
    W = WATER
    rng = np.random.default_rng(seed)
    ns = int(math.ceil(n_mol ** (1.0 / 3.0) - 1e-9))
    a = box / ns
    g = np.arange(ns)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:n_mol]
    o = (sites + 0.5) * a + rng.uniform(-jitter, jitter, size=(n_mol, 3)) * a
    th = math.radians(W["theta0_deg"])
    ref = np.array([[W["r0"], 0.0, 0.0], [W["r0"] * math.cos(th), W["r0"] * math.sin(th), 0.0]])
    R = _rotations(rng, n_mol)
    h = np.einsum("nij,kj->nki", R, ref) + o[:, None, :]
    pos = np.concatenate([o[:, None, :], h], 1).reshape(-1, 3)
    n = 3 * n_mol
    mol = np.arange(n_mol) * 3
    mass = np.tile([W["m_o"], W["m_h"], W["m_h"]], n_mol)
    charge = np.tile([W["q_o"], W["q_h"], W["q_h"]], n_mol)
    names = ["OW", "HW", "HW"] * n_mol
    bonds = np.concatenate([np.stack([mol, mol + 1], 1), np.stack([mol, mol + 2], 1)]).astype(np.int32)
    bonds = bonds[np.lexsort((bonds[:, 1], bonds[:, 0]))]
    angles = np.stack([mol + 1, mol, mol + 2], 1).astype(np.int32)
    excl = np.stack([np.stack([mol, mol + 1], 1), np.stack([mol, mol + 2], 1),
                     np.stack([mol + 1, mol + 2], 1)], 1).reshape(-1, 2).astype(np.int32)
    tstat = _thermo(thermostat, T, 0.1)
    bstat = _baro(barostat, 1.0, 1.0, 4.5e-5)
    return Workload(
        name=f"water_{n}", box=box, pos=pos, mass=mass, charge=charge, type_names=names,
        lj_pairs=[("OW", "OW", W["sig_o"], W["eps_o"])],
        run=_run(dt, n_steps, T, seed), electrostatics=_elec("pme", 1.0, spacing, 3.12),
        thermostat=tstat, barostat=bstat, lj_cutoff=1.0,
        bonds=bonds, bond_k=np.full(len(bonds), W["k_b"]), bond_r0=np.full(len(bonds), W["r0"]),
        angles=angles, angle_k=np.full(n_mol, W["k_a"]), angle_t0=np.full(n_mol, th),
        exclusions=excl,
        constraints=(np.stack([np.stack([mol, mol + 1], 1), np.stack([mol, mol + 2], 1),
                               np.stack([mol + 1, mol + 2], 1)], 1).reshape(-1, 2).astype(np.int32)
                     if rigid else np.zeros((0, 2), np.int32)),
        constraint_dist=(np.tile([W["r0"], W["r0"], 2 * W["r0"] * math.sin(th / 2)], n_mol)
                         if rigid else np.zeros(0)),
        constraint_tol=constraint_tol)


def lj_fluid(n: int, rho_star: float, t_star: float, seed: int, n_steps: int = 1000,
             dt: float = 0.002) -> Workload:
    """LJ fluid (argon parameters) on a jittered simple-cubic lattice at reduced
    density rho* and temperature T*; cutoff 2.5 sigma."""
    rng = np.random.default_rng(seed)
    rho = rho_star / AR_SIGMA ** 3
    box = (n / rho) ** (1.0 / 3.0)
    ns = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    a = box / ns
    g = np.arange(ns)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:n]
    pos = (sites + 0.5) * a + rng.uniform(-0.05, 0.05, size=(n, 3)) * a
    T = t_star * AR_EPS / KB
    rc = 2.5 * AR_SIGMA
    return Workload(
        name=f"lj_{n}", box=box, pos=pos, mass=np.full(n, AR_MASS), charge=np.zeros(n),
        type_names=["Ar"] * n, lj_pairs=[("Ar", "Ar", AR_SIGMA, AR_EPS)],
        run=_run(dt, n_steps, T, seed), electrostatics=_elec("cutoff", rc),
        thermostat=_thermo(), barostat=_baro(), lj_cutoff=rc)


DECANE = dict(sig_ch3=0.375, eps_ch3=0.814, sig_ch2=0.395, eps_ch2=0.382, m_ch3=15.035,
              m_ch2=14.027, b0=0.154, kb=200000.0, th0_deg=114.0, ka=520.0,
              dih=((1, 2.95, 0.0), (2, -0.567, math.pi), (3, 6.58, 0.0)))


def decane_melt(n_chains: int, seed: int, chains_per_nm3: float = 3.09, n_steps: int = 1000,
                dt: float = 0.002, T: float = 300.0, d_min: float = 0.25,
                impropers: bool = False) -> Workload:
    """United-atom n-decane melt.  Chains grow as seeded random walks with fixed
    bond length and angle and torsions drawn near trans/gauche; a site is
    accepted only if it is at least d_min from every site placed before it
    (other than the preceding sites of its own chain), so the melt has no
    overlaps.  1-2, 1-3 and 1-4 exclusions; the Lorentz-Berthelot cross pair is
    written explicitly (the engine has no combining rule).  ``impropers`` adds
    two harmonic impropers per chain (sites 0-3 and 6-9, k 80 kJ/mol/rad^2,
    chi0 0.6 rad): a test system for the HarmonicImproper term, not part of the
    decane model."""
    D = DECANE
    rng = np.random.default_rng(seed)
    box = (n_chains / chains_per_nm3) ** (1.0 / 3.0)
    th = math.radians(D["th0_deg"])
    b = D["b0"]
    nc = max(1, int(box / d_min))
    cs = box / nc
    grid: dict = {}
    placed: list = []
    d2 = d_min * d_min

    def cell(p):
        c = np.floor(p / cs).astype(int) % nc
        return int(c[0]), int(c[1]), int(c[2])

    def clear(p, first_own):
        cx, cy, cz = cell(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for k in grid.get(((cx + dx) % nc, (cy + dy) % nc, (cz + dz) % nc), ()):
                        if k >= first_own:
                            continue  # own chain: bonded geometry keeps these apart
                        d = placed[k] - p
                        d -= box * np.round(d / box)
                        if d @ d < d2:
                            return False
        return True

    def unit(v):
        return v / np.linalg.norm(v)

    for c in range(n_chains):
        base = len(placed)
        for attempt in range(500):
            chain = [rng.uniform(0, box, 3)]
            if not clear(chain[0], base):
                continue
            for k in range(1, 10):
                for _ in range(60):
                    if k == 1:
                        cand = chain[0] + b * unit(rng.normal(size=3))
                    else:
                        u2 = unit(chain[k - 1] - chain[k - 2])
                        if k == 2:
                            t = rng.normal(size=3)
                            t = unit(t - (t @ u2) * u2)
                            dirv = math.cos(math.pi - th) * u2 + math.sin(math.pi - th) * t
                        else:
                            u1 = chain[k - 2] - chain[k - 3]
                            nrm = unit(np.cross(u1, u2))
                            m = np.cross(nrm, u2)
                            phi = rng.choice([math.pi, math.pi / 3, -math.pi / 3], p=[0.6, 0.2, 0.2])
                            phi += rng.normal(0, 0.2)
                            dirv = (math.cos(math.pi - th) * u2 + math.sin(math.pi - th) *
                                    (-math.cos(phi) * m + math.sin(phi) * nrm))
                        cand = chain[k - 1] + b * unit(dirv)
                    own_far = all(float((q - cand) @ (q - cand)) >= d2 for q in chain[:max(0, k - 3)])
                    if own_far and clear(cand, base):
                        chain.append(cand)
                        break
                else:
                    break
            if len(chain) == 10:
                for p in chain:
                    grid.setdefault(cell(p), []).append(len(placed))
                    placed.append(p)
                break
        else:
            raise RuntimeError("decane_melt: could not place a chain without overlaps")
    pos = np.array(placed).reshape(-1, 3)
    n = 10 * n_chains
    names = (["CH3"] + ["CH2"] * 8 + ["CH3"]) * n_chains
    mass = np.tile([D["m_ch3"]] + [D["m_ch2"]] * 8 + [D["m_ch3"]], n_chains)
    off = (np.arange(n_chains) * 10)[:, None, None]
    k = np.arange(10)
    bonds = (off + np.stack([k[:9], k[:9] + 1], 1)[None]).reshape(-1, 2).astype(np.int32)
    angles = (off + np.stack([k[:8], k[:8] + 1, k[:8] + 2], 1)[None]).reshape(-1, 3).astype(np.int32)
    quads = (off + np.stack([k[:7], k[:7] + 1, k[:7] + 2, k[:7] + 3], 1)[None]).reshape(-1, 4)
    dih = np.repeat(quads, 3, axis=0).astype(np.int32)
    dn = np.tile([t[0] for t in D["dih"]], len(quads)).astype(np.int32)
    dk = np.tile([t[1] for t in D["dih"]], len(quads))
    dp = np.tile([t[2] for t in D["dih"]], len(quads))
    ex = np.concatenate([np.stack([k[:9], k[:9] + 1], 1), np.stack([k[:8], k[:8] + 2], 1),
                         np.stack([k[:7], k[:7] + 3], 1)])
    excl = (off + ex[None]).reshape(-1, 2).astype(np.int32)
    s3, s2, e3, e2 = D["sig_ch3"], D["sig_ch2"], D["eps_ch3"], D["eps_ch2"]
    pairs = [("CH3", "CH3", s3, e3), ("CH2", "CH2", s2, e2),
             ("CH2", "CH3", 0.5 * (s2 + s3), math.sqrt(e2 * e3))]
    rc = 2.5 * s2
    return Workload(
        name=f"decane_{n}", box=box, pos=pos, mass=mass, charge=np.zeros(n), type_names=names,
        lj_pairs=pairs, run=_run(dt, n_steps, T, seed), electrostatics=_elec("cutoff", rc),
        thermostat=_thermo(), barostat=_baro(), lj_cutoff=rc,
        bonds=bonds, bond_k=np.full(len(bonds), D["kb"]), bond_r0=np.full(len(bonds), b),
        angles=angles, angle_k=np.full(len(angles), D["ka"]), angle_t0=np.full(len(angles), th),
        dihedrals=dih, dih_k=dk, dih_n=dn, dih_phi0=dp, exclusions=excl,
        **(_decane_impropers(n_chains) if impropers else {}))


def _decane_impropers(n_chains: int) -> dict:
    c = np.arange(n_chains)[:, None] * 10
    q = np.concatenate([c + np.arange(4), c + 6 + np.arange(4)]).astype(np.int32)
    return dict(impropers=q, imp_k=np.full(len(q), 80.0), imp_phi0=np.full(len(q), 0.6))


def batch_256(seed: int = 1234, n_lj: int = 192, n_dec: int = 64, scale: float = 1.0):
    """The 256-replica batch: LJ fluids N~U[500, 20000], rho*~U[0.60, 0.85],
    T*~U[0.8, 1.5]; decane melts of U[50, 400] chains.  Replica k uses seed+k.
    ``scale`` < 1 shrinks every N (test-sized batches)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_lj):
        n = max(64, int(rng.integers(500, 20001) * scale))
        out.append(lj_fluid(n, float(rng.uniform(0.60, 0.85)), float(rng.uniform(0.8, 1.5)),
                            seed + k))
    for k in range(n_dec):
        nc = max(8, int(rng.integers(50, 401) * scale))
        out.append(decane_melt(nc, seed + n_lj + k))
    return out
