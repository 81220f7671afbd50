"""TEST INFRASTRUCTURE ONLY -- ctypes wrappers of the CPU checkers.

* ``Oracle``: this repository's FP64 restatement (libdmd_oracle.so, built from
  oracle/dmd_oracle.cpp), both semantic profiles.
* ``Ref``: the reference's own C++ classes compiled from source
  (oracle/_ref/libdmdref.so, built by oracle/Makefile from the reference tree).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs import this module.  The product (dmd_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libdmd_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdmdref.so")
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
KE = 138.935456
KB = 0.008314462618


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree exists, oracle/_ref: the
    reference's sources, and the adapter check once libdmdgpu.so is built)."""
    targets = ["oracle"] + (["ref", "adapter"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _d(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    return a, a.ctypes.data_as(_ip)


class orc_system(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int), ("box", C.c_double), ("q", _dp), ("type", _ip), ("n_types", C.c_int),
        ("lj_sigma", _dp), ("lj_eps", _dp), ("use_lj", C.c_int), ("lj_cutoff", C.c_double),
        ("coulomb_type", C.c_int), ("coul_cutoff", C.c_double), ("ewald", C.c_double),
        ("pme_K", C.c_int), ("pme_order", C.c_int),
        ("n_excl", C.c_int), ("excl_i", _ip), ("excl_j", _ip),
        ("n_bonds", C.c_int), ("bond_i", _ip), ("bond_j", _ip), ("bond_k", _dp), ("bond_r0", _dp),
        ("n_angles", C.c_int), ("ang_i", _ip), ("ang_j", _ip), ("ang_k", _ip), ("ang_kt", _dp),
        ("ang_t0", _dp),
        ("n_dih", C.c_int), ("dih_i", _ip), ("dih_j", _ip), ("dih_k", _ip), ("dih_l", _ip),
        ("dih_n", _ip), ("dih_kphi", _dp), ("dih_phi0", _dp),
        ("n_imp", C.c_int), ("imp_i", _ip), ("imp_j", _ip), ("imp_k", _ip), ("imp_l", _ip),
        ("imp_kphi", _dp), ("imp_phi0", _dp),
        ("profile", C.c_int),
    ]


class orc_energy(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("lj", "coul_real", "coul_recip", "coul_self",
                                          "coul_excl", "bond", "angle", "dihedral", "improper",
                                          "total", "virial")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class orc_run(C.Structure):
    _fields_ = [("dt", C.c_double), ("mass", _dp), ("x", _dp), ("y", _dp), ("z", _dp),
                ("vx", _dp), ("vy", _dp), ("vz", _dp), ("gen_vel", C.c_int), ("seed", C.c_int),
                ("init_temperature", C.c_double), ("thermostat", C.c_int),
                ("t_temp", C.c_double), ("t_tau", C.c_double), ("t_freq", C.c_double),
                ("barostat", C.c_int), ("b_pressure", C.c_double), ("b_tau", C.c_double),
                ("b_compress", C.c_double), ("rng_seed", C.c_uint64), ("brute_list", C.c_int),
                ("n_cons", C.c_int), ("cons_i", _ip), ("cons_j", _ip), ("cons_dist", _dp),
                ("cons_tol", C.c_double)]


THERMO = {"none": 0, "berendsen": 1, "nose-hoover": 2, "andersen": 3}
BARO = {"none": 0, "berendsen": 1, "andersen": 2}


def pme_mesh(cfg) -> int:
    """Mesh points per axis: max(8, int(box/spacing + 0.5)) (simulation_engine.cpp:183-185)."""
    return max(8, int(cfg.box_size / cfg.pme_grid_spacing + 0.5))


class _Sys:
    """orc_system built from a SimulationConfig (arrays kept alive)."""

    def __init__(self, cfg, profile: str):
        k = []

        def d(v):
            a, p = _d(v)
            k.append(a)
            return p

        def i(v):
            a, p = _i(v)
            k.append(a)
            return p

        n = len(cfg.masses)
        s = orc_system()
        s.n_atoms = n
        s.box = float(cfg.box_size)
        s.q = d(cfg.charges if len(cfg.charges) else np.zeros(n))
        s.type = i(cfg.atom_types if len(cfg.atom_types) else np.zeros(n, np.int32))
        s.n_types = cfg.lj_n_types
        if s.n_types:
            s.lj_sigma, s.lj_eps = d(cfg.lj_sigma), d(cfg.lj_epsilon)
        s.use_lj = int(bool(cfg.use_lj))
        s.lj_cutoff = float(cfg.lj_cutoff)
        s.coulomb_type = 1 if cfg.coulomb_type == "pme" else 0
        s.coul_cutoff = float(cfg.coulomb_cutoff)
        s.ewald = float(cfg.ewald_coeff)
        s.pme_K = pme_mesh(cfg)
        s.pme_order = int(cfg.pme_order)
        s.n_excl = len(cfg.excl_i)
        if s.n_excl:
            s.excl_i, s.excl_j = i(cfg.excl_i), i(cfg.excl_j)
        s.n_bonds = len(cfg.bond_i)
        if s.n_bonds:
            s.bond_i, s.bond_j, s.bond_k, s.bond_r0 = i(cfg.bond_i), i(cfg.bond_j), d(cfg.bond_k), d(cfg.bond_r0)
        s.n_angles = len(cfg.angle_i)
        if s.n_angles:
            s.ang_i, s.ang_j, s.ang_k = i(cfg.angle_i), i(cfg.angle_j), i(cfg.angle_k)
            s.ang_kt, s.ang_t0 = d(cfg.angle_k_theta), d(cfg.angle_theta0)
        s.n_dih = len(cfg.dihedral_i)
        if s.n_dih:
            s.dih_i, s.dih_j, s.dih_k, s.dih_l = (i(cfg.dihedral_i), i(cfg.dihedral_j),
                                                  i(cfg.dihedral_k), i(cfg.dihedral_l))
            s.dih_n, s.dih_kphi, s.dih_phi0 = (i(cfg.dihedral_periodicity), d(cfg.dihedral_k_phi),
                                               d(cfg.dihedral_phi0))
        s.n_imp = len(cfg.improper_i)
        if s.n_imp:
            s.imp_i, s.imp_j, s.imp_k, s.imp_l = (i(cfg.improper_i), i(cfg.improper_j),
                                                  i(cfg.improper_k), i(cfg.improper_l))
            s.imp_kphi, s.imp_phi0 = d(cfg.improper_k_phi), d(cfg.improper_phi0)
        s.profile = {"ref": 0, "phys": 1}[profile]
        self.s = s
        self._k = k


class Oracle:
    """FP64 CPU restatement of the reference's hot path (both profiles)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = C.CDLL(ORACLE_SO)
        vp = C.c_void_p
        sp = C.POINTER(orc_system)
        for name, res, args in [
            ("orc_min_image", None, [C.c_double] * 4 + [_dp]),
            ("orc_theta4", C.c_double, [C.c_double]),
            ("orc_dtheta4", C.c_double, [C.c_double]),
            ("orc_self_energy", C.c_double, [C.c_double, _dp, C.c_int, C.c_double]),
            ("orc_philox", None, [C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32]),
            ("orc_shake", C.c_int, [C.c_int, _ip, _ip, _dp, C.c_double, C.c_double, _dp, _dp, _dp,
                                    _dp]),
            ("orc_rattle", C.c_int, [C.c_int, _ip, _ip, C.c_double, C.c_double, _dp, _dp, _dp, _dp,
                                     _dp, _dp, _dp]),
            ("orc_rfft3", None, [C.c_int, _dp, _dp]),
            ("orc_pairs_build", vp, [C.c_int, _dp, _dp, _dp, C.c_double, C.c_double]),
            ("orc_pairs_count", C.c_long, [vp]),
            ("orc_pairs_copy", None, [vp, _ip, _ip]),
            ("orc_pairs_free", None, [vp]),
            ("orc_forces", None, [sp, _dp, _dp, _dp, _dp, _dp, _dp, C.POINTER(orc_energy)]),
            ("orc_component", None, [sp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            ("orc_engine_create", vp, [sp, C.POINTER(orc_run)]),
            ("orc_engine_step", None, [vp, C.c_int]),
            ("orc_engine_get", None, [vp, C.c_int, _dp, _dp, _dp]),
            ("orc_engine_scalars", None, [vp, _dp]),
            ("orc_engine_energy", None, [vp, C.POINTER(orc_energy)]),
            ("orc_engine_destroy", None, [vp]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L

    # -- distance constraints ------------------------------------------------
    def shake(self, pos, masses, ci, cj, dist, box, tol=1e-8):
        """Constraints::apply on a copy of pos; returns (positions, sweeps)."""
        x, y, z = (np.ascontiguousarray(pos[:, k], dtype=np.float64).copy() for k in range(3))
        i, pi = _i(ci)
        j, pj = _i(cj)
        d, pd = _d(dist)
        m, pm = _d(masses)
        it = self.L.orc_shake(len(i), pi, pj, pd, float(tol), float(box), pm, x.ctypes.data_as(_dp),
                              y.ctypes.data_as(_dp), z.ctypes.data_as(_dp))
        return np.stack([x, y, z], 1), it

    def rattle(self, pos, vel, masses, ci, cj, box, tol=1e-8):
        """Constraints::apply_rattle on a copy of vel; returns (velocities, sweeps)."""
        (x, y, z), (px, py, pz) = Ref._xyz(pos)
        vx, vy, vz = (np.ascontiguousarray(vel[:, k], dtype=np.float64).copy() for k in range(3))
        i, pi = _i(ci)
        j, pj = _i(cj)
        m, pm = _d(masses)
        it = self.L.orc_rattle(len(i), pi, pj, float(tol), float(box), pm, px, py, pz,
                               vx.ctypes.data_as(_dp), vy.ctypes.data_as(_dp), vz.ctypes.data_as(_dp))
        return np.stack([vx, vy, vz], 1), it

    # -- small functions ----------------------------------------------------
    def min_image(self, L, d):
        out = np.zeros(3)
        self.L.orc_min_image(L, d[0], d[1], d[2], out.ctypes.data_as(_dp))
        return out

    def theta4(self, u):
        return self.L.orc_theta4(u)

    def dtheta4(self, u):
        return self.L.orc_dtheta4(u)

    def self_energy(self, alpha, q, k_e=KE):
        a, p = _d(q)
        return self.L.orc_self_energy(alpha, p, len(a), k_e)

    def philox(self, ctr, key):
        c = (C.c_uint32 * 4)(*ctr)
        self.L.orc_philox(c, key & 0xFFFFFFFF, key >> 32)
        return list(c)

    def rfft3(self, real):
        K = real.shape[0]
        a, p = _d(real)
        out = np.zeros(K * K * (K // 2 + 1) * 2)
        self.L.orc_rfft3(K, p, out.ctypes.data_as(_dp))
        return out.view(np.complex128).reshape(K, K, K // 2 + 1)

    def pairs(self, pos, L, rc):
        """Sorted (i<j) pairs with minimum-image r < rc (reference expression)."""
        x, px = _d(pos[:, 0])
        y, py = _d(pos[:, 1])
        z, pz = _d(pos[:, 2])
        h = self.L.orc_pairs_build(len(x), px, py, pz, float(L), float(rc))
        n = self.L.orc_pairs_count(h)
        pi = np.empty(n, np.int32)
        pj = np.empty(n, np.int32)
        self.L.orc_pairs_copy(h, pi.ctypes.data_as(_ip), pj.ctypes.data_as(_ip))
        self.L.orc_pairs_free(h)
        return pi, pj

    # -- forces ---------------------------------------------------------------
    def forces(self, cfg, profile, pos=None, box=None):
        """(F[N,3], energy dict) of every component at pos (default: cfg positions)."""
        S = _Sys(cfg, profile)
        if box is not None:
            S.s.box = float(box)
        if pos is None:
            pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
        x, px = _d(pos[:, 0])
        y, py = _d(pos[:, 1])
        z, pz = _d(pos[:, 2])
        n = len(x)
        fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
        e = orc_energy()
        self.L.orc_forces(C.byref(S.s), px, py, pz, fx.ctypes.data_as(_dp), fy.ctypes.data_as(_dp),
                          fz.ctypes.data_as(_dp), C.byref(e))
        return np.stack([fx, fy, fz], 1), e.as_dict()

    def component(self, cfg, profile, which, pos=None, box=None):
        S = _Sys(cfg, profile)
        if box is not None:
            S.s.box = float(box)
        if pos is None:
            pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
        x, px = _d(pos[:, 0])
        y, py = _d(pos[:, 1])
        z, pz = _d(pos[:, 2])
        n = len(x)
        fx, fy, fz = np.zeros(n), np.zeros(n), np.zeros(n)
        e = C.c_double(0.0)
        v = C.c_double(0.0)
        self.L.orc_component(C.byref(S.s), which, px, py, pz, fx.ctypes.data_as(_dp),
                             fy.ctypes.data_as(_dp), fz.ctypes.data_as(_dp), C.byref(e), C.byref(v))
        return np.stack([fx, fy, fz], 1), e.value, v.value

    # -- engine ---------------------------------------------------------------
    def engine(self, cfg, profile, rng_seed=0x5EED, brute_list=False):
        return OracleEngine(self, cfg, profile, rng_seed, brute_list)


class OracleEngine:
    """The reference step sequence (SimulationEngine::step) in FP64 on the CPU."""

    def __init__(self, o: Oracle, cfg, profile, rng_seed, brute_list=False):
        self.o = o
        self.S = _Sys(cfg, profile)
        k = []

        def d(v):
            a, p = _d(v)
            k.append(a)
            return p

        r = orc_run()
        r.dt = cfg.dt
        r.mass = d(cfg.masses)
        r.x, r.y, r.z = d(cfg.pos_x), d(cfg.pos_y), d(cfg.pos_z)
        if len(cfg.vel_x):
            r.vx, r.vy, r.vz = d(cfg.vel_x), d(cfg.vel_y), d(cfg.vel_z)
        r.gen_vel = int(bool(cfg.gen_vel))
        r.seed = int(cfg.seed)
        r.init_temperature = cfg.init_temperature
        r.thermostat = THERMO[cfg.thermostat.type]
        r.t_temp, r.t_tau, r.t_freq = cfg.thermostat.temperature, cfg.thermostat.tau, cfg.thermostat.frequency
        r.barostat = BARO[cfg.barostat.type]
        if r.barostat == 2 and profile != "ref":
            raise ValueError("the Andersen barostat is restated for the ref profile only")
        r.b_pressure, r.b_tau, r.b_compress = cfg.barostat.pressure, cfg.barostat.tau, cfg.barostat.compressibility
        r.rng_seed = rng_seed
        r.brute_list = int(bool(brute_list))
        if cfg.constraint_type == "shake" and len(cfg.constraint_i):
            ci, pi = _i(cfg.constraint_i)
            cj, pj = _i(cfg.constraint_j)
            k.extend([ci, cj])
            r.n_cons, r.cons_i, r.cons_j = len(ci), pi, pj
            r.cons_dist, r.cons_tol = d(cfg.constraint_dist), float(cfg.constraint_tolerance)
        self.n = len(cfg.masses)
        self.h = o.L.orc_engine_create(C.byref(self.S.s), C.byref(r))
        self._k = k

    def step(self, n=1):
        self.o.L.orc_engine_step(self.h, int(n))

    def get(self, which):
        x, y, z = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        self.o.L.orc_engine_get(self.h, which, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                z.ctypes.data_as(_dp))
        return np.stack([x, y, z], 1)

    def scalars(self):
        out = np.zeros(8)
        self.o.L.orc_engine_scalars(self.h, out.ctypes.data_as(_dp))
        return dict(zip(["pe", "box", "time", "step", "lj_counter", "zeta", "ke", "andersen_calls"], out))

    def energy(self):
        e = orc_energy()
        self.o.L.orc_engine_energy(self.h, C.byref(e))
        return e.as_dict()

    def __del__(self):
        try:
            self.o.L.orc_engine_destroy(self.h)
        except Exception:
            pass


# ---- the reference's own classes -------------------------------------------------
class ref_run_desc(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int), ("box", C.c_double), ("mass", _dp), ("charge", _dp),
        ("x", _dp), ("y", _dp), ("z", _dp), ("vx", _dp), ("vy", _dp), ("vz", _dp), ("types", _ip),
        ("use_lj", C.c_int), ("n_types", C.c_int), ("lj_sigma", _dp), ("lj_eps", _dp),
        ("lj_cutoff", C.c_double),
        ("n_bonds", C.c_int), ("bond_i", _ip), ("bond_j", _ip), ("bond_k", _dp), ("bond_r0", _dp),
        ("n_angles", C.c_int), ("ang_i", _ip), ("ang_j", _ip), ("ang_k", _ip), ("ang_kt", _dp),
        ("ang_t0", _dp),
        ("n_dih", C.c_int), ("dih_i", _ip), ("dih_j", _ip), ("dih_k", _ip), ("dih_l", _ip),
        ("dih_n", _ip), ("dih_kphi", _dp), ("dih_phi0", _dp),
        ("n_imp", C.c_int), ("imp_i", _ip), ("imp_j", _ip), ("imp_k", _ip), ("imp_l", _ip),
        ("imp_kphi", _dp), ("imp_phi0", _dp),
        ("n_excl", C.c_int), ("excl_i", _ip), ("excl_j", _ip),
        ("coulomb_type", C.c_int), ("coul_cutoff", C.c_double), ("ewald", C.c_double),
        ("pme_spacing", C.c_double), ("pme_order", C.c_int),
        ("dt", C.c_double), ("thermostat", C.c_int), ("t_temp", C.c_double), ("t_tau", C.c_double),
        ("t_freq", C.c_double), ("barostat", C.c_int), ("b_pressure", C.c_double),
        ("b_tau", C.c_double), ("b_compress", C.c_double), ("gen_vel", C.c_int), ("seed", C.c_int),
        ("init_temperature", C.c_double),
        ("n_cons", C.c_int), ("cons_i", _ip), ("cons_j", _ip), ("cons_dist", _dp),
        ("cons_tol", C.c_double),
    ]


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class Ref:
    """The reference's own compiled classes (oracle/_ref/libdmdref.so)."""

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        L = C.CDLL(REF_SO)
        vp = C.c_void_p
        D = C.c_double
        sigs = {
            "ref_min_image": (None, [D, D, D, D, _dp]),
            "ref_wrap": (None, [D, _dp]),
            "ref_lj": (C.c_long, [C.c_int, _dp, _dp, _dp, D, _ip, C.c_int, _dp, _dp, D, _dp, _dp,
                                  _dp, _dp, _ip, _ip, C.c_long]),
            "ref_coulomb_direct": (None, [C.c_int, _dp, _dp, _dp, D, _dp, D, D, _dp, _dp, _dp, _dp]),
            "ref_exclusion": (None, [C.c_int, _dp, _dp, _dp, D, _dp, C.c_int, _ip, _ip, _dp, _dp, _dp, _dp]),
            "ref_pme": (None, [C.c_int, _dp, _dp, _dp, D, _dp, C.c_int, D, D, C.c_int, _dp, _dp, _dp, _dp]),
            "ref_bond": (None, [C.c_int, _dp, _dp, _dp, D, C.c_int, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp]),
            "ref_angle": (None, [C.c_int, _dp, _dp, _dp, D, C.c_int, _ip, _ip, _ip, _dp, _dp, _dp,
                                 _dp, _dp, _dp]),
            "ref_dihedral": (None, [C.c_int, _dp, _dp, _dp, D, C.c_int, _ip, _ip, _ip, _ip, _ip, _dp,
                                    _dp, _dp, _dp, _dp, _dp]),
            "ref_improper": (None, [C.c_int, _dp, _dp, _dp, D, C.c_int, _ip, _ip, _ip, _ip, _dp, _dp,
                                    _dp, _dp, _dp, _dp]),
            "ref_kinetic_energy": (D, [C.c_int, _dp, _dp, _dp, _dp]),
            "ref_shake": (None, [C.c_int, C.c_int, _ip, _ip, _dp, D, D, _dp, _dp, _dp, _dp]),
            "ref_rattle": (None, [C.c_int, C.c_int, _ip, _ip, _dp, D, D, _dp, _dp, _dp, _dp, _dp, _dp,
                                  _dp]),
            "ref_temperature": (D, [D, C.c_int]),
            "ref_engine_create": (vp, [C.POINTER(ref_run_desc)]),
            "ref_engine_step": (None, [vp, C.c_int]),
            "ref_engine_get": (None, [vp, C.c_int, _dp, _dp, _dp]),
            "ref_engine_scalars": (None, [vp, _dp]),
            "ref_engine_save_checkpoint": (None, [vp, C.c_char_p]),
            "ref_engine_destroy": (None, [vp]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L

    @staticmethod
    def _xyz(pos):
        x, px = _d(pos[:, 0])
        y, py = _d(pos[:, 1])
        z, pz = _d(pos[:, 2])
        return (x, y, z), (px, py, pz)

    def lj(self, cfg, pos=None, box=None):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        box = cfg.box_size if box is None else box
        keep, (px, py, pz) = self._xyz(pos)
        n = len(pos)
        f = np.zeros((3, n))
        e = C.c_double(0.0)
        t, pt = _i(cfg.atom_types if len(cfg.atom_types) else np.zeros(n, np.int32))
        s, ps = _d(cfg.lj_sigma)
        ep, pe = _d(cfg.lj_epsilon)
        cap = max(1, 400 * n)
        pi = np.empty(cap, np.int32)
        pj = np.empty(cap, np.int32)
        np_ = self.L.ref_lj(n, px, py, pz, box, pt, cfg.lj_n_types, ps, pe, cfg.lj_cutoff,
                            f[0].ctypes.data_as(_dp), f[1].ctypes.data_as(_dp),
                            f[2].ctypes.data_as(_dp), C.byref(e), pi.ctypes.data_as(_ip),
                            pj.ctypes.data_as(_ip), cap)
        assert np_ <= cap
        return f.T.copy(), e.value, (pi[:np_].copy(), pj[:np_].copy())

    def shake(self, pos, masses, ci, cj, dist, box, tol=1e-8):
        """The reference's Constraints::apply on a copy of pos."""
        x, y, z = (np.ascontiguousarray(pos[:, k], dtype=np.float64).copy() for k in range(3))
        i, pi = _i(ci)
        j, pj = _i(cj)
        d, pd = _d(dist)
        m, pm = _d(masses)
        self.L.ref_shake(len(x), len(i), pi, pj, pd, float(tol), float(box), pm,
                         x.ctypes.data_as(_dp), y.ctypes.data_as(_dp), z.ctypes.data_as(_dp))
        return np.stack([x, y, z], 1)

    def rattle(self, pos, vel, masses, ci, cj, dist, box, tol=1e-8):
        """The reference's Constraints::apply_rattle on a copy of vel."""
        (x, y, z), (px, py, pz) = self._xyz(pos)
        vx, vy, vz = (np.ascontiguousarray(vel[:, k], dtype=np.float64).copy() for k in range(3))
        i, pi = _i(ci)
        j, pj = _i(cj)
        d, pd = _d(dist)
        m, pm = _d(masses)
        self.L.ref_rattle(len(x), len(i), pi, pj, pd, float(tol), float(box), pm, px, py, pz,
                          vx.ctypes.data_as(_dp), vy.ctypes.data_as(_dp), vz.ctypes.data_as(_dp))
        return np.stack([vx, vy, vz], 1)

    def _bonded(self, fn, pos, box, n, *args):
        keep, (px, py, pz) = self._xyz(pos)
        f = np.zeros((3, n))
        e = C.c_double(0.0)
        fn(n, px, py, pz, box, *args, f[0].ctypes.data_as(_dp), f[1].ctypes.data_as(_dp),
           f[2].ctypes.data_as(_dp), C.byref(e))
        return f.T.copy(), e.value

    def bond(self, cfg, pos=None, box=None):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        a = [_i(cfg.bond_i), _i(cfg.bond_j), _d(cfg.bond_k), _d(cfg.bond_r0)]
        return self._bonded(self.L.ref_bond, pos, box or cfg.box_size, len(pos), len(cfg.bond_i),
                            *[p for _, p in a])

    def angle(self, cfg, pos=None, box=None):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        a = [_i(cfg.angle_i), _i(cfg.angle_j), _i(cfg.angle_k), _d(cfg.angle_k_theta),
             _d(cfg.angle_theta0)]
        return self._bonded(self.L.ref_angle, pos, box or cfg.box_size, len(pos), len(cfg.angle_i),
                            *[p for _, p in a])

    def dihedral(self, cfg, pos=None, box=None):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        a = [_i(cfg.dihedral_i), _i(cfg.dihedral_j), _i(cfg.dihedral_k), _i(cfg.dihedral_l),
             _i(cfg.dihedral_periodicity), _d(cfg.dihedral_k_phi), _d(cfg.dihedral_phi0)]
        return self._bonded(self.L.ref_dihedral, pos, box or cfg.box_size, len(pos),
                            len(cfg.dihedral_i), *[p for _, p in a])

    def improper(self, cfg, pos=None, box=None):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        a = [_i(cfg.improper_i), _i(cfg.improper_j), _i(cfg.improper_k), _i(cfg.improper_l),
             _d(cfg.improper_k_phi), _d(cfg.improper_phi0)]
        return self._bonded(self.L.ref_improper, pos, box or cfg.box_size, len(pos),
                            len(cfg.improper_i), *[p for _, p in a])

    def exclusion(self, cfg, pos=None, box=None):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        q = _d(cfg.charges)
        a = [_i(cfg.excl_i), _i(cfg.excl_j)]
        return self._bonded(self.L.ref_exclusion, pos, box or cfg.box_size, len(pos), q[1],
                            len(cfg.excl_i), *[p for _, p in a])

    def coulomb_direct(self, cfg, pos=None, box=None):
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        q = _d(cfg.charges)
        return self._bonded(self.L.ref_coulomb_direct, pos, box or cfg.box_size, len(pos), q[1],
                            cfg.coulomb_cutoff, cfg.ewald_coeff)

    def pme(self, cfg, pos=None, box=None):
        """CoulombPME::compute (reciprocal forces, reciprocal + self energy) on the
        mesh build_force_engine picks (K = max(8, int(L/spacing + 0.5)))."""
        pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1) if pos is None else pos
        q = _d(cfg.charges)
        box = box or cfg.box_size
        K = max(8, int(cfg.box_size / cfg.pme_grid_spacing + 0.5))
        return self._bonded(self.L.ref_pme, pos, box, len(pos), q[1], K, cfg.coulomb_cutoff,
                            cfg.ewald_coeff, int(cfg.pme_order))

    def engine(self, cfg):
        return RefEngine(self, cfg)


class RefEngine:
    """The reference's components stepped in SimulationEngine::step order."""

    def __init__(self, r: Ref, cfg):
        self.r = r
        k = []

        def d(v):
            a, p = _d(v)
            k.append(a)
            return p

        def i(v):
            a, p = _i(v)
            k.append(a)
            return p

        n = len(cfg.masses)
        s = ref_run_desc()
        s.n_atoms, s.box = n, cfg.box_size
        s.mass, s.charge = d(cfg.masses), d(cfg.charges if len(cfg.charges) else np.zeros(n))
        s.x, s.y, s.z = d(cfg.pos_x), d(cfg.pos_y), d(cfg.pos_z)
        if len(cfg.vel_x):
            s.vx, s.vy, s.vz = d(cfg.vel_x), d(cfg.vel_y), d(cfg.vel_z)
        if len(cfg.atom_types):
            s.types = i(cfg.atom_types)
        s.use_lj, s.n_types = int(bool(cfg.use_lj)), cfg.lj_n_types
        if s.n_types:
            s.lj_sigma, s.lj_eps = d(cfg.lj_sigma), d(cfg.lj_epsilon)
        s.lj_cutoff = cfg.lj_cutoff
        s.n_bonds = len(cfg.bond_i)
        if s.n_bonds:
            s.bond_i, s.bond_j, s.bond_k, s.bond_r0 = i(cfg.bond_i), i(cfg.bond_j), d(cfg.bond_k), d(cfg.bond_r0)
        s.n_angles = len(cfg.angle_i)
        if s.n_angles:
            s.ang_i, s.ang_j, s.ang_k = i(cfg.angle_i), i(cfg.angle_j), i(cfg.angle_k)
            s.ang_kt, s.ang_t0 = d(cfg.angle_k_theta), d(cfg.angle_theta0)
        s.n_dih = len(cfg.dihedral_i)
        if s.n_dih:
            s.dih_i, s.dih_j, s.dih_k, s.dih_l = (i(cfg.dihedral_i), i(cfg.dihedral_j),
                                                  i(cfg.dihedral_k), i(cfg.dihedral_l))
            s.dih_n, s.dih_kphi, s.dih_phi0 = (i(cfg.dihedral_periodicity), d(cfg.dihedral_k_phi),
                                               d(cfg.dihedral_phi0))
        s.n_imp = len(cfg.improper_i)
        if s.n_imp:
            s.imp_i, s.imp_j, s.imp_k, s.imp_l = (i(cfg.improper_i), i(cfg.improper_j),
                                                  i(cfg.improper_k), i(cfg.improper_l))
            s.imp_kphi, s.imp_phi0 = d(cfg.improper_k_phi), d(cfg.improper_phi0)
        s.n_excl = len(cfg.excl_i)
        if s.n_excl:
            s.excl_i, s.excl_j = i(cfg.excl_i), i(cfg.excl_j)
        s.coulomb_type = 1 if cfg.coulomb_type == "pme" else 0
        s.coul_cutoff, s.ewald = cfg.coulomb_cutoff, cfg.ewald_coeff
        s.pme_spacing, s.pme_order = cfg.pme_grid_spacing, int(cfg.pme_order)
        s.dt = cfg.dt
        s.thermostat = THERMO[cfg.thermostat.type]
        s.t_temp, s.t_tau, s.t_freq = cfg.thermostat.temperature, cfg.thermostat.tau, cfg.thermostat.frequency
        s.barostat = BARO[cfg.barostat.type]
        s.b_pressure, s.b_tau, s.b_compress = cfg.barostat.pressure, cfg.barostat.tau, cfg.barostat.compressibility
        s.gen_vel, s.seed, s.init_temperature = int(bool(cfg.gen_vel)), int(cfg.seed), cfg.init_temperature
        if cfg.constraint_type == "shake" and len(cfg.constraint_i):
            s.n_cons, s.cons_i, s.cons_j = len(cfg.constraint_i), i(cfg.constraint_i), i(cfg.constraint_j)
            s.cons_dist, s.cons_tol = d(cfg.constraint_dist), float(cfg.constraint_tolerance)
        self.n = n
        self.h = r.L.ref_engine_create(C.byref(s))
        self._k = k

    def step(self, n=1):
        self.r.L.ref_engine_step(self.h, int(n))

    def get(self, which):
        x, y, z = np.empty(self.n), np.empty(self.n), np.empty(self.n)
        self.r.L.ref_engine_get(self.h, which, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                z.ctypes.data_as(_dp))
        return np.stack([x, y, z], 1)

    def scalars(self):
        out = np.zeros(6)
        self.r.L.ref_engine_scalars(self.h, out.ctypes.data_as(_dp))
        return dict(zip(["pe", "box", "time", "step", "lj_counter", "zeta"], out))

    def save_checkpoint(self, path):
        self.r.L.ref_engine_save_checkpoint(self.h, path.encode())

    def __del__(self):
        try:
            self.r.L.ref_engine_destroy(self.h)
        except Exception:
            pass
