"""ctypes binding of include/dmdgpu.h (the library's C ABI).

The shared library is built in-tree (dmd_b200/libdmdgpu.so, see
dmd_b200/build.py).  There is no fallback: if the library cannot be loaded
the import of the engine fails with the loader's message.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdmdgpu.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

OK = 0
ERR_NAMES = {
    1: "NaN", 2: "BondExplosion", 3: "Mismatch", 4: "ParmError", 5: "GPUError",
    6: "OOM", 7: "Budget", 8: "Invalid", 9: "Capacity",
}

PROFILES = {"ref": 0, "phys": 1}
PRECISIONS = {"mixed": 0, "fp64": 1}
COULOMB = {"cutoff": 0, "direct": 0, "pme": 1}
THERMO = {"none": 0, "berendsen": 1, "nose-hoover": 2, "andersen": 3}
BARO = {"none": 0, "berendsen": 1, "andersen": 2}
E_TERMS = ("lj", "coul_real", "coul_recip", "coul_self", "coul_excl", "bond", "angle", "dihedral",
           "improper")


class dmdgpu_system(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32), ("box_size", C.c_double),
        ("masses", _dp), ("charges", _dp),
        ("pos_x", _dp), ("pos_y", _dp), ("pos_z", _dp),
        ("vel_x", _dp), ("vel_y", _dp), ("vel_z", _dp),
        ("atom_types", _ip),
        ("use_lj", C.c_int32), ("lj_n_types", C.c_int32),
        ("lj_sigma", _dp), ("lj_epsilon", _dp), ("lj_cutoff", C.c_double),
        ("n_bonds", C.c_int32), ("bond_i", _ip), ("bond_j", _ip), ("bond_k", _dp), ("bond_r0", _dp),
        ("n_angles", C.c_int32), ("angle_i", _ip), ("angle_j", _ip), ("angle_k", _ip),
        ("angle_k_theta", _dp), ("angle_theta0", _dp),
        ("n_dihedrals", C.c_int32), ("dihedral_i", _ip), ("dihedral_j", _ip), ("dihedral_k", _ip),
        ("dihedral_l", _ip), ("dihedral_periodicity", _ip), ("dihedral_k_phi", _dp),
        ("dihedral_phi0", _dp),
        ("n_impropers", C.c_int32), ("improper_i", _ip), ("improper_j", _ip), ("improper_k", _ip),
        ("improper_l", _ip), ("improper_k_phi", _dp), ("improper_phi0", _dp),
        ("coulomb_type", C.c_int32), ("coulomb_cutoff", C.c_double), ("ewald_coeff", C.c_double),
        ("pme_grid_spacing", C.c_double), ("pme_order", C.c_int32),
        ("n_excl", C.c_int32), ("excl_i", _ip), ("excl_j", _ip),
        ("dt", C.c_double), ("n_steps", C.c_int32), ("gen_vel", C.c_int32), ("seed", C.c_int32),
        ("init_temperature", C.c_double),
        ("thermostat_type", C.c_int32), ("thermo_temperature", C.c_double),
        ("thermo_tau", C.c_double), ("thermo_frequency", C.c_double),
        ("barostat_type", C.c_int32), ("baro_pressure", C.c_double), ("baro_tau", C.c_double),
        ("baro_compressibility", C.c_double),
        ("constraint_type", C.c_int32), ("checkpoint_interval", C.c_int32),
        ("checkpoint_path", C.c_char_p),
        ("n_constraints", C.c_int32), ("constraint_i", _ip), ("constraint_j", _ip),
        ("constraint_dist", _dp), ("constraint_tolerance", C.c_double),
    ]


class dmdgpu_options(C.Structure):
    _fields_ = [("profile", C.c_int32), ("precision", C.c_int32), ("skin", C.c_double),
                ("device", C.c_int32), ("rng_seed", C.c_uint64), ("nb_form", C.c_int32)]


NB_FORMS = {"auto": 0, "chunk32": 1, "cluster8": 2}


def launch_info_dict(info) -> dict:
    """dmdgpu_launch_info as a plain dict (form by name)."""
    names = {v: k for k, v in NB_FORMS.items()}
    return {"packed": bool(info.packed), "nb_form": names.get(info.nb_form, "none"),
            "nb_blocks_per_sm": int(info.nb_blocks_per_sm), "tuned": bool(info.tuned),
            "min_image_kernel": bool(info.min_image_kernel), "n_replicas": int(info.n_replicas),
            "n_atoms": int(info.n_atoms), "launches_per_step": int(info.launches_per_step)}


class dmdgpu_frame(C.Structure):
    _fields_ = [("step", C.c_int64), ("time", C.c_double), ("box", C.c_double), ("n_atoms", C.c_int32),
                ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)), ("z", C.POINTER(C.c_double)),
                ("vx", C.POINTER(C.c_double)), ("vy", C.POINTER(C.c_double)), ("vz", C.POINTER(C.c_double))]


FRAME_FN = C.CFUNCTYPE(None, C.POINTER(dmdgpu_frame), C.c_void_p)


class dmdgpu_timing(C.Structure):
    _fields_ = [("step_ms", C.c_double), ("nonbonded_ms", C.c_double), ("pme_ms", C.c_double),
                ("nonbonded_launches", C.c_int64), ("kernel_launches", C.c_int64),
                ("sampled_steps", C.c_int64)]


class dmdgpu_launch_info(C.Structure):
    _fields_ = [("packed", C.c_int32), ("nb_form", C.c_int32), ("nb_blocks_per_sm", C.c_int32),
                ("tuned", C.c_int32), ("min_image_kernel", C.c_int32), ("n_replicas", C.c_int32),
                ("n_atoms", C.c_int64), ("launches_per_step", C.c_int64)]


class dmdgpu_scalars(C.Structure):
    _fields_ = [("step", C.c_int64), ("time", C.c_double), ("potential_energy", C.c_double),
                ("box", C.c_double), ("kinetic_energy", C.c_double), ("temperature", C.c_double),
                ("pressure", C.c_double), ("virial", C.c_double), ("zeta", C.c_double),
                ("e_terms", C.c_double * 9), ("list_builds", C.c_int64),
                ("lj_step_since_rebuild", C.c_int32), ("status", C.c_int32),
                ("list_chunks", C.c_int64)]


_lib = None


def lib() -> C.CDLL:
    """Load libdmdgpu.so (raises OSError if it is missing or does not load)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not built: run `python -m dmd_b200.build` "
                      "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "dmdgpu_create": (C.c_int, [C.POINTER(dmdgpu_system), C.POINTER(dmdgpu_options), C.POINTER(vp)]),
        "dmdgpu_step": (C.c_int, [vp, C.c_int32]),
        "dmdgpu_repack": (C.c_int, [vp]),
        "dmdgpu_run": (C.c_int, [vp]),
        "dmdgpu_get_state": (C.c_int, [vp, C.c_int32, _dp, _dp, _dp]),
        "dmdgpu_set_state": (C.c_int, [vp, C.c_int32, _dp, _dp, _dp]),
        "dmdgpu_get_scalars": (C.c_int, [vp, C.POINTER(dmdgpu_scalars)]),
        "dmdgpu_compute_forces": (C.c_int, [vp, _dp, _dp, _dp, _dp]),
        "dmdgpu_component_compute": (C.c_int, [vp, C.c_int32, _dp, _dp, _dp, C.c_double,
                                               _dp, _dp, _dp, _dp]),
        "dmdgpu_pair_list": (C.c_int, [vp, _ip, _ip, C.c_int64, C.POINTER(C.c_int64)]),
        "dmdgpu_save_checkpoint": (C.c_int, [vp, C.c_char_p]),
        "dmdgpu_load_checkpoint": (C.c_int, [vp, C.c_char_p]),
        "dmdgpu_footprint_bytes": (C.c_int64, [C.POINTER(dmdgpu_system), C.POINTER(dmdgpu_options)]),
        "dmdgpu_kernel_launches": (C.c_int64, [vp]),
        "dmdgpu_stream": (C.c_void_p, [vp]),
        "dmdgpu_get_launch_info": (C.c_int, [vp, C.POINTER(dmdgpu_launch_info)]),
        "dmdgpu_step_timed": (C.c_int, [vp, C.c_int32, C.c_int64, C.POINTER(dmdgpu_timing)]),
        "dmdgpu_test_inject": (C.c_int, [vp, C.c_int32]),
        "dmdgpu_set_frame_writer": (C.c_int, [vp, C.c_int32, FRAME_FN, vp]),
        "dmdgpu_flush_frames": (C.c_int, [vp]),
        "dmdgpu_last_error": (C.c_char_p, [vp]),
        "dmdgpu_destroy": (None, [vp]),
        "dmdgpu_batch_create": (C.c_int, [C.c_int64, C.POINTER(dmdgpu_options), C.POINTER(vp)]),
        "dmdgpu_batch_admit": (C.c_int, [vp, C.POINTER(dmdgpu_system), C.c_int64, C.POINTER(C.c_int32)]),
        "dmdgpu_batch_step": (C.c_int, [vp, C.c_int32]),
        "dmdgpu_batch_step_timed": (C.c_int, [vp, C.c_int32, C.c_int64, C.POINTER(dmdgpu_timing)]),
        "dmdgpu_batch_poll": (C.c_int, [vp, _ip, C.c_int32, C.POINTER(C.c_int32)]),
        "dmdgpu_batch_get_state": (C.c_int, [vp, C.c_int32, C.c_int32, _dp, _dp, _dp]),
        "dmdgpu_batch_get_scalars": (C.c_int, [vp, C.c_int32, C.POINTER(dmdgpu_scalars)]),
        "dmdgpu_batch_release": (C.c_int, [vp, C.c_int32]),
        "dmdgpu_batch_used_bytes": (C.c_int64, [vp]),
        "dmdgpu_batch_get_launch_info": (C.c_int, [vp, C.POINTER(dmdgpu_launch_info)]),
        "dmdgpu_batch_active": (C.c_int32, [vp]),
        "dmdgpu_batch_last_error": (C.c_char_p, [vp]),
        "dmdgpu_batch_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names declared in include/dmdgpu.h (parsed from the header)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "dmdgpu.h")
    txt = open(hdr).read()
    return sorted(set(re.findall(r"\b(dmdgpu_[a-z_0-9]+)\s*\(", txt)))


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


class SystemDesc:
    """A dmdgpu_system filled from a SimulationConfig, with its arrays kept alive."""

    def __init__(self, cfg):
        n = len(cfg.masses)
        keep = []

        def d(v, size=None):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
            if size is not None and a.size != size:
                raise ValueError(f"array of size {a.size}, expected {size}")
            keep.append(a)
            return dptr(a)

        def i(v, size=None):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.int32))
            if size is not None and a.size != size:
                raise ValueError(f"array of size {a.size}, expected {size}")
            keep.append(a)
            return iptr(a)

        s = dmdgpu_system()
        s.n_atoms = n
        s.box_size = float(cfg.box_size)
        s.masses = d(cfg.masses, n)
        s.charges = d(cfg.charges if len(cfg.charges) else np.zeros(n), n)
        s.pos_x, s.pos_y, s.pos_z = d(cfg.pos_x, n), d(cfg.pos_y, n), d(cfg.pos_z, n)
        if len(cfg.vel_x):
            s.vel_x, s.vel_y, s.vel_z = d(cfg.vel_x, n), d(cfg.vel_y, n), d(cfg.vel_z, n)
        if len(cfg.atom_types):
            s.atom_types = i(cfg.atom_types, n)
        s.use_lj = int(bool(cfg.use_lj))
        nt = int(cfg.lj_n_types)
        s.lj_n_types = nt
        if nt:
            s.lj_sigma, s.lj_epsilon = d(cfg.lj_sigma, nt * nt), d(cfg.lj_epsilon, nt * nt)
        s.lj_cutoff = float(cfg.lj_cutoff)
        nb = len(cfg.bond_i)
        s.n_bonds = nb
        if nb:
            s.bond_i, s.bond_j = i(cfg.bond_i, nb), i(cfg.bond_j, nb)
            s.bond_k, s.bond_r0 = d(cfg.bond_k, nb), d(cfg.bond_r0, nb)
        na = len(cfg.angle_i)
        s.n_angles = na
        if na:
            s.angle_i, s.angle_j, s.angle_k = i(cfg.angle_i, na), i(cfg.angle_j, na), i(cfg.angle_k, na)
            s.angle_k_theta, s.angle_theta0 = d(cfg.angle_k_theta, na), d(cfg.angle_theta0, na)
        nd = len(cfg.dihedral_i)
        s.n_dihedrals = nd
        if nd:
            s.dihedral_i, s.dihedral_j = i(cfg.dihedral_i, nd), i(cfg.dihedral_j, nd)
            s.dihedral_k, s.dihedral_l = i(cfg.dihedral_k, nd), i(cfg.dihedral_l, nd)
            s.dihedral_periodicity = i(cfg.dihedral_periodicity, nd)
            s.dihedral_k_phi, s.dihedral_phi0 = d(cfg.dihedral_k_phi, nd), d(cfg.dihedral_phi0, nd)
        ni = len(cfg.improper_i)
        s.n_impropers = ni
        if ni:
            s.improper_i, s.improper_j = i(cfg.improper_i, ni), i(cfg.improper_j, ni)
            s.improper_k, s.improper_l = i(cfg.improper_k, ni), i(cfg.improper_l, ni)
            s.improper_k_phi, s.improper_phi0 = d(cfg.improper_k_phi, ni), d(cfg.improper_phi0, ni)
        if cfg.coulomb_type not in COULOMB:
            raise ValueError(f"unknown coulomb_type {cfg.coulomb_type!r}")
        s.coulomb_type = COULOMB[cfg.coulomb_type]
        s.coulomb_cutoff = float(cfg.coulomb_cutoff)
        s.ewald_coeff = float(cfg.ewald_coeff)
        s.pme_grid_spacing = float(cfg.pme_grid_spacing)
        s.pme_order = int(cfg.pme_order)
        ne = len(cfg.excl_i)
        s.n_excl = ne
        if ne:
            s.excl_i, s.excl_j = i(cfg.excl_i, ne), i(cfg.excl_j, ne)
        s.dt = float(cfg.dt)
        s.n_steps = int(cfg.n_steps)
        s.gen_vel = int(bool(cfg.gen_vel))
        s.seed = int(cfg.seed)
        s.init_temperature = float(cfg.init_temperature)
        t = cfg.thermostat
        if t.type not in THERMO:
            raise RuntimeError("Unknown thermostat type: " + t.type)
        s.thermostat_type = THERMO[t.type]
        s.thermo_temperature, s.thermo_tau, s.thermo_frequency = t.temperature, t.tau, t.frequency
        b = cfg.barostat
        if b.type not in BARO:
            raise RuntimeError("Unknown barostat type: " + b.type)
        s.barostat_type = BARO[b.type]
        s.baro_pressure, s.baro_tau, s.baro_compressibility = b.pressure, b.tau, b.compressibility
        s.constraint_type = 0 if cfg.constraint_type == "none" or not len(cfg.constraint_i) else 1
        if s.constraint_type:
            nc = len(cfg.constraint_i)
            s.n_constraints = nc
            s.constraint_i, s.constraint_j = i(cfg.constraint_i, nc), i(cfg.constraint_j, nc)
            s.constraint_dist = d(cfg.constraint_dist, nc)
            s.constraint_tolerance = float(cfg.constraint_tolerance)
        s.checkpoint_interval = int(cfg.checkpoint_interval)
        p = (cfg.checkpoint_path or "").encode()
        keep.append(p)
        s.checkpoint_path = p if p else None
        self.s = s
        self._keep = keep
