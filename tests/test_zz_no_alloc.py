"""dmdgpu_nonbonded_noalloc: the non-bonded evaluation for callers that cannot
allocate device memory (device memory owned by another allocator or a fixed
arena, no per-call allocation latency or allocation failure allowed).

It must give what the allocating entry point dmdgpu_component_compute gives
for the Lennard-Jones and real-space Coulomb components, within the tolerance
used by the other parity tests, on two calls in a row (the static scratch array
keeps the previous call's contents, so the second call checks that everything
that must start at zero is cleared), and what the FP64 oracle gives for the
same two components.  Its documented error paths are exercised too.  Collected
last on purpose."""
import ctypes as C

import numpy as np
import pytest

from dmd_b200 import _capi
from dmd_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "mixed": 1e-5}


class nb_params(C.Structure):
    _fields_ = [("n_atoms", C.c_int32), ("box", C.c_double), ("n_types", C.c_int32),
                ("lj_sigma", C.POINTER(C.c_double)), ("lj_epsilon", C.POINTER(C.c_double)),
                ("lj_cutoff", C.c_double), ("coul_cutoff", C.c_double), ("ewald_coeff", C.c_double),
                ("n_excl", C.c_int32), ("excl_i", C.POINTER(C.c_int32)),
                ("excl_j", C.POINTER(C.c_int32)), ("profile", C.c_int32), ("precision", C.c_int32),
                ("skin", C.c_double)]


def _noalloc(cfg, pos, profile, precision, types=None, expect=0):
    import torch
    L = _capi.lib()
    f = L.dmdgpu_nonbonded_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(nb_params)] + [C.c_void_p] * 10
    sig = np.ascontiguousarray(cfg.lj_sigma, dtype=np.float64)
    eps = np.ascontiguousarray(cfg.lj_epsilon, dtype=np.float64)
    ei = np.ascontiguousarray(cfg.excl_i, dtype=np.int32)
    ej = np.ascontiguousarray(cfg.excl_j, dtype=np.int32)
    p = nb_params(len(cfg.masses), cfg.box_size, cfg.lj_n_types, _capi.dptr(sig), _capi.dptr(eps),
                  cfg.lj_cutoff, cfg.coulomb_cutoff, cfg.ewald_coeff, len(ei), _capi.iptr(ei),
                  _capi.iptr(ej), _capi.PROFILES[profile], _capi.PRECISIONS[precision], 0.1)
    dev = torch.device("cuda:0")
    x, y, z = (torch.tensor(np.ascontiguousarray(pos[:, k]), dtype=torch.float64, device=dev) for k in range(3))
    q = torch.tensor(cfg.charges, dtype=torch.float64, device=dev)
    t = torch.tensor(cfg.atom_types if types is None else types, dtype=torch.int32, device=dev)
    fx, fy, fz = (torch.full((len(q),), 7.0, dtype=torch.float64, device=dev) for _ in range(3))
    en = torch.zeros(2, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = f(C.byref(p), x.data_ptr(), y.data_ptr(), z.data_ptr(), q.data_ptr(), t.data_ptr(),
           fx.data_ptr(), fy.data_ptr(), fz.data_ptr(), en.data_ptr(), None)
    assert rc == expect, rc
    if rc:
        return None, None
    F = torch.stack([fx, fy, fz], 1).cpu().numpy()
    return F, float(en.sum().item())


def _reference_entry(cfg, pos, profile, precision):
    from dmd_b200.core import Engine
    eng = Engine(cfg, precision=precision, profile=profile)
    f, e = eng.component_compute(0, pos, cfg.box_size)
    f, e = eng.component_compute(4, pos, cfg.box_size, forces=f, energy=e)
    eng.close()
    return f, e


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("profile", ["phys", "ref"])
def test_noalloc_matches_component_compute(oracle, profile, precision):
    n_mol = 1500
    box = (n_mol / 33.43) ** (1 / 3)
    cfg = W.water_box(n_mol=n_mol, box=box, seed=21, spacing=0.1).config()
    rng = np.random.default_rng(3)
    pos0 = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
    for call in range(2):  # two calls in a row on different coordinates
        pos = pos0 + rng.normal(0, 0.01, pos0.shape)
        F, e = _noalloc(cfg, pos, profile, precision)
        F_r, e_r = _reference_entry(cfg, pos, profile, precision)
        err = np.linalg.norm(F - F_r) / np.linalg.norm(F_r)
        assert err < TOL[precision], (call, err)
        assert abs(e - e_r) <= TOL[precision] * max(abs(e_r), 1.0), (call, e, e_r)
        # and the FP64 oracle's Lennard-Jones + real-space Coulomb components
        f0, e0, _ = oracle.component(cfg, profile, 0, pos=pos)
        f4, e4, _ = oracle.component(cfg, profile, 4, pos=pos)
        err_o = np.linalg.norm(F - (f0 + f4)) / np.linalg.norm(f0 + f4)
        assert err_o < TOL[precision], (call, err_o)
        assert abs(e - (e0 + e4)) <= TOL[precision] * max(abs(e0 + e4), 1.0) * 10, (call, e, e0 + e4)


def test_noalloc_rejects_oversize():
    import torch
    L = _capi.lib()
    f = L.dmdgpu_nonbonded_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(nb_params)] + [C.c_void_p] * 10
    sig = np.ones(1)
    eps = np.ones(1)
    p = nb_params(8193, 10.0, 1, _capi.dptr(sig), _capi.dptr(eps), 1.0, 1.0, 3.0, 0, None, None, 1, 0, 0.1)
    buf = torch.zeros(8193 * 8, dtype=torch.float64, device="cuda:0")
    ptr = buf.data_ptr()
    rc = f(C.byref(p), ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, None, None)
    assert rc == 4  # DMDGPU_ERR_PARM: more atoms than the static maximum


def test_noalloc_rejects_bad_type():
    """An atom type outside [0, n_types) is reported (and never indexes the LJ
    table)."""
    cfg = W.water_box(n_mol=300, box=(300 / 33.43) ** (1 / 3), seed=5, spacing=0.1).config()
    pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
    types = np.asarray(cfg.atom_types, np.int32).copy()
    types[11] = cfg.lj_n_types
    _noalloc(cfg, pos, "phys", "mixed", types=types, expect=4)  # DMDGPU_ERR_PARM


def test_noalloc_reports_list_overflow():
    """A pair list longer than the static chunk maximum is reported as
    DMDGPU_ERR_CAPACITY (no chunk is written past the maximum): 8,190 atoms of
    water with a 2.0 nm cutoff need more than 16,384 chunks."""
    n_mol = 2730
    cfg = W.water_box(n_mol=n_mol, box=(n_mol / 33.43) ** (1 / 3), seed=6, spacing=0.1).config()
    cfg.lj_cutoff = 2.0
    cfg.coulomb_cutoff = 2.0
    pos = np.stack([cfg.pos_x, cfg.pos_y, cfg.pos_z], 1)
    _noalloc(cfg, pos, "ref", "mixed", expect=9)
    # the array is still usable afterwards: a normal call succeeds
    small = W.water_box(n_mol=300, box=(300 / 33.43) ** (1 / 3), seed=5, spacing=0.1).config()
    pos_s = np.stack([small.pos_x, small.pos_y, small.pos_z], 1)
    F, _ = _noalloc(small, pos_s, "phys", "mixed")
    assert np.all(np.isfinite(F))
