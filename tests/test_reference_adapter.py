"""include/dmdgpu_reference.hpp -- the adapters a maintainer adds to the
reference's C++ tree (GpuForceComponent, GpuSimulationEngine, SystemView).

CPU: the header compiles against the reference's own headers
(src/force/force_component.h, src/sim/simulation_config.h, src/core/cell.h,
src/core/error.h) when the reference tree is present.
GPU: its GpuForceComponent, called through the ForceComponent interface,
gives what the reference's own LennardJones / HarmonicBond / HarmonicAngle /
PeriodicDihedral classes give on the same system (REF profile; FP64 1e-9,
mixed 1e-5 relative RMS force and energy, as the other parity tests).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from dmd_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPT_SO = os.path.join(ROOT, "oracle", "_ref", "libdmdadapt.so")
REF_TREE = os.path.join(os.path.dirname(ROOT), "reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_TREE, "src")), reason="reference tree not present")
def test_adapter_header_compiles_against_reference_headers(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text('#include "dmdgpu_reference.hpp"\n'
                   "int main() { return sizeof(dmdgpu_ref::GpuForceComponent) > 0 ? 0 : 1; }\n")
    subprocess.run(["g++", "-std=c++20", "-fsyntax-only", "-Wall", "-I", os.path.join(REF_TREE, "src"),
                    "-I", os.path.join(ROOT, "include"), str(src)], check=True)


def _arr(a, t):
    a = np.ascontiguousarray(np.asarray(a, dtype=t))
    return a, a.ctypes.data_as(C.POINTER(C.c_double if t == np.float64 else C.c_int32))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("system", ["water", "decane"])
def test_gpu_force_component_matches_reference_components(system, precision):
    if not os.path.exists(ADAPT_SO):
        pytest.skip("oracle/_ref/libdmdadapt.so not built (needs the reference tree at build time)")
    from dmd_b200 import _capi
    _capi.lib()  # libdmdgpu.so first, so the adapter resolves to this build
    L = C.CDLL(ADAPT_SO)
    rng = np.random.default_rng(4)
    if system == "water":
        c = W.water_box(n_mol=200, box=(200 / 33.43) ** (1 / 3), seed=3, spacing=0.1).config()
    else:
        c = W.decane_melt(20, 5).config()
    n = len(c.masses)
    pos = np.stack([c.pos_x, c.pos_y, c.pos_z], 1) + rng.normal(0, 0.003, (n, 3))
    keep = []

    def d(v):
        a, p = _arr(v, np.float64)
        keep.append(a)
        return p

    def i(v):
        a, p = _arr(v, np.int32)
        keep.append(a)
        return p

    f_ref = np.zeros((4, 3, n))
    f_gpu = np.zeros((4, 3, n))
    e_ref = np.zeros(4)
    e_gpu = np.zeros(4)
    err = C.create_string_buffer(512)
    nd = len(c.dihedral_i)
    rc = L.adapter_check(
        C.c_int(n), C.c_double(c.box_size), d(c.masses), d(c.charges), d(pos[:, 0]), d(pos[:, 1]),
        d(pos[:, 2]), i(c.atom_types), C.c_int(c.lj_n_types), d(c.lj_sigma), d(c.lj_epsilon),
        C.c_double(c.lj_cutoff), C.c_int(len(c.bond_i)), i(c.bond_i), i(c.bond_j), d(c.bond_k),
        d(c.bond_r0), C.c_int(len(c.angle_i)), i(c.angle_i), i(c.angle_j), i(c.angle_k),
        d(c.angle_k_theta), d(c.angle_theta0), C.c_int(nd), i(c.dihedral_i), i(c.dihedral_j),
        i(c.dihedral_k), i(c.dihedral_l), i(c.dihedral_periodicity), d(c.dihedral_k_phi),
        d(c.dihedral_phi0), C.c_int(_capi.PRECISIONS[precision]),
        f_ref.ctypes.data_as(C.POINTER(C.c_double)), e_ref.ctypes.data_as(C.POINTER(C.c_double)),
        f_gpu.ctypes.data_as(C.POINTER(C.c_double)), e_gpu.ctypes.data_as(C.POINTER(C.c_double)),
        err, C.c_int(512))
    assert rc == 0, err.value.decode()
    tol = {"fp64": 1e-9, "mixed": 1e-5}[precision]
    for k, name in enumerate(("lj", "bond", "angle", "dihedral")):
        if not np.any(f_ref[k]) and e_ref[k] == 0.0:
            assert np.abs(f_gpu[k]).max() < 1e-6 and abs(e_gpu[k]) < 1e-6, name
            continue
        err_f = np.linalg.norm(f_gpu[k] - f_ref[k]) / np.linalg.norm(f_ref[k])
        assert err_f < tol, (name, err_f)
        assert abs(e_gpu[k] - e_ref[k]) <= tol * max(abs(e_ref[k]), 1.0) * 10, (name, e_gpu[k], e_ref[k])
