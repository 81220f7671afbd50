"""C-ABI library checks that need no GPU: it loads and exports every symbol
that include/dmdgpu.h declares; host-side config handling mirrors the reference."""
import ctypes
import json
import os

import numpy as np
import pytest

from dmd_b200 import _capi, config, workloads
from dmd_b200.core import SimulationConfig
from dmd_b200.system import SystemBuilder


@pytest.fixture(scope="module")
def lib_path():
    from dmd_b200 import build
    return build.build()


def test_library_exports_header_symbols(lib_path):
    lib = ctypes.CDLL(lib_path)
    for name in _capi.exported_symbols():
        assert hasattr(lib, name), name
    L = _capi.lib()
    assert L.dmdgpu_last_error(None) == b"null context"


def test_struct_layout_matches_header(tmp_path):
    """Every field offset of the ctypes mirrors equals the C compiler's offsetof."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dmdgpu.h"', "int main(void){"]
    for cls in (_capi.dmdgpu_system, _capi.dmdgpu_options, _capi.dmdgpu_scalars, _capi.dmdgpu_timing):
        lines.append(f'printf("%zu\\n", sizeof({cls.__name__}));')
        for f in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({cls.__name__}, {f[0]}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for cls in (_capi.dmdgpu_system, _capi.dmdgpu_options, _capi.dmdgpu_scalars, _capi.dmdgpu_timing):
        want.append(ctypes.sizeof(cls))
        want.extend(getattr(cls, f[0]).offset for f in cls._fields_)
    assert got == want


def test_validate_config_errors():
    good = json.loads(config.generate_config_template())
    config.validate_config(good)
    bad = json.loads(json.dumps(good))
    del bad["run"]["dt"]
    with pytest.raises(ValueError, match="Missing required key 'run.dt'"):
        config.validate_config(bad)
    bad = json.loads(json.dumps(good))
    bad["extra"] = {}
    with pytest.raises(ValueError, match="Unknown section 'extra'"):
        config.validate_config(bad)
    bad = json.loads(json.dumps(good))
    bad["run"]["dt"] = "x"
    with pytest.raises(ValueError, match="Type mismatch"):
        config.validate_config(bad)


def test_system_builder_matches_workload_config():
    w = workloads.water_box(n_mol=27, box=1.0, seed=1, spacing=0.1)
    sys_json, cfg_json = w.to_json()
    b = SystemBuilder(sys_json).apply_config_json(cfg_json).build()
    c = w.config()
    for k in ("masses", "charges", "pos_x", "atom_types", "lj_sigma", "lj_epsilon", "bond_i",
              "bond_r0", "angle_k", "angle_theta0"):
        assert np.array_equal(getattr(b, k), getattr(c, k)), k
    assert b.excl_i == c.excl_i and b.lj_n_types == 2
    assert b.coulomb_type == "pme" and b.thermostat.type == "nose-hoover" and b.use_lj


def test_system_desc_rejects_unknown_thermostat():
    c = workloads.argon_fcc(n_cells=2).config()
    c.thermostat.type = "langevin"
    with pytest.raises(RuntimeError, match="Unknown thermostat type"):
        _capi.SystemDesc(c)
