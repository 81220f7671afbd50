"""C-ABI library checks that need no GPU: it loads and exports every symbol
that include/dmdgpu.h declares; the input reader accepts the reference's
system.json / config.json formats and refuses malformed documents."""
import ctypes
import json
import os

import numpy as np
import pytest

from dmd_b200 import _capi, workloads
from dmd_b200.core import SimulationConfig
from dmd_b200.inputs import InputError, check_config, load_inputs


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
    for cls in (_capi.dmdgpu_system, _capi.dmdgpu_options, _capi.dmdgpu_scalars, _capi.dmdgpu_timing,
                _capi.dmdgpu_frame):
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
    for cls in (_capi.dmdgpu_system, _capi.dmdgpu_options, _capi.dmdgpu_scalars, _capi.dmdgpu_timing,
                _capi.dmdgpu_frame):
        want.append(ctypes.sizeof(cls))
        want.extend(getattr(cls, f[0]).offset for f in cls._fields_)
    assert got == want


def test_config_check_errors():
    _, good = workloads.argon_fcc(n_cells=2).to_json()
    check_config(good)
    bad = json.loads(json.dumps(good))
    del bad["run"]["dt"]
    with pytest.raises(InputError, match="missing key 'run.dt'"):
        check_config(bad)
    bad = json.loads(json.dumps(good))
    del bad["barostat"]
    with pytest.raises(InputError, match="missing section 'barostat'"):
        check_config(bad)
    bad = json.loads(json.dumps(good))
    bad["extra"] = {}
    with pytest.raises(InputError, match="unknown section 'extra'"):
        check_config(bad)
    bad = json.loads(json.dumps(good))
    bad["lj"]["shift"] = True
    with pytest.raises(InputError, match="unknown key 'lj.shift'"):
        check_config(bad)
    bad = json.loads(json.dumps(good))
    bad["run"]["dt"] = "x"
    with pytest.raises(InputError, match="'run.dt' must be a float"):
        check_config(bad)
    bad = json.loads(json.dumps(good))
    bad["constraints"]["type"] = "shake"  # no constraint pairs in the argon system
    sysj, _ = workloads.argon_fcc(n_cells=2).to_json()
    with pytest.raises(InputError, match="shake"):
        load_inputs(sysj, bad)


@pytest.mark.parametrize("system", ["water", "decane", "rigid_water"])
def test_reader_matches_workload_config(system, tmp_path):
    """The reader rebuilds from the reference's input format exactly the
    configuration the generators build directly (dicts, JSON text and files)."""
    w = {"water": lambda: workloads.water_box(n_mol=27, box=1.0, seed=1, spacing=0.1),
         "decane": lambda: workloads.decane_melt(6, 3, impropers=True),
         "rigid_water": lambda: workloads.water_box(n_mol=27, box=1.0, seed=1, spacing=0.1,
                                                    rigid=True)}[system]()
    sys_json, cfg_json = w.to_json()
    c = w.config()
    (tmp_path / "s.json").write_text(json.dumps(sys_json))
    for b in (load_inputs(sys_json, cfg_json), load_inputs(json.dumps(sys_json), json.dumps(cfg_json)),
              load_inputs(str(tmp_path / "s.json"), cfg_json)):
        for k in SimulationConfig._F64 + SimulationConfig._I32:
            assert np.array_equal(getattr(b, k), getattr(c, k)), k
        for k in ("excl_i", "excl_j", "constraint_i", "constraint_j", "constraint_dist"):
            assert list(getattr(b, k)) == list(getattr(c, k)), k
        assert b.lj_n_types == c.lj_n_types and b.use_lj
        for k in ("box_size", "lj_cutoff", "coulomb_type", "coulomb_cutoff", "dt", "seed", "gen_vel",
                  "constraint_type", "constraint_tolerance"):
            assert getattr(b, k) == getattr(c, k), k
        assert b.thermostat.type == c.thermostat.type and b.barostat.tau == c.barostat.tau


def test_system_desc_rejects_unknown_thermostat():
    c = workloads.argon_fcc(n_cells=2).config()
    c.thermostat.type = "langevin"
    with pytest.raises(RuntimeError, match="Unknown thermostat type"):
        _capi.SystemDesc(c)
