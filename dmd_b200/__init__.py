"""dmd_b200 -- B200 (sm_100a) implementation of DMD's per-step force-and-integrate path.

The engine runs on the GPU through the C ABI of include/dmdgpu.h
(libdmdgpu.so); there is no CPU fallback.  ``SimulationConfig`` and ``Engine``
carry the surface of the reference's pybind module (python/dmd/core.cpp), so
the reference's own Python package can import them in place of its CPU core;
``load_inputs`` reads the reference's system.json / config.json formats;
``Batch`` and ``serve`` advance many systems in one device table.
"""
from .core import BarostatConfig, DmdGpuError, Engine, SimulationConfig, ThermostatConfig
from .inputs import InputError, load_inputs

__all__ = [
    "SimulationConfig", "Engine", "ThermostatConfig", "BarostatConfig", "DmdGpuError",
    "load_inputs", "InputError",
]
