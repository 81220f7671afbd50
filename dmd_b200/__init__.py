"""dmd_b200 -- B200 (sm_100a) implementation of DMD's per-step force-and-integrate path.

Drop-in for the reference's Python API (python/dmd/__init__.py): SimulationConfig,
Engine, SystemBuilder, run, validate_config, apply_config, generate_config_template.
The engine runs on the GPU through the C ABI of include/dmdgpu.h (libdmdgpu.so);
there is no CPU fallback.
"""
from .config import apply_config, generate_config_template, validate_config
from .core import BarostatConfig, DmdGpuError, Engine, SimulationConfig, ThermostatConfig
from .system import SystemBuilder
from .runner import run

__all__ = [
    "SimulationConfig", "Engine", "SystemBuilder", "run", "validate_config", "apply_config",
    "generate_config_template", "ThermostatConfig", "BarostatConfig", "DmdGpuError",
]
