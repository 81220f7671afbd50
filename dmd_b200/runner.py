"""dmd.run() drop-in (python/dmd/runner.py:10-60) on the GPU engine."""
from __future__ import annotations

import json

from .core import Engine
from .status import SimulationStatus
from .system import SystemBuilder


def run(system_data: str | dict | None = None, config_data: str | dict | None = None,
        system_json: str | None = None, config_json: str | None = None,
        checkpoint: str | None = None, progress_interval: int = 100, **engine_kw) -> Engine:
    """Build the system from system.json/config.json data and run n_steps.

    As in the reference, the run proceeds in chunks of ``progress_interval``
    steps; each chunk is one ``Engine.run_n`` call, i.e. one device call.
    ``engine_kw`` (precision, profile, skin, device) select the backend.
    """
    if system_json and system_data is None:
        with open(system_json) as f:
            system_data = json.load(f)
    if config_json and config_data is None:
        with open(config_json) as f:
            config_data = json.load(f)
    if checkpoint:
        from .checkpoint import checkpoint_to_system_data, read_checkpoint
        system_data = checkpoint_to_system_data(read_checkpoint(checkpoint))
    if not system_data:
        raise ValueError("Provide one of: system_data or checkpoint")
    if isinstance(system_data, str):
        system_data = json.loads(system_data)
    builder = SystemBuilder(system_data)
    if config_data:
        if isinstance(config_data, str):
            config_data = json.loads(config_data)
        builder.apply_config_json(config_data)
    cfg = builder.build()
    engine = Engine(cfg, **engine_kw)
    if progress_interval > 0 and cfg.n_steps > 0:
        status = SimulationStatus(engine, dt=cfg.dt, interval=progress_interval)
        status.start()
        remaining = cfg.n_steps
        while remaining > 0:
            take = min(progress_interval, remaining)
            engine.run_n(take)
            remaining -= take
            status.step()
        status.finish()
    else:
        engine.run()
    return engine
