"""Batched replicas and continuous serving over the C ABI batch API.

A ``Batch`` packs many independent systems ("slots") of different sizes into
one device table; ``step(n)`` advances every running slot with the same kernel
launches (one CUDA graph per step over the packed table).  Slots are admitted
while the HBM budget allows (``BudgetExceeded`` otherwise) and released when
done; admitting or releasing repacks the table between steps, carrying the
state of running slots over unchanged.  A slot's trajectory does not depend on
which other slots share the batch (fixed-point force sums, per-replica
reductions in a fixed order).

No counterpart in the reference, which runs one SimulationEngine per process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .core import DmdGpuError, _options


class BudgetExceeded(DmdGpuError):
    """Admission refused: the system does not fit the HBM budget (or slot table)."""


class Batch:
    def __init__(self, budget_bytes: int = 150 * 10**9, precision=None, profile=None, skin=None,
                 device=None, rng_seed=None):
        self._lib = _capi.lib()
        self._opt = _options(precision, profile, skin, device, rng_seed)
        h = C.c_void_p()
        rc = self._lib.dmdgpu_batch_create(int(budget_bytes), C.byref(self._opt), C.byref(h))
        if rc != 0:
            msg = self._lib.dmdgpu_batch_last_error(h) if h else b"dmdgpu_batch_create failed"
            if h:
                self._lib.dmdgpu_batch_destroy(h)
            raise DmdGpuError(rc, (msg or b"").decode())
        self._h = h
        self._n = {}            # slot -> n_atoms
        self.budget_bytes = int(budget_bytes)

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.dmdgpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            msg = (self._lib.dmdgpu_batch_last_error(self._h) or b"").decode()
            if rc == 7:
                raise BudgetExceeded(rc, msg)
            raise DmdGpuError(rc, msg)

    # -- slots -------------------------------------------------------------
    def admit(self, cfg, n_steps: int) -> int:
        """Admit a system (SimulationConfig) to run ``n_steps`` steps; returns its slot."""
        desc = _capi.SystemDesc(cfg)
        slot = C.c_int32(-1)
        self._check(self._lib.dmdgpu_batch_admit(self._h, C.byref(desc.s), int(n_steps),
                                                 C.byref(slot)))
        self._n[slot.value] = int(len(cfg.masses))
        return slot.value

    def release(self, slot: int):
        self._check(self._lib.dmdgpu_batch_release(self._h, int(slot)))
        self._n.pop(slot, None)

    def step(self, n: int = 1):
        """Advance every running slot by up to n steps (each stops at its own target)."""
        self._check(self._lib.dmdgpu_batch_step(self._h, int(n)))

    def step_timed(self, n: int, l2_flush_bytes: int = 0) -> dict:
        """step(n) as one CUDA graph with device timing of every step and of every
        non-bonded / PME launch (optional L2 flush between steps)."""
        t = _capi.dmdgpu_timing()
        self._check(self._lib.dmdgpu_batch_step_timed(self._h, int(n), int(l2_flush_bytes),
                                                      C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def poll(self) -> list[int]:
        """Slots that reached their step target since the last poll."""
        cap = max(1, len(self._n))
        buf = np.empty(cap, np.int32)
        n = C.c_int32(0)
        self._check(self._lib.dmdgpu_batch_poll(self._h, _capi.iptr(buf), cap, C.byref(n)))
        return buf[:min(n.value, cap)].tolist()

    def _state(self, slot, which):
        n = self._n[slot]
        x, y, z = np.empty(n), np.empty(n), np.empty(n)
        self._check(self._lib.dmdgpu_batch_get_state(self._h, int(slot), which, _capi.dptr(x),
                                                     _capi.dptr(y), _capi.dptr(z)))
        return np.stack([x, y, z], axis=1)

    def positions(self, slot: int) -> np.ndarray:
        return self._state(slot, 0)

    def velocities(self, slot: int) -> np.ndarray:
        return self._state(slot, 1)

    def forces(self, slot: int) -> np.ndarray:
        return self._state(slot, 2)

    def scalars(self, slot: int) -> _capi.dmdgpu_scalars:
        s = _capi.dmdgpu_scalars()
        self._check(self._lib.dmdgpu_batch_get_scalars(self._h, int(slot), C.byref(s)))
        return s

    # -- accounting --------------------------------------------------------
    @property
    def used_bytes(self) -> int:
        return int(self._lib.dmdgpu_batch_used_bytes(self._h))

    @property
    def active(self) -> int:
        return int(self._lib.dmdgpu_batch_active(self._h))

    def launch_info(self) -> dict:
        """Launch configuration of the current device table (see Engine.launch_info)."""
        info = _capi.dmdgpu_launch_info()
        self._check(self._lib.dmdgpu_batch_get_launch_info(self._h, C.byref(info)))
        return _capi.launch_info_dict(info)

    @property
    def slots(self) -> list[int]:
        return sorted(self._n)

    def n_atoms(self, slot: int) -> int:
        return self._n[slot]

    @staticmethod
    def footprint(cfg, precision=None, profile=None, skin=None) -> int:
        """Device bytes a system would hold (the admission estimate)."""
        desc = _capi.SystemDesc(cfg)
        opt = _options(precision, profile, skin, None, None)
        return int(_capi.lib().dmdgpu_footprint_bytes(C.byref(desc.s), C.byref(opt)))
