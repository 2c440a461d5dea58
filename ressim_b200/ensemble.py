"""`Ensemble`: many independent decks (sensitivity variants of uneven sizes) stepped together.

Each variant has its own device context; `step(dt)` advances every variant by one report step
through `rf_batch_step`, which drives the variants from a pool of host threads so their kernels
run concurrently on the GPU.  The reference simulator steps one deck per object; this is the
batched form of the same step API.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _lib
from .deck import Deck
from .simulator import DeviceError, _ptr


class Ensemble:
    def __init__(self, decks: list[Deck], host_threads: int = 0, precision: str = "fp64"):
        L = _lib.load()
        self.decks = list(decks)
        self._abis = [d.to_abi() for d in self.decks]
        arr = (C.POINTER(_abi.RfDeck) * len(self.decks))(*[C.pointer(a[0]) for a in self._abis])
        h = C.c_void_p()
        rc = L.rf_batch_create(arr, len(self.decks), int(host_threads), C.byref(h))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_batch_create failed ({rc}): {_lib.last_error(None)}")
        self._h = h
        self._ctx = [L.rf_batch_context(h, i) for i in range(len(self.decks))]
        codes = {"fp64": _abi.RF_PRECISION_FP64, "mixed": _abi.RF_PRECISION_MIXED}
        for i, d in enumerate(self.decks):
            p = np.ascontiguousarray(d.pressure, dtype=np.float64)
            sw = np.ascontiguousarray(d.sat_water, dtype=np.float64)
            sg = np.ascontiguousarray(d.sat_gas, dtype=np.float64)
            rs = np.ascontiguousarray(d.rs, dtype=np.float64)
            rc = L.rf_set_state(self._ctx[i], _ptr(p), _ptr(sw), _ptr(sg), _ptr(rs), 0.0)
            if rc != _abi.RF_OK:
                raise DeviceError(f"rf_set_state failed for variant {i}: {_lib.last_error(self._ctx[i])}")
            rc = L.rf_set_linear_precision(self._ctx[i], codes[precision])
            if rc != _abi.RF_OK:
                raise DeviceError(f"rf_set_linear_precision failed for variant {i}")

    def __len__(self):
        return len(self.decks)

    @property
    def cells(self) -> int:
        return sum(d.n_cells for d in self.decks)

    def step(self, target_dt_days: float) -> list[dict]:
        n = len(self.decks)
        reps = (_abi.RfStepReport * n)()
        rc = _lib.load().rf_batch_step(self._h, float(target_dt_days), reps)
        if rc < 0:
            msgs = [f"variant {i}: {m}" for i, m in ((i, _lib.last_error(c)) for i, c in enumerate(self._ctx)) if m]
            raise DeviceError(f"rf_batch_step failed ({rc}): " + "; ".join(msgs[:3]))
        return [r.as_dict() for r in reps]

    def state(self, i: int) -> dict:
        n = self.decks[i].n_cells
        p, sw, so, sg, rs = (np.zeros(n) for _ in range(5))
        t = C.c_double()
        rc = _lib.load().rf_get_state(self._ctx[i], _ptr(p), _ptr(sw), _ptr(so), _ptr(sg), _ptr(rs), C.byref(t))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_get_state failed for variant {i}: {_lib.last_error(self._ctx[i])}")
        return {"pressure": p, "sat_water": sw, "sat_oil": so, "sat_gas": sg, "rs": rs, "time": t.value}

    def kernel_launches(self) -> int:
        L = _lib.load()
        return sum(int(L.rf_kernel_launches(c)) for c in self._ctx)

    def profile(self, i: int, enable=None, reset=False) -> dict:
        out = np.zeros(len(_lib.PHASES) + 4)
        en = -1 if enable is None else int(bool(enable))
        _lib.load().rf_profile(self._ctx[i], en, int(reset), _ptr(out), len(out))
        d = {k: float(v) for k, v in zip(_lib.PHASES, out)}
        k = len(_lib.PHASES)
        d["bicgstab_iterations"] = int(out[k])
        d["bicgstab_launches"] = int(out[k + 1])
        d["nnzb"] = int(out[k + 2])
        d["level_kernels"] = bool(out[k + 3])
        return d

    def set_mode(self, mode: str) -> None:
        """"groups" (default: fibers on per-group threads, one batched launch per group for the
        pressure solves and block-ILU0 sweeps) or "threads" (a stream and a host-thread turn per
        variant)."""
        codes = {"groups": 0, "threads": 1}
        if mode not in codes:
            raise ValueError(f"batch mode must be one of {sorted(codes)}")
        rc = _lib.load().rf_batch_set_mode(self._h, codes[mode])
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_batch_set_mode failed ({rc})")

    def batch_profile(self, enable=None, reset=False) -> dict:
        """Batched-launch statistics: groups, then launches / solves / device ms per kind."""
        out = np.zeros(10)
        en = -1 if enable is None else int(bool(enable))
        _lib.load().rf_batch_profile(self._h, en, int(reset), _ptr(out), len(out))
        d = {"groups": int(out[0])}
        for k, name in enumerate(("pressure", "block_sweep", "factor")):
            d[f"{name}_launches"] = int(out[1 + 3 * k])
            d[f"{name}_items"] = int(out[2 + 3 * k])
            d[f"{name}_ms"] = float(out[3 + 3 * k])
        return d

    def set_controller_options(self, one_substep_per_report_step: bool = False, cnv_tol: float = 0.0,
                               mb_tol: float = 0.0) -> None:
        """rf_set_controller_options on every variant (see ReservoirSimulator.set_controller_options)."""
        L = _lib.load()
        for i, c in enumerate(self._ctx):
            rc = L.rf_set_controller_options(c, int(bool(one_substep_per_report_step)), float(cnv_tol), float(mb_tol))
            if rc != _abi.RF_OK:
                raise DeviceError(f"rf_set_controller_options failed for variant {i}: {_lib.last_error(c)}")

    def set_linear_refinement(self, rtol: float = 0.0, max_passes: int = 0) -> None:
        """rf_set_linear_refinement on every variant (see ReservoirSimulator.set_linear_refinement)."""
        L = _lib.load()
        for i, c in enumerate(self._ctx):
            rc = L.rf_set_linear_refinement(c, float(rtol), int(max_passes))
            if rc != _abi.RF_OK:
                raise DeviceError(f"rf_set_linear_refinement failed for variant {i}: {_lib.last_error(c)}")

    def well_bhp(self, i: int) -> np.ndarray:
        n = len(self.decks[i].wells)
        out = np.zeros(n)
        rc = _lib.load().rf_get_well_bhp(self._ctx[i], _ptr(out), n)
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_get_well_bhp failed for variant {i}: {_lib.last_error(self._ctx[i])}")
        return out

    def rate_history(self, i: int) -> list[dict]:
        L = _lib.load()
        out = []
        for k in range(L.rf_rate_history_len(self._ctx[i])):
            r = _abi.RfTimePointRates()
            L.rf_rate_history_get(self._ctx[i], k, C.byref(r))
            out.append(r.as_dict())
        return out

    def close(self):
        if self._h is not None:
            _lib.load().rf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
