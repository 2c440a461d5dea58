"""`ReservoirSimulator`: the reference simulator's construction/step API over the device path.

Construction and setters mirror the reference (`Deck`); `step(dt)` runs one report step of the
fully implicit controller on the GPU through the C ABI.  The device context is created at the
first step, from the deck and the current state.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _lib
from .deck import Deck


class DeviceError(RuntimeError):
    pass


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class ReservoirSimulator(Deck):
    """Drop-in for the reference `ReservoirSimulator` (src/lib/ressim/src/frontend.rs) on the
    FIM path.  Setters are inherited from `Deck`; the device context is built lazily."""

    def __init__(self, nx, ny, nz, porosity_val, **kw):
        super().__init__(nx, ny, nz, porosity_val, **kw)
        self._h = None
        self._keep = None
        self.time_days = 0.0
        self.last_solver_warning = ""
        self.last_step_report = None

    @classmethod
    def from_deck(cls, deck: Deck) -> "ReservoirSimulator":
        sim = cls.__new__(cls)
        sim.__dict__.update({k: v for k, v in deck.__dict__.items()})
        sim.wells = list(deck.wells)
        sim._h = None
        sim._keep = None
        sim.time_days = 0.0
        sim.last_solver_warning = ""
        sim.last_step_report = None
        return sim

    # ---- device context ----
    def _context(self):
        if self._h is not None:
            return self._h
        L = _lib.load()
        d, keep = self.to_abi()
        h = C.c_void_p()
        rc = L.rf_create(C.byref(d), C.byref(h))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_create failed ({rc}): {_lib.last_error(None)}")
        self._h, self._keep = h, (d, keep)
        p = np.ascontiguousarray(self.pressure, dtype=np.float64)
        sw = np.ascontiguousarray(self.sat_water, dtype=np.float64)
        sg = np.ascontiguousarray(self.sat_gas, dtype=np.float64)
        rs = np.ascontiguousarray(self.rs, dtype=np.float64)
        rc = L.rf_set_state(h, _ptr(p), _ptr(sw), _ptr(sg), _ptr(rs), float(self.time_days))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_set_state failed ({rc}): {_lib.last_error(h)}")
        return h

    def close(self):
        if self._h is not None:
            _lib.load().rf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- stepping (frontend.rs:345-349) ----
    def step(self, target_dt_days: float) -> dict:
        h = self._context()
        rep = _abi.RfStepReport()
        rc = _lib.load().rf_step(h, float(target_dt_days), C.byref(rep))
        if rc < 0:
            raise DeviceError(f"rf_step failed ({rc}): {_lib.last_error(h)}")
        self.time_days = rep.time_days
        self.last_step_report = rep.as_dict()
        self.last_solver_warning = "" if rep.warning == 0 else f"solver warning {rep.warning}"
        return self.last_step_report

    # ---- getters (frontend.rs:523-605) ----
    def _state(self):
        h = self._context()
        n = self.n_cells
        out = {k: np.zeros(n) for k in ("pressure", "sat_water", "sat_oil", "sat_gas", "rs")}
        t = C.c_double()
        rc = _lib.load().rf_get_state(h, _ptr(out["pressure"]), _ptr(out["sat_water"]), _ptr(out["sat_oil"]),
                                      _ptr(out["sat_gas"]), _ptr(out["rs"]), C.byref(t))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_get_state failed ({rc}): {_lib.last_error(h)}")
        out["time"] = t.value
        return out

    def get_pressures(self):
        return self._state()["pressure"]

    def get_sat_water(self):
        return self._state()["sat_water"]

    def get_sat_oil(self):
        return self._state()["sat_oil"]

    def get_time(self):
        return self.time_days

    def get_well_bhp(self):
        b = np.zeros(len(self.wells))
        _lib.load().rf_get_well_bhp(self._context(), _ptr(b), len(b))
        return b

    def get_rate_history(self):
        h = self._context()
        L = _lib.load()
        out = []
        for i in range(L.rf_rate_history_len(h)):
            r = _abi.RfTimePointRates()
            L.rf_rate_history_get(h, i, C.byref(r))
            out.append(r.as_dict())
        return out

    def get_last_solver_warning(self):
        return self.last_solver_warning

    def profile(self, enable=None, reset=False) -> dict:
        """Phase timings (ms, CUDA events) and the BiCGStab iteration total; `enable` switches the
        profiler on/off."""
        out = np.zeros(len(_lib.PHASES) + 4)
        en = -1 if enable is None else int(bool(enable))
        rc = _lib.load().rf_profile(self._context(), en, int(reset), _ptr(out), len(out))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_profile failed ({rc}): {_lib.last_error(self._context())}")
        d = {k: float(v) for k, v in zip(_lib.PHASES, out)}
        k = len(_lib.PHASES)
        d["bicgstab_iterations"] = int(out[k])
        d["bicgstab_launches"] = int(out[k + 1])
        d["nnzb"] = int(out[k + 2])
        d["level_kernels"] = bool(out[k + 3])
        return d

    def set_linear_precision(self, mode: str) -> None:
        """"fp64" (default, the reference's arithmetic) or "mixed" (FP32 block-ILU0 and pressure
        stage under the FP64 FGMRES)."""
        codes = {"fp64": _abi.RF_PRECISION_FP64, "mixed": _abi.RF_PRECISION_MIXED}
        if mode not in codes:
            raise ValueError(f"precision must be one of {sorted(codes)}")
        rc = _lib.load().rf_set_linear_precision(self._context(), codes[mode])
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_set_linear_precision failed ({rc}): {_lib.last_error(self._context())}")

    def set_cluster_size(self, ctas: int = 0) -> int:
        """CTAs of the cluster running the level-scheduled kernels (0: automatic); returns the size
        in use."""
        rc = _lib.load().rf_set_cluster_size(self._context(), int(ctas))
        if rc <= 0:
            raise DeviceError(f"rf_set_cluster_size failed ({rc}): {_lib.last_error(self._context())}")
        return rc

    def set_pressure_solver(self, kind: str = "auto", threads: int = 0) -> None:
        """Kernels of the CPR's level-scheduled solves: "cluster" (the thread-block cluster
        kernels), "level" (one thread block in level order, `threads` threads, 0 automatic) or
        "auto"."""
        codes = {"auto": 0, "cluster": 1, "level": 2}
        if kind not in codes:
            raise ValueError(f"pressure solver must be one of {sorted(codes)}")
        rc = _lib.load().rf_set_pressure_solver(self._context(), codes[kind], int(threads))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_set_pressure_solver failed ({rc}): {_lib.last_error(self._context())}")

    def set_controller_options(self, one_substep_per_report_step: bool = False, cnv_tol: float = 0.0,
                               mb_tol: float = 0.0) -> None:
        """Controller options of the device path (no counterpart in the reference): take every
        report step as one substep without retries, and/or converge Newton to fixed CNV / MB
        tolerances instead of the reference's tiers.  Defaults restore the reference controller."""
        rc = _lib.load().rf_set_controller_options(self._context(), int(bool(one_substep_per_report_step)),
                                                   float(cnv_tol), float(mb_tol))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_set_controller_options failed ({rc}): {_lib.last_error(self._context())}")

    def set_linear_refinement(self, rtol: float = 0.0, max_passes: int = 0) -> None:
        """Refine every CPR-FGMRES solve of the Newton systems to |b - A x| <= rtol |b| (at most
        max_passes solves, 0: 12); no counterpart in the reference.  With tight CNV / MB tolerances
        this is the matched profile for comparisons at 1e-6.  rtol = 0 restores the reference's
        single solve."""
        rc = _lib.load().rf_set_linear_refinement(self._context(), float(rtol), int(max_passes))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_set_linear_refinement failed ({rc}): {_lib.last_error(self._context())}")

    def adjoint_record(self, enable: bool = True) -> None:
        """Start (clearing the tape) or stop recording report-step checkpoints for `backward`."""
        rc = _lib.load().rf_adjoint_record(self._context(), int(bool(enable)))
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_adjoint_record failed ({rc}): {_lib.last_error(self._context())}")

    def backward(self):
        """Discrete adjoint over the recorded report steps (no counterpart in the reference).
        Returns (cumulative surface oil produced [Sm3], d/d ln(permeability multiplier) per cell,
        d/d(active control) per physical well)."""
        h = self._context()
        L = _lib.load()
        nw = int(L.rf_well_count(h))
        g = np.zeros(self.n_cells)
        gc = np.zeros(max(nw, 1))
        val = C.c_double()
        obj = _abi.RfObjective(_abi.RF_OBJECTIVE_CUMULATIVE_OIL)
        rc = L.rf_backward(h, C.byref(obj), C.byref(val), _ptr(g), _ptr(gc), nw)
        if rc != _abi.RF_OK:
            raise DeviceError(f"rf_backward failed ({rc}): {_lib.last_error(h)}")
        return val.value, g, gc[:nw]

    def kernel_launches(self) -> int:
        return int(_lib.load().rf_kernel_launches(self._context()))

    def state(self):
        return self._state()


def linear_solve_bsr(sim: ReservoirSimulator, row_ptr, cols, vals, rhs):
    """Linear-solver seam: CPR-FGMRES on a tail-free 3x3 block system on `sim`'s grid."""
    h = sim._context()
    n = sim.n_cells
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(cols, dtype=np.int32)
    vl = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(3 * n)
    rep = _abi.RfLinearReport()
    rc = _lib.load().rf_linear_solve_bsr(h, n, rp.ctypes.data_as(C.POINTER(C.c_int32)),
                                         cl.ctypes.data_as(C.POINTER(C.c_int32)), _ptr(vl), _ptr(b), _ptr(x),
                                         C.byref(rep))
    if rc != _abi.RF_OK:
        raise DeviceError(f"rf_linear_solve_bsr failed ({rc}): {_lib.last_error(h)}")
    return x, rep


def linear_solve_csr(sim: ReservoirSimulator, row_ptr, cols, vals, rhs):
    """Linear-solver seam on the full Newton system with its well tail (scalar CSR, rows ordered
    cells x 3, well BHPs, perforation rates): direct LU for at most 512 rows, else well
    elimination, CPR-FGMRES and tail recovery on the device."""
    h = sim._context()
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cl = np.ascontiguousarray(cols, dtype=np.int32)
    vl = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    n_rows = len(rp) - 1
    if len(b) != n_rows:
        raise ValueError(f"rhs has {len(b)} values for {n_rows} rows")
    x = np.zeros(n_rows)
    rep = _abi.RfLinearReport()
    rc = _lib.load().rf_linear_solve_csr(h, n_rows, rp.ctypes.data_as(C.POINTER(C.c_int32)),
                                         cl.ctypes.data_as(C.POINTER(C.c_int32)), _ptr(vl), _ptr(b), _ptr(x),
                                         C.byref(rep))
    if rc != _abi.RF_OK:
        raise DeviceError(f"rf_linear_solve_csr failed ({rc}): {_lib.last_error(h)}")
    return x, rep


def dense_solve_noalloc(n: int, a_ptr: int, b_ptr: int, x_ptr: int, stream: int = 0) -> None:
    """x = A^{-1} b through rf_dense_solve_noalloc, for callers that may not allocate device
    memory.  `a_ptr` (dense row-major n x n), `b_ptr` and `x_ptr` are device addresses of float64
    data owned by the caller; n <= 299.  The call allocates nothing; calls must not overlap."""
    err = C.create_string_buffer(256)
    rc = _lib.load().rf_dense_solve_noalloc(int(n), C.c_void_p(a_ptr), C.c_void_p(b_ptr), C.c_void_p(x_ptr),
                                            C.c_void_p(stream or None), err, len(err))
    if rc != _abi.RF_OK:
        raise DeviceError(f"rf_dense_solve_noalloc failed ({rc}): {err.value.decode(errors='replace')}")
