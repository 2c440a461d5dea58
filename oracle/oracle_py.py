"""ORACLE — test infrastructure only.

ctypes wrapper of the CPU oracle (oracle/_build/liborc_fim.so, built by oracle/Makefile).  Only
tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this module; the product
(ressim_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from ressim_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
# RESSIM_ORACLE_SO selects another build of the same sources (the CPU baseline's -march=native one)
_SO = os.environ.get("RESSIM_ORACLE_SO") or os.path.join(_HERE, "_build", "liborc_fim.so")
NATIVE_SO = os.path.join(_HERE, "_build", "liborc_fim_native.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def build_native() -> str | None:
    """Builds the oracle with -O3 -march=native for the host that runs it (the timed CPU baseline)
    and returns its path, or None when the build fails."""
    r = subprocess.run(["make", "-s", "-B", "-C", _HERE, "native"], capture_output=True)
    return NATIVE_SO if r.returncode == 0 and os.path.exists(NATIVE_SO) else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        L.orc_create.argtypes = [C.POINTER(_abi.RfDeck), C.POINTER(C.c_void_p)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_double]
        L.orc_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_get_well_bhp.argtypes = [C.c_void_p, _dp, C.c_int32]
        L.orc_step.argtypes = [C.c_void_p, C.c_double, C.POINTER(_abi.RfStepReport)]
        L.orc_rate_history_len.argtypes = [C.c_void_p]
        L.orc_rate_history_get.argtypes = [C.c_void_p, C.c_int32, C.POINTER(_abi.RfTimePointRates)]
        L.orc_set_controller_options.argtypes = [C.c_int32, C.c_double, C.c_double]
        L.orc_set_linear_refinement.argtypes = [C.c_double, C.c_int32]
        L.orc_assemble_current.argtypes = [C.c_void_p, C.c_double, _ip, _ip, _dp, _ip, _ip, _dp]
        L.orc_initial_well_state.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_linear_solve_csr.argtypes = [C.c_int32, _ip, _ip, _dp, _dp, C.c_int32, _dp,
                                           C.POINTER(_abi.RfLinearReport)]
        L.orc_cnv_mb_from_parts.argtypes = [C.c_int32, _dp, _dp, _dp, C.c_int32, _dp]
        L.orc_opm_chop.argtypes = [C.c_int32, _dp, C.c_int32, _dp, _dp, C.c_double, _dp]
        L.orc_pid_dt.argtypes = [C.c_double, _dp]
        L.orc_pid_dt.restype = C.c_double
        L.orc_iteration_count_dt.argtypes = [C.c_double, C.c_int32]
        L.orc_iteration_count_dt.restype = C.c_double
        L.orc_growth_decision.argtypes = [C.c_double, C.c_int32, _dp, C.c_int32, _ip]
        L.orc_growth_decision.restype = C.c_double
        L.orc_relative_change.argtypes = [C.c_int32, _dp, _dp]
        L.orc_relative_change.restype = C.c_double
        L.orc_corey_table.argtypes = [C.POINTER(_abi.RfDeck), C.c_double, _dp]
        L.orc_water_inverse_fvf.argtypes = [C.c_double] * 4
        L.orc_water_inverse_fvf.restype = C.c_double
        L.orc_well_index.argtypes = [C.POINTER(_abi.RfDeck), C.c_int32]
        L.orc_well_index.restype = C.c_double
        L.orc_ad_probe.argtypes = [C.c_int32, C.c_double, C.c_double, _dp]
        L.orc_set_sum_order.argtypes = [C.c_int32]
        L.orc_head_offsets.argtypes = [C.c_void_p, _dp, C.c_int32]
        L.orc_assemble_state.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp, _dp, _ip, _ip, _dp, _ip, _ip, _dp]
        L.orc_topology.argtypes = [C.c_void_p, _ip, _ip]
        L.orc_assemble_state_regimes.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _ip, _ip, _dp, _dp, _ip, _ip,
                                                 _dp, _ip, _ip, _dp]
        L.orc_blackoil_probe.argtypes = [_dp, C.c_int32, C.c_double, C.c_int32, _dp, _dp]
        _lib = L
    return _lib


def ptr(a):
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)


class OracleSimulator:
    """The oracle behind the same deck/state/step surface as ressim_b200.ReservoirSimulator."""

    def __init__(self, deck):
        self.deck = deck
        self._abi, self._keep = deck.to_abi()
        h = C.c_void_p()
        rc = lib().orc_create(C.byref(self._abi), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle rejected the deck (status {rc})")
        self._h = h
        n = deck.n_cells
        p = np.ascontiguousarray(deck.pressure, dtype=np.float64)
        sw = np.ascontiguousarray(deck.sat_water, dtype=np.float64)
        sg = np.ascontiguousarray(deck.sat_gas, dtype=np.float64)
        rs = np.ascontiguousarray(deck.rs, dtype=np.float64)
        lib().orc_set_state(self._h, ptr(p), ptr(sw), ptr(sg), ptr(rs), 0.0)
        self.n = n

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt):
        rep = _abi.RfStepReport()
        rc = lib().orc_step(self._h, dt, C.byref(rep))
        return rc, rep

    def state(self):
        out = {k: np.zeros(self.n) for k in ("pressure", "sat_water", "sat_oil", "sat_gas", "rs")}
        t = C.c_double()
        lib().orc_get_state(self._h, ptr(out["pressure"]), ptr(out["sat_water"]), ptr(out["sat_oil"]),
                            ptr(out["sat_gas"]), ptr(out["rs"]), C.byref(t))
        out["time"] = t.value
        return out

    def well_bhp(self):
        b = np.zeros(len(self.deck.wells))
        lib().orc_get_well_bhp(self._h, ptr(b), len(b))
        return b

    def rate_history(self):
        n = lib().orc_rate_history_len(self._h)
        out = []
        for i in range(n):
            r = _abi.RfTimePointRates()
            lib().orc_rate_history_get(self._h, i, C.byref(r))
            out.append(r.as_dict())
        return out

    def assemble_current(self, dt):
        nu, nnz = C.c_int32(), C.c_int32()
        lib().orc_assemble_current(self._h, dt, C.byref(nu), C.byref(nnz), None, None, None, None)
        res = np.zeros(nu.value)
        ptr_ = np.zeros(nu.value + 1, dtype=np.int32)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        lib().orc_assemble_current(self._h, dt, C.byref(nu), C.byref(nnz), ptr(res), iptr(ptr_), iptr(col),
                                   ptr(val))
        return res, ptr_, col, val

    def head_offsets(self):
        """Completion head offsets (bar) of the current state, one per deck well entry."""
        out = np.zeros(len(self.deck.wells))
        lib().orc_head_offsets(self._h, ptr(out), len(out))
        return out

    def topology(self):
        w, p = C.c_int32(), C.c_int32()
        lib().orc_topology(self._h, C.byref(w), C.byref(p))
        return w.value, p.value

    def assemble_state(self, dt, prev, cur, bhp, q):
        """Residual and CSR Jacobian at (cur, bhp, q) against `prev`; prev/cur are (n, 3) arrays."""
        prev = np.ascontiguousarray(prev, dtype=np.float64).ravel()
        cur = np.ascontiguousarray(cur, dtype=np.float64).ravel()
        bhp = np.ascontiguousarray(bhp, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        nu, nnz = C.c_int32(), C.c_int32()
        args = (self._h, dt, ptr(prev), ptr(cur), ptr(bhp) if bhp.size else None, ptr(q) if q.size else None)
        lib().orc_assemble_state(*args, C.byref(nu), C.byref(nnz), None, None, None, None)
        res = np.zeros(nu.value)
        ptr_ = np.zeros(nu.value + 1, dtype=np.int32)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        lib().orc_assemble_state(*args, C.byref(nu), C.byref(nnz), ptr(res), iptr(ptr_), iptr(col), ptr(val))
        return res, ptr_, col, val

    def assemble_state_regimes(self, dt, prev, cur, prev_regime, cur_regime, bhp, q):
        """assemble_state with explicit cell regimes (0 saturated, 1 undersaturated)."""
        prev = np.ascontiguousarray(prev, dtype=np.float64).ravel()
        cur = np.ascontiguousarray(cur, dtype=np.float64).ravel()
        pr = np.ascontiguousarray(prev_regime, dtype=np.int32)
        cr = np.ascontiguousarray(cur_regime, dtype=np.int32)
        bhp = np.ascontiguousarray(bhp, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        nu, nnz = C.c_int32(), C.c_int32()
        args = (self._h, dt, ptr(prev), ptr(cur), iptr(pr), iptr(cr), ptr(bhp) if bhp.size else None,
                ptr(q) if q.size else None)
        lib().orc_assemble_state_regimes(*args, C.byref(nu), C.byref(nnz), None, None, None, None)
        res = np.zeros(nu.value)
        ptr_ = np.zeros(nu.value + 1, dtype=np.int32)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        lib().orc_assemble_state_regimes(*args, C.byref(nu), C.byref(nnz), ptr(res), iptr(ptr_), iptr(col), ptr(val))
        return res, ptr_, col, val

    def initial_well_state(self, n_wells, n_perfs):
        b = np.zeros(max(n_wells, 1))
        q = np.zeros(max(n_perfs, 1))
        lib().orc_initial_well_state(self._h, ptr(b), ptr(q))
        return b[:n_wells], q[:n_perfs]


def blackoil_probe(rows, c_o, mode, inputs, n_out=16):
    """orc_blackoil_probe: black-oil known-answer evaluations on a PVT table (see orc_driver.inc)."""
    r = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).reshape(-1, 6))
    x = np.ascontiguousarray(np.asarray(inputs, dtype=np.float64))
    out = np.zeros(n_out)
    rc = lib().orc_blackoil_probe(ptr(r), len(r), float(c_o), int(mode), ptr(x), ptr(out))
    if rc != 0:
        raise ValueError(f"probe mode {mode} rejected")
    return out


def linear_solve_csr(ptr_, col, val, rhs, n_cells):
    n = len(ptr_) - 1
    x = np.zeros(n)
    rep = _abi.RfLinearReport()
    p = np.ascontiguousarray(ptr_, dtype=np.int32)
    c = np.ascontiguousarray(col, dtype=np.int32)
    v = np.ascontiguousarray(val, dtype=np.float64)
    r = np.ascontiguousarray(rhs, dtype=np.float64)
    lib().orc_linear_solve_csr(n, iptr(p), iptr(c), ptr(v), ptr(r), n_cells, ptr(x), C.byref(rep))
    return x, rep
