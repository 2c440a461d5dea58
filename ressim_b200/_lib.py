"""Loader of the device FIM library (libressim_fim.so, built in-tree for sm_100a).

There is no fallback: if the library is missing or fails to load, importing the simulator raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(HERE, "libressim_fim.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO_PATH):
        raise RuntimeError(f"device FIM library not built: {SO_PATH} (run python -m ressim_b200.build)")
    L = C.CDLL(SO_PATH)
    L.rf_create.argtypes = [C.POINTER(_abi.RfDeck), C.POINTER(C.c_void_p)]
    L.rf_destroy.argtypes = [C.c_void_p]
    L.rf_last_error.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    L.rf_set_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, C.c_double]
    L.rf_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]
    L.rf_get_well_bhp.argtypes = [C.c_void_p, _dp, C.c_int32]
    L.rf_step.argtypes = [C.c_void_p, C.c_double, C.POINTER(_abi.RfStepReport)]
    L.rf_rate_history_len.argtypes = [C.c_void_p]
    L.rf_rate_history_get.argtypes = [C.c_void_p, C.c_int32, C.POINTER(_abi.RfTimePointRates)]
    L.rf_linear_solve_bsr.argtypes = [C.c_void_p, C.c_int32, _ip, _ip, _dp, _dp, _dp, C.POINTER(_abi.RfLinearReport)]
    L.rf_linear_solve_csr.argtypes = [C.c_void_p, C.c_int32, _ip, _ip, _dp, _dp, _dp, C.POINTER(_abi.RfLinearReport)]
    L.rf_kernel_launches.argtypes = [C.c_void_p]
    L.rf_kernel_launches.restype = C.c_int64
    L.rf_profile.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _dp, C.c_int32]
    L.rf_set_linear_precision.argtypes = [C.c_void_p, C.c_int32]
    L.rf_set_cluster_size.argtypes = [C.c_void_p, C.c_int32]
    L.rf_set_pressure_solver.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    L.rf_batch_create.argtypes = [C.POINTER(C.POINTER(_abi.RfDeck)), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.rf_batch_destroy.argtypes = [C.c_void_p]
    L.rf_batch_size.argtypes = [C.c_void_p]
    L.rf_batch_context.argtypes = [C.c_void_p, C.c_int32]
    L.rf_batch_context.restype = C.c_void_p
    L.rf_batch_step.argtypes = [C.c_void_p, C.c_double, C.POINTER(_abi.RfStepReport)]
    L.rf_batch_set_mode.argtypes = [C.c_void_p, C.c_int32]
    L.rf_batch_profile.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _dp, C.c_int32]
    L.rf_dense_solve_noalloc.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p,
                                         C.c_size_t]
    L.rf_set_controller_options.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_double]
    L.rf_set_linear_refinement.argtypes = [C.c_void_p, C.c_double, C.c_int32]
    L.rf_adjoint_record.argtypes = [C.c_void_p, C.c_int32]
    L.rf_backward.argtypes = [C.c_void_p, C.POINTER(_abi.RfObjective), _dp, _dp, _dp, C.c_int32]
    L.rf_well_count.argtypes = [C.c_void_p]
    _lib = L
    return L


def last_error(handle) -> str:
    buf = C.create_string_buffer(1024)
    load().rf_last_error(handle, buf, len(buf))
    return buf.value.decode(errors="replace")


EXPORTED_SYMBOLS = (
    "rf_create", "rf_destroy", "rf_last_error", "rf_set_state", "rf_get_state", "rf_get_well_bhp",
    "rf_step", "rf_rate_history_len", "rf_rate_history_get", "rf_linear_solve_bsr", "rf_linear_solve_csr", "rf_kernel_launches",
    "rf_profile", "rf_set_linear_precision", "rf_set_cluster_size", "rf_batch_create", "rf_batch_destroy", "rf_batch_size",
    "rf_batch_context", "rf_batch_step", "rf_dense_solve_noalloc", "rf_set_controller_options", "rf_adjoint_record",
    "rf_backward", "rf_well_count", "rf_set_pressure_solver", "rf_batch_set_mode", "rf_batch_profile",
    "rf_set_linear_refinement",
)

PHASES = ("assembly", "well_elimination", "cpr_build", "pressure_stage", "block_ilu_smoother", "krylov", "update",
          "bicgstab_kernel", "direct_lu")
