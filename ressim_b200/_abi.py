"""ctypes mirror of include/ressim_fim.h (the C ABI of the device FIM library)."""
from __future__ import annotations

import ctypes as C

RF_ABI_VERSION = 4
RF_BACKEND_FGMRES_CPR = 0
RF_BACKEND_SPARSE_LU = 1

RF_OK = 0
RF_STEP_WARNING = 1
RF_ERR_INVALID = -1
RF_ERR_UNSUPPORTED = -2
RF_ERR_CUDA = -3
RF_ERR_DEVICE_STATUS = -4
RF_PRECISION_FP64 = 0
RF_PRECISION_MIXED = 1

_dp = C.POINTER(C.c_double)


class RfWell(C.Structure):
    _fields_ = [
        ("i", C.c_int32), ("j", C.c_int32), ("k", C.c_int32),
        ("injector", C.c_int32),
        ("physical_well_id", C.c_int32),
        ("has_schedule", C.c_int32),
        ("schedule_enabled", C.c_int32),
        ("schedule_control", C.c_int32),
        ("bhp", C.c_double),
        ("well_radius", C.c_double),
        ("skin", C.c_double),
        ("schedule_target_rate", C.c_double),
        ("schedule_target_surface_rate", C.c_double),
        ("schedule_bhp_limit", C.c_double),
        ("datum_depth_m", C.c_double),
        ("wellbore_density_kg_m3", C.c_double),
    ]


class RfDeck(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double),
        ("dz", _dp), ("porosity", _dp), ("perm_x", _dp), ("perm_y", _dp), ("perm_z", _dp),
        ("mu_o", C.c_double), ("mu_w", C.c_double), ("c_o", C.c_double), ("c_w", C.c_double),
        ("rho_o", C.c_double), ("rho_w", C.c_double),
        ("b_o", C.c_double), ("b_w", C.c_double),
        ("water_pvt_reference_pressure_bar", C.c_double),
        ("rock_compressibility", C.c_double),
        ("rock_reference_pressure_bar", C.c_double),
        ("depth_reference_m", C.c_double),
        ("gravity_enabled", C.c_int32),
        ("s_wc", C.c_double), ("s_or", C.c_double), ("n_w", C.c_double), ("n_o", C.c_double),
        ("k_rw_max", C.c_double), ("k_ro_max", C.c_double),
        ("corey_table_points", C.c_int32),
        ("pc_entry", C.c_double), ("pc_lambda", C.c_double),
        ("n_wells", C.c_int32),
        ("wells", C.POINTER(RfWell)),
        ("injector_rate_controlled", C.c_int32),
        ("producer_rate_controlled", C.c_int32),
        ("injector_enabled", C.c_int32),
        ("target_injector_rate_m3_day", C.c_double),
        ("target_producer_rate_m3_day", C.c_double),
        ("target_injector_surface_rate_m3_day", C.c_double),
        ("target_producer_surface_rate_m3_day", C.c_double),
        ("well_bhp_min", C.c_double), ("well_bhp_max", C.c_double),
        ("three_phase_mode", C.c_int32),
        ("injected_fluid", C.c_int32),
        ("n_pvt_rows", C.c_int32),
        ("pvt_rows", _dp),
        ("pvt_c_o", C.c_double),
        ("has_scal_3p", C.c_int32),
        ("s_wc_3p", C.c_double), ("s_or_3p", C.c_double), ("n_w_3p", C.c_double), ("n_o_3p", C.c_double),
        ("k_rw_max_3p", C.c_double), ("k_ro_max_3p", C.c_double),
        ("s_gc", C.c_double), ("s_gr", C.c_double), ("s_org", C.c_double), ("n_g", C.c_double),
        ("k_rg_max", C.c_double),
        ("has_pc_og", C.c_int32),
        ("pc_og_entry", C.c_double), ("pc_og_lambda", C.c_double),
        ("mu_g", C.c_double), ("c_g", C.c_double), ("rho_g", C.c_double),
        ("gas_redissolution_enabled", C.c_int32),
        ("n_swof_rows", C.c_int32), ("swof_rows", C.POINTER(C.c_double)),
        ("n_sgof_rows", C.c_int32), ("sgof_rows", C.POINTER(C.c_double)),
    ]


class RfStepReport(C.Structure):
    _fields_ = [
        ("substeps", C.c_int32), ("retries", C.c_int32), ("newton_iterations", C.c_int32),
        ("linear_iterations", C.c_int32), ("linear_solves", C.c_int32), ("warning", C.c_int32),
        ("time_days", C.c_double), ("advanced_days", C.c_double), ("last_dt_days", C.c_double),
        ("device_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class RfTimePointRates(C.Structure):
    _fields_ = [(name, C.c_double) for name in (
        "time", "total_production_oil", "total_production_liquid",
        "total_production_liquid_reservoir", "total_injection", "total_injection_reservoir",
        "material_balance_error_m3", "material_balance_error_oil_m3", "avg_reservoir_pressure",
        "avg_water_saturation", "producer_bhp_limited_fraction", "injector_bhp_limited_fraction",
        "total_production_gas", "avg_gas_saturation", "material_balance_error_gas_m3", "producing_gor",
    )]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class RfLinearReport(C.Structure):
    _fields_ = [
        ("converged", C.c_int32), ("iterations", C.c_int32),
        ("rhs_norm", C.c_double), ("final_residual_norm", C.c_double),
        ("used_fallback", C.c_int32), ("backend", C.c_int32),
    ]


RF_OBJECTIVE_CUMULATIVE_OIL = 0


class RfObjective(C.Structure):
    _fields_ = [("kind", C.c_int32)]
