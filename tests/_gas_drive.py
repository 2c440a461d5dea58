"""The reference's solution-gas-drive acceptance case (three_phase_acceptance.rs:82-127, graded by
`three_phase_gas_drive_matches_opm_flow_reference`, :209-290) from the fixture
tests/golden/gas_drive_case.json (written by tests/golden/make_gas_drive_fixture.py).

A 20x1x1 row of cells at its 200 bar bubble point with 8 % free gas, produced by one BHP
producer at 100 bar in the last cell, no injector, gas redissolution on, no gravity.  The
fixture holds the setter sequence, the 20-row PVT table and the OPM Flow solution it is graded
against.  `set_fim_enabled` (the device path is FIM) and `set_stability_params` (IMPES only) are
skipped.
"""
from __future__ import annotations

import json
import os

import numpy as np

from ressim_b200 import Deck

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gas_drive_case.json")


def fixture() -> dict:
    with open(FIXTURE) as fh:
        return json.load(fh)


def gas_drive_deck() -> Deck:
    f = fixture()
    d = Deck(*f["grid"], f["porosity"])
    for kind, name, args in f["ops"]:
        if kind == "set":
            if name == "pvt_table":
                d.set_pvt_table(f["pvt_rows"])
            elif name == "injector_enabled":
                d.set_injector_enabled(args == "true")
            elif name == "pc_og":
                d.pc_og = None
            else:
                raise ValueError(f"unhandled field assignment {name}")
            continue
        if name in ("set_fim_enabled", "set_stability_params"):
            continue
        if name == "add_well":
            args = [int(args[0]), int(args[1]), int(args[2]), *args[3:]]
        getattr(d, name)(*args)
    return d


def in_place(deck: Deck) -> tuple[float, float]:
    """(stock-tank oil, free plus dissolved gas) in place [Sm3] at the saturated initial state:
    So PV / Bo and Sg PV / Bg + So PV / Bo Rs (three_phase_acceptance.rs:155-163 and the gas
    inventory it divides by), Bo and Bg from the table at each cell's pressure."""
    r = np.array(fixture()["pvt_rows"])
    p = np.asarray(deck.pressure, dtype=float)
    bo = np.interp(p, r[:, 0], r[:, 2])
    bg = np.interp(p, r[:, 0], r[:, 4])
    dz = np.repeat(np.asarray(deck.dz, dtype=float), deck.nx * deck.ny)
    pv = deck.dx * deck.dy * dz * np.asarray(deck.porosity, dtype=float)
    sg = np.asarray(deck.sat_gas, dtype=float)
    so = 1.0 - np.asarray(deck.sat_water, dtype=float) - sg
    rs = np.asarray(deck.rs, dtype=float)
    return float(np.sum(so * pv / bo)), float(np.sum(sg * pv / bg + so * pv / bo * rs))


def cumulative_oil(history) -> float:
    """three_phase_acceptance.rs:144-153."""
    total, prev = 0.0, 0.0
    for pt in history:
        total += pt["total_production_oil"] * (pt["time"] - prev)
        prev = pt["time"]
    return total


def checkpoint(history, t_ref, stoiip, giip) -> dict:
    """Relative errors of one OPM point, and the material-balance drifts, as the test asserts."""
    f = fixture()
    row = next(r for r in f["opm_series"] if r[0] == t_ref)
    _, p_ref, q_ref, cum_ref, gor_ref = row
    pt = history[-1]
    out = {"pressure": abs(pt["avg_reservoir_pressure"] - p_ref) / p_ref,
           "gor": abs(pt["producing_gor"] - gor_ref) / gor_ref,
           "cumulative_oil": abs(cumulative_oil(history) - cum_ref) / cum_ref,
           "mb_oil": abs(pt["material_balance_error_oil_m3"]) / stoiip,
           "mb_gas": abs(pt["material_balance_error_gas_m3"]) / giip}
    if q_ref >= f["scalars"]["GAS_DRIVE_MIN_GRADED_OIL_RATE_SC_DAY"]:
        out["oil_rate"] = abs(pt["total_production_oil"] - q_ref) / q_ref
    return out


TOLERANCE_KEYS = {"pressure": "GAS_DRIVE_PRESSURE_TOLERANCE", "gor": "GAS_DRIVE_GOR_TOLERANCE",
                  "cumulative_oil": "GAS_DRIVE_CUMULATIVE_OIL_TOLERANCE", "oil_rate": "GAS_DRIVE_OIL_RATE_TOLERANCE",
                  "mb_oil": "GAS_DRIVE_OIL_MATERIAL_BALANCE_TOLERANCE",
                  "mb_gas": "GAS_DRIVE_GAS_MATERIAL_BALANCE_TOLERANCE"}
