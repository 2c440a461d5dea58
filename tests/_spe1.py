"""SPE1 Case 1 (Odeh 1981) as the reference's acceptance test builds and grades it, from the fixture
tests/golden/spe1_case.json (written by tests/golden/make_spe1_fixture.py from
src/lib/ressim/src/lib.rs `make_spe1_like_grid_sim` and src/lib/ressim/src/tests/
spe1_acceptance.rs).

- `spe1_deck(nx)` replays the helper's setter calls on a `Deck`: the 3048 m square domain in
  nx x nx x 3 cells, per-layer thickness and permeability, the SPE1 PVT table (set as the helper
  sets it, with the oil compressibility of the time, before the initial Rs), SWOF/SGOF tables,
  gas injection at a surface-rate target in the corner cell of the top layer, an oil surface-rate
  producer with a BHP limit in the opposite corner of the bottom layer, gas redissolution off.
  `set_stability_params` only feeds the IMPES path and is skipped.
- `checkpoint_errors` / `material_balance_drift` restate the acceptance test's measures
  (spe1_acceptance.rs:112-123, 151-201, 244-275).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from ressim_b200 import Deck

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "spe1_case.json")


def fixture() -> dict:
    with open(FIXTURE) as fh:
        return json.load(fh)


def spe1_deck(nx: int = 10) -> Deck:
    f = fixture()
    d = Deck(nx, nx, f["nz"], f["porosity"])
    env = {"cell_dx": f["domain_m"] / nx, "cell_dy": f["domain_m"] / nx, "producer_i": nx - 1,
           "producer_j": nx - 1, "layer_perms_z": f["acceptance_layer_perms_z"]}
    for name, args in f["calls"]:
        if name == "set_stability_params":
            continue
        args = [env[a[1:]] if isinstance(a, str) and a.startswith("$") else a for a in args]
        if name == "set_initial_rs":
            # `sim.pvt_table = Some(PvtTable::new(rows, sim.pvt.c_o))` precedes it in the helper
            d.set_pvt_table(f["pvt_rows"])
        if name == "add_well":
            args = [int(args[0]), int(args[1]), int(args[2]), *args[3:]]
        getattr(d, name)(*args)
        if name == "set_three_phase_rel_perm_props":
            d.set_three_phase_scal_tables(f["swof"], f["sgof"])
    return d


def interpolate(series, t):
    """spe1_acceptance.rs:107-123."""
    if t <= series[0][0]:
        return series[0][1]
    for (t0, v0), (t1, v1) in zip(series, series[1:]):
        if t <= t1:
            return v0 + (v1 - v0) * (t - t0) / (t1 - t0)
    return series[-1][1]


def checkpoint_errors(point: dict, t: float) -> dict:
    s = fixture()["series"]
    ref = {"pressure": interpolate(s["REF_PRESSURE_BAR"], t), "oil_rate": interpolate(s["REF_OIL_RATE"], t),
           "gor": interpolate(s["REF_GOR"], t)}
    got = {"pressure": point["avg_reservoir_pressure"], "oil_rate": point["total_production_oil"],
           "gor": point["producing_gor"]}
    return {k: abs(got[k] - ref[k]) / ref[k] for k in ref}


def _bo_undersaturated(rows, c_o, p, rs):
    """Bo of oil holding `rs` at pressure `p` above its bubble point: the saturated Bo at the
    bubble point, shrunk by the table's undersaturated compressibility (a denominator only)."""
    r = np.array(rows)
    pb = float(np.interp(rs, r[:, 1], r[:, 0]))
    bob = float(np.interp(pb, r[:, 0], r[:, 2]))
    return bob * math.exp(-c_o * max(p - pb, 0.0))


def in_place(deck: Deck) -> tuple[float, float]:
    """(stock-tank oil, total surface gas) initially in place [Sm3], as spe1_acceptance.rs:151-173
    sums them over cells: So PV / Bo and Sg PV / Bg + So PV / Bo Rs."""
    f = fixture()
    n = deck.n_cells
    dz = np.repeat(np.asarray(deck.dz, dtype=float), deck.nx * deck.ny)
    pv = deck.dx * deck.dy * dz * np.asarray(deck.porosity, dtype=float)
    so = 1.0 - np.asarray(deck.sat_water, dtype=float)
    bo = np.array([_bo_undersaturated(f["pvt_rows"], deck.pvt_c_o, float(deck.pressure[i]), float(deck.rs[i]))
                   for i in range(n)])
    oil = float(np.sum(so * pv / bo))
    gas = float(np.sum(so * pv / bo * np.asarray(deck.rs, dtype=float)))
    return oil, gas


def material_balance_drift(point: dict, time_days: float, stoiip: float, giip: float) -> tuple[float, float]:
    """spe1_acceptance.rs:244-275: oil drift over STOIIP, gas drift over gas handled."""
    s = fixture()["scalars"]
    oil = abs(point["material_balance_error_oil_m3"]) / stoiip
    gas = abs(point["material_balance_error_gas_m3"]) / (giip + s["TARGET_GAS_INJECTION_SC_DAY"] * time_days)
    return oil, gas
