"""Three-phase black-oil decks: the device FIM path against the CPU oracle (GPU tests).

Parity bar as for the two-phase decks: pressure, water saturation, gas saturation, Rs and well
BHP within 1e-6 relative after every report step with the Newton counts within one, on decks
small enough for the direct route and on decks whose pressure stage runs the BiCGStab; where the
pressure BiCGStab stops at its iteration cap, three times the oracle's own rounding floor.
"""
import numpy as np
import pytest

from _parity import rel_err
from oracle.oracle_py import OracleSimulator, lib
from ressim_b200 import Ensemble, ReservoirSimulator, decks

pytestmark = pytest.mark.gpu

RTOL = 1e-6
FIELDS = ("pressure", "sat_water", "sat_gas", "rs")


def _fields_err(gs, cs):
    return {k: rel_err(gs[k], cs[k]) for k in FIELDS}


def run_pair(deck, dt, steps):
    gpu = ReservoirSimulator.from_deck(deck)
    cpu = OracleSimulator(deck)
    rows = []
    for s in range(steps):
        rg = gpu.step(dt)
        rc_, rc = cpu.step(dt)
        assert rc_ == 0, f"oracle warning at step {s}"
        e = _fields_err(gpu.state(), cpu.state())
        e["bhp"] = rel_err(gpu.get_well_bhp(), cpu.well_bhp())
        e["newton"] = (rg["newton_iterations"], rc.newton_iterations)
        print(f"step {s}: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items() if k != "newton") +
              f", newton {e['newton']}")
        rows.append(e)
    return gpu, cpu, rows


def check(rows, tol=RTOL):
    for e in rows:
        for k in (*FIELDS, "bhp"):
            assert e[k] < tol, e
        assert abs(e["newton"][0] - e["newton"][1]) <= 1, e


def test_blackoil_small_direct_route_parity():
    """6 x 6 x 2 (216 + 10 well unknowns): the Newton systems take the direct LU route; gas comes
    out of solution near the producer."""
    deck = decks.black_oil_3d(6, 6, 2, seed=4, rate_per_perf=10.0)
    gpu, cpu, rows = run_pair(deck, 5.0, 4)
    check(rows)
    assert np.max(gpu.state()["sat_gas"]) > 0.01
    hg, hc = gpu.get_rate_history(), cpu.rate_history()
    assert len(hg) == len(hc)
    for a, b in zip(hg, hc):
        for key in ("total_production_oil", "total_production_gas", "total_injection", "avg_reservoir_pressure",
                    "avg_water_saturation", "avg_gas_saturation", "producing_gor"):
            assert abs(a[key] - b[key]) <= RTOL * max(abs(b[key]), 1.0), (key, a[key], b[key])


def test_blackoil_gas_injection_with_gas_oil_pc_parity():
    deck = decks.black_oil_3d(5, 5, 2, seed=6, rate_per_perf=400.0, pc_og=True, injected_fluid="gas")
    gpu, cpu, rows = run_pair(deck, 5.0, 3)
    check(rows)


def test_blackoil_cpr_bicgstab_parity():
    """14 x 14 x 4 (784 cells): CPR-FGMRES with the device pressure BiCGStab + ILU0."""
    deck = decks.black_oil_3d(14, 14, 4, seed=8, rate_per_perf=15.0)
    runs = {}
    try:
        for mode in (0, 2, 61):
            lib().orc_set_sum_order(mode)
            o = OracleSimulator(deck)
            runs[mode] = []
            for _ in range(3):
                rc, r = o.step(5.0)
                assert rc == 0
                runs[mode].append((o.state(), r.newton_iterations))
            o.close()
    finally:
        lib().orc_set_sum_order(0)
    gpu = ReservoirSimulator.from_deck(deck)
    diverged = False
    for s in range(3):
        rg = gpu.step(5.0)
        gs = gpu.state()
        ref, n0 = runs[0][s]
        for k in FIELDS:
            floor = max(rel_err(runs[m][s][0][k], ref[k]) for m in runs if m != 0)
            err = rel_err(gs[k], ref[k])
            print(f"step {s} {k}: {err:.2e} (floor {floor:.2e}), newton {rg['newton_iterations']} vs {n0}")
            if diverged:
                assert err <= (1e-4 if k == "pressure" else 2e-3), (s, k, err)
            else:
                assert err <= 3 * floor + RTOL, (s, k, err, floor)
        assert abs(rg["newton_iterations"] - n0) <= 1
        diverged = diverged or rg["newton_iterations"] != n0


def test_blackoil_batch_equals_sequential_runs():
    """Three-phase variants of uneven size stepped concurrently in one batch give exactly the
    results of the same decks stepped one by one."""
    ds = [decks.black_oil_3d(6, 5, 2, seed=11, rate_per_perf=10.0), decks.black_oil_3d(9, 7, 3, seed=12)]
    ens = Ensemble(ds, host_threads=2)
    singles = [ReservoirSimulator.from_deck(d) for d in ds]
    for _ in range(2):
        reps = ens.step(5.0)
        for i, s in enumerate(singles):
            r = s.step(5.0)
            assert reps[i]["newton_iterations"] == r["newton_iterations"]
    for i, s in enumerate(singles):
        a, b = ens.state(i), s.state()
        for k in FIELDS:
            assert np.array_equal(a[k], b[k]), k
    ens.close()


def test_blackoil_mixed_precision_error_vs_fp64_oracle():
    """The mixed form (FP32 block-ILU0 and pressure stage under FP64 FGMRES) on a three-phase deck:
    its field error against the FP64 oracle, printed per report step, stays within the Newton
    tolerance's reach."""
    deck = decks.black_oil_3d(14, 14, 4, seed=8, rate_per_perf=15.0)
    gpu = ReservoirSimulator.from_deck(deck)
    gpu.set_linear_precision("mixed")
    cpu = OracleSimulator(deck)
    for s in range(3):
        rg = gpu.step(5.0)
        rc_, rc = cpu.step(5.0)
        assert rc_ == 0
        e = _fields_err(gpu.state(), cpu.state())
        print(f"mixed step {s}: " + ", ".join(f"{k} {v:.2e}" for k, v in e.items()) +
              f", newton {rg['newton_iterations']} vs {rc.newton_iterations}")
        assert e["pressure"] < 1e-3 and e["sat_water"] < 1e-2 and e["sat_gas"] < 1e-2


def test_blackoil_drsdt0_parity():
    """Gas redissolution off (DRSDT0): Rs capped at each cell's Rs at the substep start in the
    flash, the regimes, the properties and the write-back; gas that comes out stays out."""
    deck = decks.black_oil_3d(6, 6, 2, seed=4, rate_per_perf=10.0)
    deck.set_gas_redissolution_enabled(False)
    gpu, cpu, rows = run_pair(deck, 5.0, 4)
    check(rows)
    assert np.max(gpu.state()["sat_gas"]) > 0.01


def test_blackoil_scal_tables_parity():
    """SWOF/SGOF tables in place of the three-phase Corey curves (relperm.rs:391-429)."""
    from test_blackoil_rows import _tables

    deck = _tables(decks.black_oil_3d(6, 6, 2, seed=4, rate_per_perf=10.0))
    gpu, cpu, rows = run_pair(deck, 5.0, 4)
    check(rows)


def test_spe1_on_device_matches_oracle_and_published_series():
    """The reference's SPE1 acceptance test (spe1_acceptance.rs:277-396) replayed on the device:
    ten years of 30-day report steps on the 10x10x3 deck (SWOF/SGOF tables, gas injection at a
    surface target, oil surface-rate producer, DRSDT0).  At every year end the device's own rate
    history lies within the reference test's bands of the published pressure, oil rate and GOR
    with material-balance drift within 1 %, and its fields match the oracle's: within 1e-6 while
    every report step took the oracle's Newton count, within the Newton tolerance's reach after."""
    from _spe1 import checkpoint_errors, fixture, in_place, material_balance_drift, spe1_deck

    sc = fixture()["scalars"]
    deck = spe1_deck(10)
    stoiip, giip = in_place(deck)
    gpu = ReservoirSimulator.from_deck(deck)
    cpu = OracleSimulator(deck)
    t = 0.0
    same_path = True
    for year in range(1, 11):
        target = 365.0 * year
        while t < target - 1e-9:
            dt = min(30.0, target - t)
            rg = gpu.step(dt)
            rc_, rc = cpu.step(dt)
            assert rc_ == 0 and rg["warning"] == 0, (t, rc_, rg["warning"])
            same_path = same_path and rg["newton_iterations"] == rc.newton_iterations
            t = rg["time_days"]
        e = _fields_err(gpu.state(), cpu.state())
        pg, pc = gpu.get_rate_history()[-1], cpu.rate_history()[-1]
        acc = checkpoint_errors(pg, target)
        oil, gas = material_balance_drift(pg, t, stoiip, giip)
        print(f"t={target:7.1f} device vs published: pressure {100 * acc['pressure']:.3f}% oil rate "
              f"{100 * acc['oil_rate']:.3f}% GOR {100 * acc['gor']:.3f}%; vs oracle: "
              + ", ".join(f"{k} {v:.1e}" for k, v in e.items())
              + f", GOR {abs(pg['producing_gor'] - pc['producing_gor']) / pc['producing_gor']:.1e}, same Newton path {same_path}")
        assert acc["pressure"] <= sc["PRESSURE_TOLERANCE"] and acc["oil_rate"] <= sc["OIL_RATE_TOLERANCE"]
        assert acc["gor"] <= sc["GOR_TOLERANCE"]
        assert oil <= sc["OIL_MATERIAL_BALANCE_TOLERANCE"] and gas <= sc["GAS_MATERIAL_BALANCE_TOLERANCE"]
        tol = RTOL if same_path else 1e-3
        for k in FIELDS:
            assert e[k] <= tol, (target, k, e[k], same_path)
    gpu.close()
    cpu.close()


def test_gas_drive_on_device_matches_oracle_and_opm_flow():
    """The reference's solution-gas-drive acceptance case (three_phase_acceptance.rs:209-290) on
    the device: inside every band of the reference test at the eleven OPM Flow points, with the
    fields within 1e-6 of the oracle at each."""
    from _gas_drive import TOLERANCE_KEYS, checkpoint, fixture, gas_drive_deck, in_place

    f = fixture()
    deck = gas_drive_deck()
    stoiip, giip = in_place(deck)
    gpu = ReservoirSimulator.from_deck(deck)
    cpu = OracleSimulator(deck)
    t = 0.0
    for row in f["opm_series"]:
        while t < row[0] - 1e-9:
            dt = min(f["max_dt_days"], row[0] - t)
            rg = gpu.step(dt)
            rc_, rc = cpu.step(dt)
            assert rc_ == 0 and rg["warning"] == 0
            assert abs(rg["newton_iterations"] - rc.newton_iterations) <= 1
            t = rg["time_days"]
        e = checkpoint(gpu.get_rate_history(), row[0], stoiip, giip)
        fe = _fields_err(gpu.state(), cpu.state())
        print(f"t={row[0]:6.1f} " + " ".join(f"{k} {100 * v:.3f}%" for k, v in e.items()) + "; vs oracle "
              + ", ".join(f"{k} {v:.1e}" for k, v in fe.items()))
        for k, v in e.items():
            assert v <= f["scalars"][TOLERANCE_KEYS[k]], (row[0], k, v)
        for k in FIELDS:
            assert fe[k] <= RTOL, (row[0], k, fe[k])
    gpu.close()
    cpu.close()
