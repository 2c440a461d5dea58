"""Device FIM path vs the CPU oracle on the same seeded decks (GPU tests).

Parity bar: pressure, water saturation, well BHP and well rates within 1e-6 relative after every
report step, and Newton iteration counts within one per report step.  Where the reference's own
rounding moves a run by more than that (pressure BiCGStab stopped at its iteration cap), the bar
is three times the oracle-vs-oracle difference under a changed summation order, plus 1e-6.
"""
import numpy as np
import pytest

from _parity import check_within_floor, oracle_runs, rel_err
from oracle.oracle_py import OracleSimulator, linear_solve_csr
from ressim_b200 import ReservoirSimulator, decks, linear_solve_bsr

pytestmark = pytest.mark.gpu

FIELD_RTOL = 1e-6


def run_pair(deck, dt, steps):
    gpu = ReservoirSimulator.from_deck(deck)
    cpu = OracleSimulator(deck)
    rows = []
    for s in range(steps):
        rg = gpu.step(dt)
        rc_, rc = cpu.step(dt)
        assert rc_ == 0, f"oracle warning at step {s}"
        gs, cs = gpu.state(), cpu.state()
        rows.append({
            "step": s,
            "p": rel_err(gs["pressure"], cs["pressure"]),
            "sw": rel_err(gs["sat_water"], cs["sat_water"]),
            "bhp": rel_err(gpu.get_well_bhp(), cpu.well_bhp()),
            "newton_gpu": rg["newton_iterations"],
            "newton_cpu": rc.newton_iterations,
            "substeps_gpu": rg["substeps"],
            "substeps_cpu": rc.substeps,
        })
    hg, hc = gpu.get_rate_history(), cpu.rate_history()
    return gpu, cpu, rows, hg, hc


def check_rows(rows, hg, hc):
    for r in rows:
        assert r["p"] < FIELD_RTOL, r
        assert r["sw"] < FIELD_RTOL, r
        assert r["bhp"] < FIELD_RTOL, r
        assert abs(r["newton_gpu"] - r["newton_cpu"]) <= 1, r
    assert len(hg) == len(hc)
    for a, b in zip(hg, hc):
        for key in ("total_production_oil", "total_injection", "total_production_liquid_reservoir",
                    "avg_reservoir_pressure", "avg_water_saturation"):
            assert abs(a[key] - b[key]) <= FIELD_RTOL * max(abs(b[key]), 1.0), (key, a, b)


def test_waterflood_1d_parity():
    deck, dt, _ = decks.waterflood_1d()
    gpu, cpu, rows, hg, hc = run_pair(deck, dt, 12)
    check_rows(rows, hg, hc)
    assert gpu.kernel_launches() > 0


def test_waterflood_3d_small_parity():
    deck = decks.waterflood_3d(12, 10, 3, seed=3, rate_per_perf=20.0)
    gpu, cpu, rows, hg, hc = run_pair(deck, 5.0, 4)
    check_rows(rows, hg, hc)


def test_waterflood_3d_bicgstab_parity():
    # 20 x 20 x 2 = 800 coarse rows: the pressure stage runs the device BiCGStab + ILU0
    deck = decks.waterflood_3d(20, 20, 2, seed=5, rate_per_perf=40.0)
    gpu, cpu, rows, hg, hc = run_pair(deck, 10.0, 3)
    check_rows(rows, hg, hc)


def test_waterflood_3d_gravity_with_wells_parity():
    """Gravity on, with fully perforated wells whose BHPs are quoted at the shallowest completion:
    the completion heads are refreshed at every report step (12 x 10 x 4, dz 4 m)."""
    deck = decks.waterflood_3d(12, 10, 4, seed=3, dz=4.0, rate_per_perf=20.0, gravity=True)
    runs = oracle_runs(deck, 5.0, 3)
    gpu = ReservoirSimulator.from_deck(deck)
    state = {}
    for s in range(3):
        rg = gpu.step(5.0)
        gs = gpu.state()
        check_within_floor(s, gs["pressure"], gs["sat_water"], rg["newton_iterations"], runs, state=state)


def test_waterflood_3d_mid_parity_at_rounding_floor():
    """30 x 30 x 10 (9,000 cells): the pressure BiCGStab stops at its 50-iteration cap, so a
    different summation order alone moves the Newton end state by more than 1e-6 in saturation.
    The oracle run twice, with the reference's left-to-right dot products and with interleaved
    partial sums, measures that rounding floor; the device path must stay within it (x3, plus
    1e-6), with Newton counts within one.  After a report step that took one Newton iteration
    more or fewer than the oracle, the bound is the Newton tolerance (tests/_parity.py)."""
    deck = decks.waterflood_3d(30, 30, 10, seed=7)
    dt, steps = 10.0, 3
    runs = oracle_runs(deck, dt, steps)
    gpu = ReservoirSimulator.from_deck(deck)
    state = {}
    for s in range(steps):
        rg = gpu.step(dt)
        gs = gpu.state()
        check_within_floor(s, gs["pressure"], gs["sat_water"], rg["newton_iterations"], runs, state=state)


def _csr_to_bsr(n_cells, ptr, col, val):
    """Tail-free 3x3 block CSR from a scalar CSR with 3 unknowns per cell."""
    blocks = {}
    for r in range(3 * n_cells):
        for k in range(ptr[r], ptr[r + 1]):
            c = col[k]
            if c >= 3 * n_cells:
                continue
            b = blocks.setdefault((r // 3, c // 3), np.zeros(9))
            b[3 * (r % 3) + (c % 3)] = val[k]
    rp, cols, vals = [0], [], []
    for i in range(n_cells):
        row = sorted(j for (ii, j) in blocks if ii == i)
        for j in row:
            cols.append(j)
            vals.append(blocks[(i, j)])
        rp.append(len(cols))
    return np.array(rp), np.array(cols), np.concatenate(vals)


# dense coarse inverse | BiCGStab coarse | BiCGStab over 38 levels
@pytest.mark.parametrize("dims", [(10, 9, 3), (12, 10, 3), (24, 24, 8)])
def test_linear_seam_matches_oracle(dims):
    """One CPR-FGMRES solve through rf_linear_solve_bsr against the oracle's solve of the same
    system: same iteration count and convergence flag, and x within 1e-5 relative.  The pressure
    stage stops BiCGStab at a residual of 1e-6 relative, so the correction it returns is only
    determined to about that level; any change of summation order moves x by up to ~1e-6."""
    deck = decks.waterflood_3d(*dims, seed=11, rate_per_perf=20.0)
    deck.wells = []  # tail-free system
    deck.pressure = deck.pressure + np.linspace(0.0, 30.0, deck.n_cells)
    cpu = OracleSimulator(deck)
    res, ptr, col, val = cpu.assemble_current(2.0)
    n = deck.n_cells
    rhs = -res[: 3 * n]
    x_cpu, rep_cpu = linear_solve_csr(ptr, col, val, -res, n)
    gpu = ReservoirSimulator.from_deck(deck)
    rp, cols, vals = _csr_to_bsr(n, ptr, col, val)
    x_gpu, rep_gpu = linear_solve_bsr(gpu, rp, cols, vals, rhs)
    assert rep_gpu.iterations == rep_cpu.iterations
    assert rep_gpu.converged == rep_cpu.converged
    scale = max(np.max(np.abs(x_cpu)), 1.0)
    assert np.max(np.abs(x_gpu - x_cpu)) <= 1e-5 * scale, np.max(np.abs(x_gpu - x_cpu)) / scale
