"""The single-CTA level-order kernels (pressure BiCGStab, block-ILU0 sweep) against the cluster
kernels and the oracle (GPU tests).

Both kernel families compute the reference's preconditioner: the same ILU0 factors, applied by
sweeps whose rows take the reference's operations in the reference's order.  The solves differ
only in the order their dot products are summed, so their results agree to the BiCGStab's own
stopping tolerance, and each agrees with the oracle at the parity bar of the other device tests.
The decks carry fully perforated wells, whose fill gives the sweeps rows longer than the 7-point
stencil's and dependencies more than one level away (the far-row cache of the kernels).
"""
import numpy as np
import pytest

from _parity import rel_err
from oracle.oracle_py import OracleSimulator, linear_solve_csr
from ressim_b200 import ReservoirSimulator, decks, linear_solve_bsr
from ressim_b200.simulator import DeviceError

pytestmark = pytest.mark.gpu


def _csr_to_bsr(n_cells, ptr, col, val):
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
        for j in sorted(j for (ii, j) in blocks if ii == i):
            cols.append(j)
            vals.append(blocks[(i, j)])
        rp.append(len(cols))
    return np.array(rp), np.array(cols), np.concatenate(vals)


@pytest.mark.parametrize("dims", [(12, 10, 3), (24, 24, 8)])
def test_level_kernel_linear_seam_matches_cluster_and_oracle(dims):
    """One CPR-FGMRES solve of the same system with each kernel family: same FGMRES iteration
    count as the oracle, x within 1e-5 of the oracle's and within 1e-6 of each other (the
    pressure BiCGStab stops at 1e-6 relative)."""
    deck = decks.waterflood_3d(*dims, seed=11, rate_per_perf=20.0)
    deck.wells = []
    deck.pressure = deck.pressure + np.linspace(0.0, 30.0, deck.n_cells)
    cpu = OracleSimulator(deck)
    res, ptr, col, val = cpu.assemble_current(2.0)
    n = deck.n_cells
    x_cpu, rep_cpu = linear_solve_csr(ptr, col, val, -res, n)
    rp, cols, vals = _csr_to_bsr(n, ptr, col, val)
    out = {}
    for kind in ("cluster", "level"):
        gpu = ReservoirSimulator.from_deck(deck)
        gpu.set_pressure_solver(kind)
        x, rep = linear_solve_bsr(gpu, rp, cols, vals, -res[: 3 * n])
        assert rep.iterations == rep_cpu.iterations, (kind, rep.iterations, rep_cpu.iterations)
        assert rep.converged == rep_cpu.converged
        out[kind] = x
        gpu.close()
    scale = max(np.max(np.abs(x_cpu)), 1.0)
    for kind, x in out.items():
        assert np.max(np.abs(x - x_cpu)) <= 1e-5 * scale, (kind, np.max(np.abs(x - x_cpu)) / scale)
    assert np.max(np.abs(out["level"] - out["cluster"])) <= 1e-6 * scale


@pytest.mark.parametrize("dims,dt,steps", [((20, 20, 2), 10.0, 3), ((16, 14, 6), 5.0, 3)])
def test_level_kernel_with_well_fill_matches_oracle(dims, dt, steps):
    """Fully perforated wells: pressure, saturation and BHP within 1e-6 of the oracle after every
    report step, Newton counts within one."""
    deck = decks.waterflood_3d(*dims, seed=5, rate_per_perf=40.0)
    gpu = ReservoirSimulator.from_deck(deck)
    gpu.set_pressure_solver("level")
    cpu = OracleSimulator(deck)
    for s in range(steps):
        rg = gpu.step(dt)
        rc, rep = cpu.step(dt)
        assert rc == 0
        gs, cs = gpu.state(), cpu.state()
        ep, es = rel_err(gs["pressure"], cs["pressure"]), rel_err(gs["sat_water"], cs["sat_water"])
        eb = rel_err(gpu.get_well_bhp(), cpu.well_bhp())
        print(f"{dims} step {s}: p {ep:.2e} sw {es:.2e} bhp {eb:.2e} newton {rg['newton_iterations']} "
              f"vs {rep.newton_iterations}")
        assert ep < 1e-6 and es < 1e-6 and eb < 1e-6, (s, ep, es, eb)
        assert abs(rg["newton_iterations"] - rep.newton_iterations) <= 1


def test_level_kernel_thread_counts_and_precisions_agree():
    """Thread counts change only the summation order of the dot products: after two report steps
    the fields agree with the cluster kernels' to 1e-6.  The mixed form runs the same kernels in
    FP32 and stays within the mixed form's bound of the FP64 results."""
    deck = decks.waterflood_3d(18, 16, 5, seed=9, rate_per_perf=30.0)
    ref = ReservoirSimulator.from_deck(deck)
    ref.set_pressure_solver("cluster")
    for _ in range(2):
        ref.step(10.0)
    p0, s0 = ref.state()["pressure"], ref.state()["sat_water"]
    for threads in (64, 160, 512):
        g = ReservoirSimulator.from_deck(deck)
        g.set_pressure_solver("level", threads)
        for _ in range(2):
            g.step(10.0)
        ep, es = rel_err(g.state()["pressure"], p0), rel_err(g.state()["sat_water"], s0)
        print(f"threads {threads}: p {ep:.2e} sw {es:.2e}")
        assert ep < 1e-6 and es < 1e-6, (threads, ep, es)
        g.close()
    m = ReservoirSimulator.from_deck(deck)
    m.set_linear_precision("mixed")
    m.set_pressure_solver("level")
    for _ in range(2):
        m.step(10.0)
    ep, es = rel_err(m.state()["pressure"], p0), float(np.max(np.abs(m.state()["sat_water"] - s0)))
    print(f"mixed: p {ep:.2e} sw {es:.2e}")
    assert ep < 1e-4 and es < 1e-3


def test_level_kernel_is_deterministic_and_validates_arguments():
    deck = decks.waterflood_3d(14, 12, 4, seed=2, rate_per_perf=25.0)
    runs = []
    for _ in range(2):
        g = ReservoirSimulator.from_deck(deck)
        g.set_pressure_solver("level", 128)
        g.step(10.0)
        runs.append(g.state()["pressure"].copy())
        with pytest.raises(DeviceError):
            g.set_pressure_solver("level", 1024)
        with pytest.raises(ValueError):
            g.set_pressure_solver("warp")
        g.close()
    assert np.array_equal(runs[0], runs[1])


@pytest.mark.parametrize("kind", ["level", "cluster"])
def test_factorisation_update_lists_equal_searching_form(kind, monkeypatch):
    """The factorisation from update lists (short rows by one thread each; a perforated cell's row
    with its well's fill, here 7 + 11 blocks, by a warp holding the row in registers) gives the
    factors of the searching form bit for bit: a deck whose wells perforate 12 layers, stepped with
    each form (RESSIM_FACTOR_RECIPES=0 keeps the searching one), ends with identical states and
    Newton counts, on both kernel families."""
    deck = decks.waterflood_3d(14, 12, 12, seed=5, rate_per_perf=30.0)
    runs = []
    for recipes in ("1", "0"):
        monkeypatch.setenv("RESSIM_FACTOR_RECIPES", recipes)
        g = ReservoirSimulator.from_deck(deck)
        g.set_pressure_solver(kind)
        newton = [g.step(5.0)["newton_iterations"] for _ in range(2)]
        runs.append((g.state(), g.get_well_bhp().copy(), newton))
        g.close()
    (s1, b1, n1), (s0, b0, n0) = runs
    assert n1 == n0, (n1, n0)
    for k in ("pressure", "sat_water"):
        assert np.array_equal(s1[k], s0[k]), k
    assert np.array_equal(b1, b0)
