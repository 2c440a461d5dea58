"""The direct route for small systems on the device against the oracle (GPU tests).

A full Newton system of at most 512 rows is factored densely on one thread-block cluster
(k_direct_lu) and solved, as the reference routes such systems to its sparse direct LU
(src/lib/ressim/src/fim/linear/mod.rs:15, 262-300).  The device and the oracle update every
element in the same order with the same operations, so on the linear seam their solutions are
equal bit for bit.  Through rf_step the bar is the rounding-floor bar of tests/_parity.py.
"""
import numpy as np
import pytest

from _parity import check_within_floor, oracle_runs
from oracle.oracle_py import OracleSimulator, linear_solve_csr
from ressim_b200 import ReservoirSimulator, _abi, decks, linear_solve_bsr
from test_gpu_parity import _csr_to_bsr

pytestmark = pytest.mark.gpu


def seam_system(dims, seed=11):
    deck = decks.waterflood_3d(*dims, seed=seed, rate_per_perf=20.0)
    deck.wells = []
    deck.pressure = deck.pressure + np.linspace(0.0, 30.0, deck.n_cells)
    res, ptr, col, val = OracleSimulator(deck).assemble_current(2.0)
    return deck, -res, ptr, col, val


# 120 rows (one CTA column slice per 8 rows) | 510 rows, the largest direct system | 513 rows
@pytest.mark.parametrize("dims, backend", [((5, 4, 2), 1), ((10, 17, 1), 1), ((19, 9, 1), 0)])
def test_seam_routing_and_bitwise_solution(dims, backend):
    deck, rhs, ptr, col, val = seam_system(dims)
    n = deck.n_cells
    x_cpu, rep_cpu = linear_solve_csr(ptr, col, val, rhs, n)
    gpu = ReservoirSimulator.from_deck(deck)
    x_gpu, rep_gpu = linear_solve_bsr(gpu, *_csr_to_bsr(n, ptr, col, val), rhs)
    assert rep_cpu.backend == backend and rep_gpu.backend == backend
    assert not rep_gpu.used_fallback and not rep_cpu.used_fallback
    assert rep_gpu.converged == rep_cpu.converged == 1
    assert rep_gpu.iterations == rep_cpu.iterations
    if backend == _abi.RF_BACKEND_SPARSE_LU:
        assert np.array_equal(x_gpu, x_cpu), np.max(np.abs(x_gpu - x_cpu))
        assert rep_gpu.final_residual_norm == rep_cpu.final_residual_norm
        assert rep_gpu.rhs_norm == rep_cpu.rhs_norm
    else:
        scale = max(np.max(np.abs(x_cpu)), 1.0)
        assert np.max(np.abs(x_gpu - x_cpu)) <= 1e-5 * scale


def test_seam_singular_system_falls_back_to_cpr():
    """The last cell's third equation and unknown removed: a zero pivot ends the factorisation
    and CPR-FGMRES solves the consistent system instead, on both sides."""
    deck, rhs, ptr, col, val = seam_system((5, 4, 2))
    n = deck.n_cells
    drop = 3 * n - 1
    val = val.copy()
    for r in range(3 * n):
        for k in range(ptr[r], ptr[r + 1]):
            if r == drop or col[k] == drop:
                val[k] = 0.0
    rhs = rhs.copy()
    rhs[drop] = 0.0
    x_cpu, rep_cpu = linear_solve_csr(ptr, col, val, rhs, n)
    gpu = ReservoirSimulator.from_deck(deck)
    x_gpu, rep_gpu = linear_solve_bsr(gpu, *_csr_to_bsr(n, ptr, col, val), rhs)
    assert rep_cpu.used_fallback and rep_gpu.used_fallback
    assert rep_cpu.backend == rep_gpu.backend == _abi.RF_BACKEND_FGMRES_CPR
    assert rep_gpu.converged == rep_cpu.converged
    assert rep_gpu.iterations == rep_cpu.iterations
    scale = max(np.max(np.abs(x_cpu)), 1.0)
    assert np.max(np.abs(x_gpu - x_cpu)) <= 1e-5 * scale


def run_within_floor(deck, dt, steps):
    runs = oracle_runs(deck, dt, steps)
    gpu = ReservoirSimulator.from_deck(deck)
    gpu.profile(enable=True, reset=True)
    state = {}
    for s in range(steps):
        rg = gpu.step(dt)
        gs = gpu.state()
        check_within_floor(s, gs["pressure"], gs["sat_water"], rg["newton_iterations"], runs, state=state)
    return gpu.profile()


# Small decks sit close to Newton-tolerance decisions, so the bar is the oracle's own rounding
# floor (three times the spread over summation orders, plus 1e-6), as for the mid-size deck.
def test_waterflood_1d_150_cells_direct_parity():
    """150 cells, 2 wells: 454 rows.  Near Newton convergence |b| is tiny and the 1e-12 absolute
    floor of the residual bound can reject the direct solve, so CPR-FGMRES also runs on some
    iterations, on both sides alike."""
    deck, _, _ = decks.waterflood_1d(150)
    prof = run_within_floor(deck, 2.0, 6)
    assert prof["direct_lu"] > 0.0


def test_five_spot_6x6x3_direct_parity():
    """108 cells, 5 wells, 15 perforations: 344 rows."""
    deck = decks.waterflood_3d(6, 6, 3, seed=3, rate_per_perf=5.0)
    prof = run_within_floor(deck, 5.0, 4)
    assert prof["direct_lu"] > 0.0


def test_five_spot_gravity_6x6x4_direct_parity():
    """144 cells with gravity and completion heads: 457 rows."""
    deck = decks.waterflood_3d(6, 6, 4, seed=5, dz=4.0, rate_per_perf=5.0, gravity=True)
    run_within_floor(deck, 5.0, 2)


def test_five_spot_8x7x3_small_iterative_parity():
    """504 cell rows: accepted now, and iterative because the 20 well rows take the full system
    past 512 rows."""
    deck = decks.waterflood_3d(8, 7, 3, seed=3, rate_per_perf=5.0)
    prof = run_within_floor(deck, 5.0, 4)
    assert prof["direct_lu"] == 0.0
