"""The direct route for small systems in the oracle (CPU tests).

The reference sends a full Newton system of at most 512 rows to a sparse direct LU before any
iterative solver, and falls back to CPR-FGMRES when that solve does not converge
(src/lib/ressim/src/fim/linear/mod.rs:15, 262-300; sparse_lu_debug.rs:148-232).  These restate
the reference's routing tests (mod.rs:416-478) on systems with the FIM layout, and check that
decks of at most 512 rows now step.
"""
import numpy as np
import pytest

from oracle.oracle_py import OracleSimulator, linear_solve_csr
from ressim_b200 import _abi, decks


def to_csr(dense):
    ptr, col, val = [0], [], []
    for r in range(dense.shape[0]):
        nz = np.nonzero(dense[r])[0]
        col.extend(nz)
        val.extend(dense[r, nz])
        ptr.append(len(col))
    return np.array(ptr), np.array(col), np.array(val)


def test_small_system_takes_the_direct_lu():
    # default_fim_solver_uses_iterative_fallback_before_sparse_lu (mod.rs:416-435), on a
    # three-cell system: converged, no fallback, direct backend, the exact solution
    rng = np.random.default_rng(1)
    a = np.eye(9) * 4.0 + 0.3 * rng.standard_normal((9, 9))
    b = rng.standard_normal(9)
    x, rep = linear_solve_csr(*to_csr(a), b, 3)
    assert rep.converged and not rep.used_fallback
    assert rep.backend == _abi.RF_BACKEND_SPARSE_LU
    assert rep.iterations == 1
    assert np.max(np.abs(x - np.linalg.solve(a, b))) < 1e-14


def test_singular_direct_solve_falls_back_to_cpr():
    # failed_forced_direct_solve_preserves_requested_cpr_fallback (mod.rs:437-458): an empty last
    # row and column makes the factorisation fail; CPR-FGMRES then converges on the consistent rhs
    rng = np.random.default_rng(1)
    a = np.eye(9) * 4.0 + 0.3 * rng.standard_normal((9, 9))
    a[:, 8] = 0.0
    a[8, :] = 0.0
    b = rng.standard_normal(9)
    b[8] = 0.0
    x, rep = linear_solve_csr(*to_csr(a), b, 3)
    assert rep.converged and rep.used_fallback
    assert rep.backend == _abi.RF_BACKEND_FGMRES_CPR


def test_system_above_512_rows_stays_iterative():
    # large_default_fim_system_still_uses_iterative_backend (mod.rs:460-478): 513 rows
    n = 513
    x, rep = linear_solve_csr(*to_csr(np.eye(n) * 2.0), np.ones(n), n // 3)
    assert rep.converged and not rep.used_fallback
    assert rep.backend == _abi.RF_BACKEND_FGMRES_CPR
    assert np.max(np.abs(x - 0.5)) < 1e-12


def test_direct_lu_refines_a_badly_scaled_solve():
    # rows scaled over 24 decades: the first solve's residual is still far below 5e-3 |b|, so the
    # report shows one solve and the residual bound
    rng = np.random.default_rng(4)
    a = np.eye(9) * 3.0 + 0.5 * rng.standard_normal((9, 9))
    a = np.diag(10.0 ** np.linspace(-12, 12, 9)) @ a
    b = a @ rng.standard_normal(9)
    x, rep = linear_solve_csr(*to_csr(a), b, 3)
    assert rep.backend == _abi.RF_BACKEND_SPARSE_LU and rep.converged
    assert rep.final_residual_norm <= 1e-12 + 5e-3 * np.linalg.norm(b)


@pytest.mark.parametrize("name", ["1d_100", "3d_6x6x3", "3d_8x7x3"])
def test_small_decks_step(name):
    """Decks of at most 512 rows (1D 100 cells: 304 rows; 6x6x3 five-spot: 344 rows) take the
    direct route; 8x7x3 (504 cell rows plus 20 well rows) stays iterative."""
    deck, dt = {
        "1d_100": (decks.waterflood_1d(100)[0], 10.0),
        "3d_6x6x3": (decks.waterflood_3d(6, 6, 3, seed=3, rate_per_perf=5.0), 5.0),
        "3d_8x7x3": (decks.waterflood_3d(8, 7, 3, seed=3, rate_per_perf=5.0), 5.0),
    }[name]
    sim = OracleSimulator(deck)
    for _ in range(3):
        rc, rep = sim.step(dt)
        assert rc == 0
        assert rep.newton_iterations > 0
    st = sim.state()
    assert np.all(np.isfinite(st["pressure"])) and np.all((st["sat_water"] >= 0.0) & (st["sat_water"] <= 1.0))
