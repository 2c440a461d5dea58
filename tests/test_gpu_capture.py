"""Replay of a captured linear system on the device seam (GPU test).

A tail-free Newton system assembled by the oracle is written in the reference's capture format,
read back, and solved by `rf_linear_solve_bsr`; the oracle solves the same re-read system.  The
bar is the linear seam's: same FGMRES iteration count and convergence flag, x within 1e-5
relative (the pressure BiCGStab stops at a 1e-6 relative residual, so summation order alone
moves x by about that much).
"""
import numpy as np
import pytest

from oracle.oracle_py import linear_solve_csr
from ressim_b200 import ReservoirSimulator, capture as cap
from test_capture import oracle_capture

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(10, 9, 3), (20, 20, 2)])
def test_replay_captured_system(tmp_path, dims):
    deck, s = oracle_capture(dims)
    cap.write_capture(tmp_path, 0, s)
    t = cap.load_captures(tmp_path)[0]
    n = deck.n_cells
    x_cpu, rep_cpu = linear_solve_csr(t.jacobian.ptr, t.jacobian.col, t.jacobian.val, t.rhs, n)
    sim = ReservoirSimulator.from_deck(deck)
    x_gpu, rep_gpu = cap.replay(sim, t)
    assert rep_gpu.iterations == rep_cpu.iterations
    assert rep_gpu.converged == rep_cpu.converged
    scale = max(np.max(np.abs(x_cpu)), 1.0)
    assert np.max(np.abs(x_gpu - x_cpu)) <= 1e-5 * scale, np.max(np.abs(x_gpu - x_cpu)) / scale


def oracle_capture_with_wells(dims, seed=11):
    """The oracle's full Newton system of a waterflood deck, well tail included, as a capture."""
    from oracle.oracle_py import OracleSimulator
    from ressim_b200 import decks

    deck = decks.waterflood_3d(*dims, seed=seed, rate_per_perf=20.0)
    deck.pressure = deck.pressure + np.linspace(0.0, 30.0, deck.n_cells)
    o = OracleSimulator(deck)
    n_wells, n_perfs = o.topology()
    res, ptr, col, val = o.assemble_current(2.0)
    o.close()
    n = deck.n_cells
    rows = 3 * n + n_wells + n_perfs
    assert len(res) == rows
    jac = cap.csr_from_arrays(rows, rows, ptr, col, val)
    lay = cap.Layout(n, 3, n_wells, 3 * n + n_wells)
    return deck, cap.CapturedSystem(0, "none", "water", 0, lay, jac, -res)


@pytest.mark.parametrize("dims,route", [((4, 4, 2), "direct"), ((10, 9, 3), "cpr")])
def test_replay_captured_system_with_well_tail(tmp_path, dims, route):
    """A full system with its well tail (111 rows: the direct LU; 830 rows: well elimination,
    CPR-FGMRES and tail recovery) replays through rf_linear_solve_csr: the same iteration count
    and convergence flag as the oracle, x within 1e-5 relative (1e-8 on the direct route)."""
    deck, s = oracle_capture_with_wells(dims)
    cap.write_capture(tmp_path, 0, s)
    t = cap.load_captures(tmp_path)[0]
    assert (t.jacobian.rows <= 512) == (route == "direct")
    x_cpu, rep_cpu = linear_solve_csr(t.jacobian.ptr, t.jacobian.col, t.jacobian.val, t.rhs, deck.n_cells)
    sim = ReservoirSimulator.from_deck(deck)
    x_gpu, rep_gpu = cap.replay(sim, t)
    assert rep_gpu.converged == rep_cpu.converged == 1
    assert rep_gpu.iterations == rep_cpu.iterations
    assert rep_gpu.used_fallback == rep_cpu.used_fallback
    scale = max(np.max(np.abs(x_cpu)), 1.0)
    err = np.max(np.abs(x_gpu - x_cpu)) / scale
    print(f"{route}: {t.jacobian.rows} rows, {rep_gpu.iterations} iterations, x within {err:.2e}")
    assert err <= (1e-8 if route == "direct" else 1e-5), err
    # the tail itself (well BHP and perforation rate corrections) carries the same bar
    n3 = 3 * deck.n_cells
    terr = np.max(np.abs(x_gpu[n3:] - x_cpu[n3:])) / max(np.max(np.abs(x_cpu[n3:])), 1.0)
    assert terr <= (1e-8 if route == "direct" else 1e-5), terr
    sim.close()


def test_full_system_seam_rejects_entries_outside_the_well_couplings():
    from ressim_b200.simulator import DeviceError, linear_solve_csr as seam

    deck, s = oracle_capture_with_wells((4, 4, 2))
    j = s.jacobian
    a = j.to_dense()
    n3 = 3 * deck.n_cells
    sim = ReservoirSimulator.from_deck(deck)
    x, rep = seam(sim, j.ptr, j.col, j.val, s.rhs)
    assert rep.converged

    def csr(m):
        r, c = np.nonzero(m)
        ptr_ = np.searchsorted(r, np.arange(m.shape[0] + 1)).astype(np.int32)
        return ptr_, c.astype(np.int32), m[r, c]

    bad = a.copy()
    bad[0, n3] = 1.0  # a cell row coupled to a well BHP
    with pytest.raises(DeviceError, match="outside"):
        seam(sim, *csr(bad), s.rhs)
    bad = a.copy()
    last = a.shape[0] - 1
    bad[last, last] = 2.0  # a perforation row's rate coefficient
    with pytest.raises(DeviceError, match="diagonal"):
        seam(sim, *csr(bad), s.rhs)
    with pytest.raises(DeviceError, match="rows"):
        seam(sim, j.ptr[:-1], j.col, j.val, s.rhs[:-1])
    # the context stays usable: the same system solves again to the same answer
    x2, _ = seam(sim, j.ptr, j.col, j.val, s.rhs)
    assert np.array_equal(x, x2)
    sim.close()
