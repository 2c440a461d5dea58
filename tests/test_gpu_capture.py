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
