"""The allocation-free dense pressure solve (rf_dense_solve_noalloc) against the existing linear
solver entry point (GPU tests).  This file is collected last on purpose.

rf_dense_solve_noalloc exists for callers that may not call cudaMalloc themselves or have it
called for them (a host that reserves its device memory up front, an embedding framework that
owns the allocator).  It runs the context's dense coarse-solve kernels with fixed scratch.  The
test builds a block system whose only coupling sits in the pressure unknowns. On that system the
CPR-FGMRES of rf_linear_solve_bsr reduces to the same dense pressure inverse (the grid has 270
cells, under the 299-row dense threshold), so both entry points must return the same pressure
solution.  The device buffers below belong to the test; the entry point itself allocates none.
"""
import numpy as np
import pytest
import torch

from ressim_b200 import ReservoirSimulator, decks, linear_solve_bsr
from ressim_b200.simulator import DeviceError, dense_solve_noalloc

pytestmark = pytest.mark.gpu

DIMS = (10, 9, 3)  # 270 cells


def _pressure_system(nx, ny, nz, seed):
    """A diagonally dominant 7-point pressure matrix P (dense) and the tail-free 3x3 block system
    whose (0,0) entries are P, whose other unknowns are identity rows, plus a right-hand side."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    P = np.zeros((n, n))
    rp, cols, vals = [0], [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                r = (k * ny + j) * nx + i
                nb = []
                for di, dj, dk in ((0, 0, -1), (0, -1, 0), (-1, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)):
                    ii, jj, kk = i + di, j + dj, k + dk
                    if 0 <= ii < nx and 0 <= jj < ny and 0 <= kk < nz:
                        nb.append((kk * ny + jj) * nx + ii)
                for c in nb:
                    P[r, c] = -1.0 + 0.3 * rng.random()
                P[r, r] = 7.0 + rng.random()
                for c in sorted(nb + [r]):
                    blk = np.zeros(9)
                    blk[0] = P[r, c]
                    if c == r:
                        blk[4] = blk[8] = 1.0
                    cols.append(c)
                    vals.append(blk)
                rp.append(len(cols))
    rhs = np.zeros(3 * n)
    rhs[0::3] = rng.standard_normal(n) * 10.0
    rhs[1::3] = rng.standard_normal(n)
    rhs[2::3] = rng.standard_normal(n)
    return P, np.array(rp), np.array(cols), np.concatenate(vals), rhs


def _noalloc(P, b):
    n = P.shape[0]
    a_d = torch.tensor(P, dtype=torch.float64, device="cuda")
    b_d = torch.tensor(b, dtype=torch.float64, device="cuda")
    x_d = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    dense_solve_noalloc(n, a_d.data_ptr(), b_d.data_ptr(), x_d.data_ptr())
    torch.cuda.synchronize()
    return x_d.cpu().numpy()


def test_noalloc_dense_solve_matches_linear_solver_on_two_calls():
    deck = decks.waterflood_3d(*DIMS, seed=11, rate_per_perf=20.0)
    deck.wells = []
    sim = ReservoirSimulator.from_deck(deck)
    for seed in (1, 2):  # two calls in a row, different systems: no state may leak between them
        P, rp, cols, vals, rhs = _pressure_system(*DIMS, seed)
        x_ref, rep = linear_solve_bsr(sim, rp, cols, vals, rhs)
        assert rep.converged
        x = _noalloc(P, rhs[0::3])
        scale = max(float(np.max(np.abs(x_ref[0::3]))), 1.0)
        assert np.all(np.isfinite(x))
        assert np.max(np.abs(x - x_ref[0::3])) <= 1e-9 * scale, np.max(np.abs(x - x_ref[0::3])) / scale
        assert np.max(np.abs(P @ x - rhs[0::3])) <= 1e-9 * max(float(np.max(np.abs(rhs))), 1.0)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    n = 300
    a_d = torch.eye(n, dtype=torch.float64, device="cuda")
    b_d = torch.ones(n, dtype=torch.float64, device="cuda")
    x_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(DeviceError, match="299"):
        dense_solve_noalloc(n, a_d.data_ptr(), b_d.data_ptr(), x_d.data_ptr())


def test_noalloc_singular_matrix_fails_cleanly_and_leaves_x_unchanged():
    """A matrix with an all-zero first column has an exactly zero first pivot: the call reports
    the singular matrix, x keeps the caller's values, and the next call on a good system is still
    correct (the shared scratch carries nothing over)."""
    n = 40
    rng = np.random.default_rng(3)
    A = rng.standard_normal((n, n)) + n * np.eye(n)
    A[:, 0] = 0.0
    a_d = torch.tensor(A, dtype=torch.float64, device="cuda")
    b_d = torch.ones(n, dtype=torch.float64, device="cuda")
    x_d = torch.full((n,), 7.5, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(DeviceError, match="singular"):
        dense_solve_noalloc(n, a_d.data_ptr(), b_d.data_ptr(), x_d.data_ptr())
    torch.cuda.synchronize()
    assert np.all(x_d.cpu().numpy() == 7.5)
    G = rng.standard_normal((n, n)) + n * np.eye(n)
    rhs = rng.standard_normal(n)
    x = _noalloc(G, rhs)
    assert np.max(np.abs(G @ x - rhs)) <= 1e-10 * max(float(np.max(np.abs(rhs))), 1.0)
