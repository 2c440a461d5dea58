"""Shared parity helpers: relative field error and the oracle's own rounding floor."""
import numpy as np

from oracle.oracle_py import OracleSimulator, lib


def rel_err(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = np.maximum(np.abs(b), 1.0)
    return float(np.max(np.abs(a - b) / scale)) if a.size else 0.0


FLOOR_ORDERS = (2, 61, 256, 1031)


def oracle_runs(deck, dt, steps, orders=FLOOR_ORDERS):
    """The oracle stepped `steps` report steps with the reference's left-to-right dot products
    (mode 0) and again with each w-way interleaved summation in `orders`.  Returns {mode: [(p, sw,
    newton_iterations) per step]}; the largest difference of a reordered run from mode 0 is the
    rounding floor of the reference algorithm on that deck."""
    runs = {}
    try:
        for mode in (0, *orders):
            lib().orc_set_sum_order(mode)
            o = OracleSimulator(deck)
            runs[mode] = []
            for _ in range(steps):
                rc, r = o.step(dt)
                assert rc == 0
                st = o.state()
                runs[mode].append((st["pressure"].copy(), st["sat_water"].copy(), r.newton_iterations))
            o.close()
    finally:
        lib().orc_set_sum_order(0)
    return runs


# Once a report step ends after a different number of Newton iterations (one more or one fewer,
# which the parity bar allows), the runs stop at different points inside the Newton tolerance and
# the next substep sizes differ; from then on the fields agree to the Newton tolerance, not to the
# rounding floor.
NEWTON_TOL_P, NEWTON_TOL_SW = 1e-4, 2e-3


def check_within_floor(step, p, sw, newton, runs, rtol=1e-6, state=None):
    """Device fields within three times the rounding floor plus `rtol` while every report step so
    far took the oracle's Newton count; within the Newton tolerance after a step that did not.
    Newton count within one of the range the oracle itself takes under the reordered summations
    (where the pressure BiCGStab stops at its cap, a changed summation order alone can move a
    report step's count by more than one).  `state` (a dict carried across steps) records the
    divergence."""
    state = {} if state is None else state
    p0, sw0, n0 = runs[0][step]
    fp = max(rel_err(runs[m][step][0], p0) for m in runs if m != 0)
    fs = max(rel_err(runs[m][step][1], sw0) for m in runs if m != 0)
    ep, es = rel_err(p, p0), rel_err(sw, sw0)
    counts = [runs[m][step][2] for m in runs]
    print(f"step {step}: pressure {ep:.2e} (floor {fp:.2e}), sw {es:.2e} (floor {fs:.2e}), "
          f"newton {newton} vs {n0} (oracle range {min(counts)}..{max(counts)})")
    assert min(counts) - 1 <= newton <= max(counts) + 1, (step, newton, counts)
    if newton != n0:
        state["diverged"] = True
    if state.get("diverged"):
        assert ep <= NEWTON_TOL_P and es <= NEWTON_TOL_SW, (step, ep, es)
    else:
        assert ep <= 3 * fp + rtol, (step, "pressure", ep, fp)
        assert es <= 3 * fs + rtol, (step, "sat_water", es, fs)
