"""Shared parity helpers: relative field error and the oracle's own rounding floor."""
import numpy as np

from oracle.oracle_py import OracleSimulator, lib


def rel_err(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = np.maximum(np.abs(b), 1.0)
    return float(np.max(np.abs(a - b) / scale)) if a.size else 0.0


def oracle_runs(deck, dt, steps):
    """The oracle stepped `steps` report steps twice: with the reference's left-to-right dot
    products (mode 0) and with interleaved partial sums (mode 1).  Returns {mode: [(p, sw,
    newton_iterations) per step]}; the mode-0 vs mode-1 difference is the rounding floor."""
    runs = {}
    try:
        for mode in (0, 1):
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


def check_within_floor(step, p, sw, newton, runs, rtol=1e-6):
    """Device fields within three times the rounding floor plus `rtol`; Newton count within one."""
    p0, sw0, n0 = runs[0][step]
    p1, sw1, _ = runs[1][step]
    fp, fs = rel_err(p1, p0), rel_err(sw1, sw0)
    assert rel_err(p, p0) <= 3 * fp + rtol, (step, "pressure", rel_err(p, p0), fp)
    assert rel_err(sw, sw0) <= 3 * fs + rtol, (step, "sat_water", rel_err(sw, sw0), fs)
    assert abs(newton - n0) <= 1, (step, newton, n0)
