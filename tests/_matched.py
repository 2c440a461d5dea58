"""The matched tight-tolerance profile shared by the device and the oracle, and oracle runs under it
in spawned worker processes (the oracle's controller options are process-wide).

Profile: the reference's controller unchanged (PID substep sizes, 0.33 retry factor, iteration-count
growth; timestep.rs:989-1848), with every Newton attempt accepted only at CNV <= 1e-8 and MB <= 1e-10
on each component (no relaxed tiers, no pore-volume relaxation) instead of the reference's
CNV 1e-2 / MB 1e-7 tiers, and every CPR-FGMRES solve of a Newton system refined to a relative
residual of 1e-10 (x += solve(b - A x), the reference's solver inside each pass) instead of the
reference's single solve to 5e-3.  The reference's single solve leaves each Newton update
uncertain at the 5e-3 level, so the preconditioner's rounding moves Newton counts and, through
the iteration-count dt rule, the substep sizes; refined, a Newton update is determined to about
1e-10 and a state that meets CNV 1e-8 to about that level, whatever the summation order or the
precision of the preconditioner.  (At CNV 1e-9 / MB 1e-11 some decks' Newton iterations stall near
the residual's rounding level, so acceptance there, and with it the retries, turns on rounding.)  Both sides then take the same Newton path and converge to the
same discrete solution, and the report-step fields can be compared at 1e-6.  This deviates from
the reference's default tolerances; it is used for parity and for the matched-error comparison
of the mixed form.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MATCHED_CNV, MATCHED_MB = 1e-8, 1e-10
MATCHED_LIN_RTOL, MATCHED_LIN_PASSES = 1e-10, 12


def apply_matched(obj):
    """The matched profile on a device ReservoirSimulator or Ensemble."""
    obj.set_controller_options(False, MATCHED_CNV, MATCHED_MB)
    obj.set_linear_refinement(MATCHED_LIN_RTOL, MATCHED_LIN_PASSES)


def make_deck(spec):
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from ressim_b200 import decks

    kind = spec[0]
    if kind == "1d":
        return decks.waterflood_1d()[0]
    if kind == "bo":
        return decks.black_oil_3d(*spec[1], seed=7)
    if kind == "variant":
        return decks.ensemble_variant(spec[1])
    raise ValueError(spec)


def oracle_run(spec, dt, steps, matched=True, sum_order=0):
    """The oracle on deck `spec` for `steps` report steps of `dt` days.  Returns (per-step list of
    (state dict, well BHPs, Newton iterations, substeps, rc), rate history)."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle.oracle_py import OracleSimulator, lib

    if matched:
        lib().orc_set_controller_options(0, MATCHED_CNV, MATCHED_MB)
        lib().orc_set_linear_refinement(MATCHED_LIN_RTOL, MATCHED_LIN_PASSES)
    lib().orc_set_sum_order(sum_order)
    deck = make_deck(spec)
    o = OracleSimulator(deck)
    out = []
    for _ in range(steps):
        rc, r = o.step(dt)
        out.append((o.state(), o.well_bhp().copy(), r.newton_iterations, r.substeps, rc, r.retries))
    hist = o.rate_history()
    o.close()
    return out, hist


def oracle_runs_parallel(jobs):
    """oracle_run over several (spec, dt, steps[, matched]) jobs in spawned processes, in job order."""
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        return pool.starmap(oracle_run, jobs)


FLOOR_ORDERS = (2, 61)


def oracle_floor_runs(specs, dt, steps, orders=FLOOR_ORDERS):
    """The oracle at the reference's own tolerances on each deck spec, with the reference's
    left-to-right dot products and with each interleaved summation order in `orders` (spawned
    processes).  Returns, per spec, {order: oracle_run output}; the spread over the orders is the
    reference algorithm's rounding floor on that deck."""
    jobs = [(spec, dt, steps, False, m) for spec in specs for m in (0, *orders)]
    res = oracle_runs_parallel(jobs)
    out, k = [], 0
    for _ in specs:
        d = {}
        for m in (0, *orders):
            d[m] = res[k]
            k += 1
        out.append(d)
    return out
