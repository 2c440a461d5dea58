"""Autotuner of the ensemble form: the thread-block cluster size of each variant's level-scheduled
kernels (block-ILU0 factorisation and sweeps, the pressure BiCGStab).

No counterpart in the reference, which solves one deck on one CPU thread.  The cluster size is
the device path's one launch-shape choice: the smallest size whose slices fit the shared-memory
form is the automatic default, while a larger cluster shortens each level step's work and a
smaller one leaves more SMs to the other variants of a batch.

- `tune` measures, for each candidate size, the device time of one report step of a deck from
  the same state, and persists the curve as JSON keyed by grid dimensions and precision
  (`ressim_b200/tuning/cluster_b200.json` holds one measured on a B200).
- `plan` picks a size for every variant of a batch from those curves (nearest measured grid by
  cell count, time scaled by the cell ratio).  A batch step ends when its last variant does; its
  variants run from `host_threads` host threads over `sms` SMs, so the step takes at least
  sum(T_i) / host_threads (latency bound) and sum(T_i cs_i) / sms (SM bound).  The plan starts
  from every variant's fastest size and moves variants to smaller clusters, best SM-time saving
  per latency added first, while that lowers the larger of the two bounds.
- `criterion="sm_time"` (least T cs per variant) and `"latency"` (fastest per variant) keep the
  per-variant choices; on the 256-variant ensemble the SM-time choice alone was slower than the
  automatic sizes (312k against 526k cell-steps/s), because the batch is latency bound too.
"""
from __future__ import annotations

import json
import os

import numpy as np

CANDIDATES = (1, 2, 4, 8, 16)


def _key(deck, precision: str) -> str:
    return f"{deck.nx}x{deck.ny}x{deck.nz}:{precision}"


def tune_deck(deck, dt: float, precision: str = "fp64", candidates=CANDIDATES, criterion: str = "sm_time",
              warmup_steps: int = 1) -> dict:
    """Times one report step of `deck` (after `warmup_steps` report steps) at every launchable
    candidate cluster size, each from the same state.  Returns {"best": size, "auto": size,
    "ms": {size: device ms}, "criterion": ...}."""
    from .simulator import ReservoirSimulator

    sim = ReservoirSimulator.from_deck(deck)
    sim.set_linear_precision(precision)
    auto = sim.set_cluster_size(0)
    for _ in range(warmup_steps):
        sim.step(dt)
    st = sim.state()
    t0 = sim.time_days
    import ctypes as C

    from . import _lib
    from .simulator import _ptr

    L = _lib.load()
    h = sim._context()
    arrays = [np.ascontiguousarray(st[k]) for k in ("pressure", "sat_water", "sat_gas", "rs")]
    ms = {}
    for want in candidates:
        got = sim.set_cluster_size(want)
        if got in ms:
            continue
        rc = L.rf_set_state(h, *(_ptr(a) for a in arrays), C.c_double(t0))
        if rc != 0:
            raise RuntimeError(f"rf_set_state failed: {_lib.last_error(h)}")
        sim.step(dt)  # the first step at a new size also pays one-time launch set-up; time the second
        rc = L.rf_set_state(h, *(_ptr(a) for a in arrays), C.c_double(t0))
        if rc != 0:
            raise RuntimeError(f"rf_set_state failed: {_lib.last_error(h)}")
        ms[got] = float(sim.step(dt)["device_ms"])
    sim.close()
    cost = {cs: (t * cs if criterion == "sm_time" else t) for cs, t in ms.items()}
    best = min(cost, key=cost.get)
    return {"best": int(best), "auto": int(auto), "ms": {str(k): v for k, v in ms.items()}, "criterion": criterion,
            "cells": int(deck.n_cells)}


def tune(decks, dt: float, precision: str = "fp64", criterion: str = "sm_time", path: str | None = None,
         candidates=CANDIDATES) -> dict:
    """Tunes every distinct grid of `decks` and merges the results into the JSON table at `path`
    (created if missing).  Returns the table."""
    table = load(path) if path and os.path.exists(path) else {}
    for d in decks:
        k = _key(d, precision)
        if k not in table:
            table[k] = tune_deck(d, dt, precision, candidates, criterion)
    if path:
        with open(path, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    return table


def load(path: str) -> dict:
    with open(path) as f:
        return json.load(f)


def choose(table: dict, deck, precision: str = "fp64") -> int:
    """The tuned size for `deck`: its own entry, else the entry of the nearest cell count with the
    same precision; 0 (automatic) when the table has none."""
    k = _key(deck, precision)
    if k in table:
        return int(table[k]["best"])
    same = [v for key, v in table.items() if key.endswith(":" + precision)]
    if not same:
        return 0
    n = deck.n_cells
    return int(min(same, key=lambda v: abs(np.log(v["cells"] / n)))["best"])


def _curve(table: dict, deck, precision: str) -> dict:
    same = {k: v for k, v in table.items() if k.endswith(":" + precision)}
    if not same:
        return {}
    k = _key(deck, precision)
    e = same[k] if k in same else min(same.values(), key=lambda v: abs(np.log(v["cells"] / deck.n_cells)))
    scale = deck.n_cells / e["cells"]
    return {int(cs): t * scale for cs, t in e["ms"].items()}


def plan(table: dict, decks, precision: str = "fp64", host_threads: int = 32, sms: int = 148) -> list[int]:
    """Cluster size per variant for a batch (see the module docstring); 0 where the table has no
    curve for the precision (automatic size)."""
    curves = [_curve(table, d, precision) for d in decks]
    cs = [min(c, key=c.get) if c else 0 for c in curves]

    def bounds(sizes):
        lat = sum(c[s] for c, s in zip(curves, sizes) if c) / host_threads
        smb = sum(c[s] * s for c, s in zip(curves, sizes) if c) / sms
        return lat, smb

    lat, smb = bounds(cs)
    while smb > lat:
        best, best_rate = None, 0.0
        for i, c in enumerate(curves):
            if not c:
                continue
            for s in sorted(c):
                if s >= cs[i]:
                    break
                d_sm = (c[cs[i]] * cs[i] - c[s] * s) / sms
                d_lat = (c[s] - c[cs[i]]) / host_threads
                if d_sm <= 0.0:
                    continue
                rate = d_sm / max(d_lat, 1e-12)
                if rate > best_rate:
                    best, best_rate = (i, s), rate
        if best is None:
            break
        trial = list(cs)
        trial[best[0]] = best[1]
        tl, ts = bounds(trial)
        if max(tl, ts) >= max(lat, smb):
            break
        cs, lat, smb = trial, tl, ts
    return cs


def apply(ensemble, table: dict, precision: str = "fp64", sizes=None) -> list[int]:
    """Sets every variant's cluster size from the table (or from `sizes`, e.g. a `plan`); returns
    the sizes in use."""
    from . import _lib

    L = _lib.load()
    want = sizes if sizes is not None else [choose(table, d, precision) for d in ensemble.decks]
    sizes = []
    for i, d in enumerate(ensemble.decks):
        rc = L.rf_set_cluster_size(ensemble._ctx[i], int(want[i]))
        if rc <= 0:
            raise RuntimeError(f"rf_set_cluster_size failed for variant {i}: {_lib.last_error(ensemble._ctx[i])}")
        sizes.append(int(rc))
    return sizes
