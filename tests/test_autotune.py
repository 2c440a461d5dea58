"""Host logic of the cluster-size autotuner (no GPU): table keys and the nearest-size choice."""
from ressim_b200 import autotune, decks


def test_choose_uses_own_entry_then_nearest_cell_count():
    small, large = decks.ensemble_variant(142), decks.ensemble_variant(0)
    table = {
        autotune._key(small, "fp64"): {"best": 2, "cells": small.n_cells},
        autotune._key(large, "fp64"): {"best": 8, "cells": large.n_cells},
        autotune._key(large, "mixed"): {"best": 4, "cells": large.n_cells},
    }
    assert autotune.choose(table, small) == 2
    assert autotune.choose(table, large) == 8
    assert autotune.choose(table, large, "mixed") == 4
    other = decks.ensemble_variant(215)
    nearest = min((small, large), key=lambda d: abs(d.n_cells - other.n_cells) / min(d.n_cells, other.n_cells))
    assert autotune.choose(table, other) in (2, 8)
    assert autotune.choose(table, other) == (2 if nearest is small else 8)
    assert autotune.choose({}, other) == 0


def test_plan_balances_latency_and_sm_bounds():
    """With many variants over few host threads the plan keeps the fastest sizes; with few SMs it
    moves variants to smaller clusters and lowers the larger of the two bounds."""
    ds = [decks.ensemble_variant(i) for i in (142, 0, 215, 206)]
    table = {autotune._key(d, "fp64"): {"best": 1, "cells": d.n_cells,
                                        "ms": {"1": 400.0, "2": 250.0, "4": 160.0, "8": 120.0, "16": 110.0}}
             for d in ds}
    fast = autotune.plan(table, ds, host_threads=1, sms=1000)
    assert all(cs == 16 for cs in fast)

    def bound(sizes, host_threads, sms):
        curves = [autotune._curve(table, d, "fp64") for d in ds]
        lat = sum(c[s] for c, s in zip(curves, sizes)) / host_threads
        smb = sum(c[s] * s for c, s in zip(curves, sizes)) / sms
        return max(lat, smb)
    lean = autotune.plan(table, ds, host_threads=32, sms=8)
    assert max(lean) < 16
    assert bound(lean, 32, 8) < bound(fast, 32, 8)
