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
