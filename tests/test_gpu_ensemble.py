"""Ensemble batch (rf_batch_*) on the GPU: variants stepped concurrently from several host threads
give exactly the results of the same decks stepped one by one, and a variant matches the oracle."""
import numpy as np
import pytest

from _parity import check_within_floor, oracle_runs
from ressim_b200 import Ensemble, ReservoirSimulator, decks

pytestmark = pytest.mark.gpu

SMALL_VARIANTS = (142, 215, 226, 206)  # 3,300 to 4,050 cells


def test_batch_equals_sequential_runs():
    ds = [decks.ensemble_variant(i) for i in SMALL_VARIANTS]
    ens = Ensemble(ds, host_threads=4)
    singles = [ReservoirSimulator.from_deck(d) for d in ds]
    for _ in range(2):
        reps = ens.step(10.0)
        for i, s in enumerate(singles):
            r = s.step(10.0)
            assert reps[i]["newton_iterations"] == r["newton_iterations"]
    for i, s in enumerate(singles):
        a, b = ens.state(i), s.state()
        assert np.array_equal(a["pressure"], b["pressure"])
        assert np.array_equal(a["sat_water"], b["sat_water"])
    assert ens.kernel_launches() > 0
    ens.close()


@pytest.mark.parametrize("mode,threads", [("groups", 1), ("groups", 2), ("threads", 4)])
def test_batched_launches_equal_sequential_runs(mode, threads):
    """Several variants per group: their factorisations, pressure solves and block-ILU0 sweeps run
    as batched launches (a thread block per variant, the launch sized for the largest); the states
    equal the variants stepped alone, bit for bit, as do the variants of the thread mode."""
    ids = (142, 215, 226, 206, 7)  # 3,300 to 6,578 cells
    ds = [decks.ensemble_variant(i) for i in ids]
    ens = Ensemble(ds, host_threads=threads)
    ens.set_mode(mode)
    ens.batch_profile(enable=True, reset=True)
    singles = [ReservoirSimulator.from_deck(d) for d in ds]
    for _ in range(2):
        reps = ens.step(10.0)
        for i, s in enumerate(singles):
            r = s.step(10.0)
            assert reps[i]["newton_iterations"] == r["newton_iterations"], (mode, i)
    for i, s in enumerate(singles):
        a, b = ens.state(i), s.state()
        assert np.array_equal(a["pressure"], b["pressure"]), (mode, i)
        assert np.array_equal(a["sat_water"], b["sat_water"]), (mode, i)
    prof = ens.batch_profile(enable=False, reset=True)
    print(mode, threads, prof)
    if mode == "groups":
        assert prof["pressure_items"] > prof["pressure_launches"] > 0  # launches carried several solves
    else:
        assert prof["pressure_launches"] == 0
    ens.close()


def test_batch_variant_matches_oracle():
    """A variant stepped inside a batch against the oracle, within the oracle's rounding floor."""
    d = decks.ensemble_variant(SMALL_VARIANTS[0])
    runs = oracle_runs(d, 10.0, 2)
    ens = Ensemble([d, decks.ensemble_variant(SMALL_VARIANTS[1])], host_threads=2)
    state = {}
    for s in range(2):
        reps = ens.step(10.0)
        g = ens.state(0)
        check_within_floor(s, g["pressure"], g["sat_water"], reps[0]["newton_iterations"], runs, state=state)
    ens.close()


def test_batch_with_larger_variant_created_first():
    """Contexts created later with smaller shared-memory needs must not break the launches of a
    larger context created before them (kernel launch limits are process-wide)."""
    ds = [decks.ensemble_variant(i) for i in (206, 142)]  # 4,050 then 3,300 cells
    ens = Ensemble(ds, host_threads=2)
    reps = ens.step(10.0)
    assert all(r["newton_iterations"] > 0 for r in reps)
    ens.close()
