"""Parity at the configurations' own sizes under the matched tight-tolerance profile (GPU tests).

The profile (tests/_matched.py) keeps the reference's controller and tightens only the Newton
acceptance to CNV 1e-9 / MB 1e-11 on both the device and the oracle, so both converge each substep
to the same discrete solution.  Bar, per report step: pressure, water saturation (gas saturation and
Rs in three-phase mode) and well BHP within 1e-6 relative (scale max(|x|, 1)), the same number of
substeps, Newton iterations within one, and every rate-history record (oil, liquid, injection,
average pressure and saturation) within 1e-6 relative.

  configuration 1: the 200-cell 1D waterflood, all 100 report steps
  configuration 2: the 60x60x20 three-phase black-oil deck (72,000 cells), 3 report steps of 10 d
  configuration 4: one ensemble variant from each size quartile, 3 report steps of 10 d, stepped
                   together through the batch API

The oracle runs in spawned processes (its controller options are process-wide).
"""
import pytest

from _matched import MATCHED_CNV, MATCHED_MB, make_deck, oracle_runs_parallel
from _parity import rel_err
from ressim_b200 import Ensemble, ReservoirSimulator, decks

pytestmark = pytest.mark.gpu

RTOL = 1e-6
RATE_KEYS = ("total_production_oil", "total_production_liquid", "total_injection", "avg_reservoir_pressure",
             "avg_water_saturation")


def _check_step(tag, s, gs, gbhp, gnewton, gsub, ref, three):
    cs, cbhp, cnewton, csub, crc = ref
    assert crc == 0, (tag, s, "oracle warning")
    keys = ("pressure", "sat_water", "sat_gas", "rs") if three else ("pressure", "sat_water")
    errs = {k: rel_err(gs[k], cs[k]) for k in keys}
    errs["bhp"] = rel_err(gbhp, cbhp)
    print(f"{tag} step {s}: " + ", ".join(f"{k} {v:.1e}" for k, v in errs.items()) +
          f", newton {gnewton}/{cnewton}, substeps {gsub}/{csub}")
    for k, v in errs.items():
        assert v <= RTOL, (tag, s, k, v)
    assert gsub == csub, (tag, s, gsub, csub)
    assert abs(gnewton - cnewton) <= 1, (tag, s, gnewton, cnewton)


def _check_rates(tag, hg, hc):
    assert len(hg) == len(hc), (tag, len(hg), len(hc))
    worst = 0.0
    for a, b in zip(hg, hc):
        for key in RATE_KEYS:
            e = abs(a[key] - b[key]) / max(abs(b[key]), 1.0)
            worst = max(worst, e)
            assert e <= RTOL, (tag, key, a[key], b[key])
    print(f"{tag}: {len(hg)} rate records, worst {worst:.1e}")


def _device(deck):
    g = ReservoirSimulator.from_deck(deck)
    g.set_controller_options(False, MATCHED_CNV, MATCHED_MB)
    return g


def test_config1_waterflood_1d_all_100_report_steps_matched():
    deck, dt, steps = decks.waterflood_1d()
    refs, hist = oracle_runs_parallel([(("1d",), dt, steps)])[0]
    g = _device(deck)
    for s in range(steps):
        r = g.step(dt)
        assert r["warning"] == 0
        _check_step("config 1", s, g.state(), g.get_well_bhp(), r["newton_iterations"], r["substeps"], refs[s], False)
    _check_rates("config 1", g.get_rate_history(), hist)


def test_config2_blackoil_72k_three_report_steps_matched():
    spec, dt, steps = ("bo", (60, 60, 20)), 10.0, 3
    refs, hist = oracle_runs_parallel([(spec, dt, steps)])[0]
    g = _device(make_deck(spec))
    for s in range(steps):
        r = g.step(dt)
        assert r["warning"] == 0
        _check_step("config 2", s, g.state(), g.get_well_bhp(), r["newton_iterations"], r["substeps"], refs[s], True)
    _check_rates("config 2", g.get_rate_history(), hist)


def quartile_variants(n_variants=256):
    """One variant per size quartile of the ensemble: the variants at the 12.5/37.5/62.5/87.5th
    percentiles of the cell count."""
    sizes = [decks.ensemble_variant(i).n_cells for i in range(n_variants)]
    order = sorted(range(n_variants), key=lambda i: (sizes[i], i))
    return [order[int(q * (n_variants - 1))] for q in (0.125, 0.375, 0.625, 0.875)], sizes


def test_config4_ensemble_one_variant_per_size_quartile_matched():
    picks, sizes = quartile_variants()
    dt, steps = 10.0, 3
    refs = oracle_runs_parallel([(("variant", i), dt, steps) for i in picks])
    ens = Ensemble([decks.ensemble_variant(i) for i in picks])
    ens.set_controller_options(False, MATCHED_CNV, MATCHED_MB)
    for s in range(steps):
        reps = ens.step(dt)
        for j, i in enumerate(picks):
            r = reps[j]
            assert r["warning"] == 0
            _check_step(f"variant {i} ({sizes[i]} cells)", s, ens.state(j), ens.well_bhp(j), r["newton_iterations"],
                        r["substeps"], refs[j][0][s], False)
    for j, i in enumerate(picks):
        _check_rates(f"variant {i}", ens.rate_history(j), refs[j][1])
    ens.close()


def test_config1_waterflood_1d_all_100_report_steps_default_profile():
    """The reference's own tolerances: the 1D deck's pressure stage is the dense coarse inverse, so
    no iteration cap leaves rounding in the Newton end state and the 1e-6 bar holds at all steps."""
    deck, dt, steps = decks.waterflood_1d()
    refs, hist = oracle_runs_parallel([(("1d",), dt, steps, False)])[0]
    g = ReservoirSimulator.from_deck(deck)
    for s in range(steps):
        r = g.step(dt)
        _check_step("config 1 default", s, g.state(), g.get_well_bhp(), r["newton_iterations"], r["substeps"], refs[s],
                    False)
    _check_rates("config 1 default", g.get_rate_history(), hist)
