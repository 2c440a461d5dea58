"""Host logic on the CPU: deck setters/validation (mirroring the reference's error behaviour),
the C ABI library's exported symbols, and deck generation."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from ressim_b200 import Deck, _abi, _lib, decks

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ressim_fim.h")


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = set()
    for line in open(HEADER):
        line = line.strip()
        if line.startswith(("int32_t rf_", "int64_t rf_", "RfCtx* rf_")):
            declared.add(line.split("(")[0].split()[-1])
    assert declared == set(_lib.EXPORTED_SYMBOLS)
    for name in declared:
        assert getattr(lib, name) is not None


def test_abi_struct_sizes_are_stable():
    # explicit layout check: the C side is compiled with the same header
    assert C.sizeof(_abi.RfWell) == 8 * 4 + 8 * 8
    assert C.sizeof(_abi.RfTimePointRates) == 16 * 8
    assert C.sizeof(_abi.RfLinearReport) == 8 + 16 + 8


def test_setter_validation_matches_reference_messages():
    d = Deck(3, 2, 1, 0.2)
    with pytest.raises(ValueError, match="S_wc must be in"):
        d.set_rel_perm_props(1.2, 0.1, 2, 2, 1, 1)
    with pytest.raises(ValueError, match="S_wc \\+ S_or must be < 1.0"):
        d.set_rel_perm_props(0.6, 0.5, 2, 2, 1, 1)
    with pytest.raises(ValueError, match="Fluid viscosities must be positive"):
        d.set_fluid_properties(-1.0, 0.5)
    with pytest.raises(ValueError, match="Well indices out of bounds"):
        d.add_well(5, 0, 0, 100.0, 0.1, 0.0, False)
    d.add_well(0, 0, 0, 100.0, 0.1, 0.0, False)
    with pytest.raises(ValueError, match="Multiple well completions in the same cell"):
        d.add_well(0, 0, 0, 120.0, 0.1, 0.0, True)
    with pytest.raises(ValueError, match="Invalid BHP limits"):
        d.set_well_bhp_limits(100.0, 50.0)
    with pytest.raises(ValueError, match="No well found for physical well id"):
        d.set_well_schedule("P1", "rate", 10.0, math.nan, 50.0, True)


def test_surface_rate_zero_means_none():
    d = Deck(1, 1, 1, 0.2)
    d.set_target_well_surface_rates(0.0, 5.0)
    assert d.target_injector_surface_rate_m3_day is None
    assert d.target_producer_surface_rate_m3_day == 5.0


def test_initial_pressure_sets_reference_pressures():
    d = Deck(2, 1, 1, 0.2)
    d.set_initial_pressure(250.0)
    assert np.all(d.pressure == 250.0)
    assert d.water_pvt_reference_pressure_bar == 250.0 and d.rock_reference_pressure_bar == 250.0


def test_schedule_serialises_explicit_control():
    d = Deck(2, 2, 1, 0.2)
    d.add_well_with_id(0, 0, 0, 300.0, 0.1, 0.0, True, "I1")
    d.add_well_with_id(1, 1, 0, 100.0, 0.1, 0.0, False, "P1")
    d.set_well_schedule("P1", "rate", 12.0, math.nan, 40.0, True)
    abi, keep = d.to_abi()
    w = abi.wells[1]
    assert w.has_schedule == 1 and w.schedule_control == 2 and w.schedule_target_rate == 12.0
    assert math.isnan(w.schedule_target_surface_rate) and w.schedule_bhp_limit == 40.0
    assert abi.wells[0].physical_well_id == 0 and w.physical_well_id == 1


def test_lognormal_field_statistics():
    k, z = decks.lognormal_field((6, 40, 40), seed=1, ln_mean=math.log(100.0), sigma=1.0, corr_cells=5.0)
    assert abs(z.mean()) < 1e-9 and abs(z.std() - 1.0) < 1e-9
    assert abs(np.log(k).mean() - math.log(100.0)) < 1e-9


def test_deck_digest_is_seeded():
    a = decks.waterflood_3d(8, 8, 2, seed=4)
    b = decks.waterflood_3d(8, 8, 2, seed=4)
    c = decks.waterflood_3d(8, 8, 2, seed=5)
    assert decks.deck_digest(a) == decks.deck_digest(b) != decks.deck_digest(c)


def test_scal_table_setter_checks_and_abi_fields():
    """setThreePhaseScalTables (frontend.rs:1145-1158) with ThreePhaseScalTables::validate
    (relperm.rs:65-122): at least two rows, finite values within [0, 1], strictly increasing
    saturation, and the Corey props first; new Corey props drop the tables."""
    import numpy as np
    import pytest

    from ressim_b200 import Deck

    swof = [(0.1, 0.0, 1.0), (0.5, 0.2, 0.3), (0.9, 0.8, 0.0)]
    sgof = [{"sg": 0.0, "krg": 0.0, "krog": 1.0, "pcog": 0.0}, {"sg": 0.8, "krg": 0.9, "krog": 0.0, "pcog": 0.0}]
    d = Deck(3, 1, 1, 0.2)
    with pytest.raises(ValueError, match="must be configured before SWOF/SGOF"):
        d.set_three_phase_scal_tables(swof, sgof)
    d.set_three_phase_rel_perm_props(0.1, 0.1, 0.05, 0.05, 0.15, 2.0, 2.0, 1.5, 1.0, 1.0, 1.0)
    with pytest.raises(ValueError, match="SWOF table must contain at least two rows"):
        d.set_three_phase_scal_tables(swof[:1], sgof)
    with pytest.raises(ValueError, match="SWOF saturation must be strictly increasing at row 2"):
        d.set_three_phase_scal_tables([swof[0], swof[1], swof[1]], sgof)
    with pytest.raises(ValueError, match="SGOF row 1 must stay within"):
        d.set_three_phase_scal_tables(swof, [sgof[0], {"sg": 0.8, "krg": 1.2, "krog": 0.0}])
    with pytest.raises(ValueError, match="SWOF row 0 must contain finite values"):
        d.set_three_phase_scal_tables([(0.1, float("nan"), 1.0), swof[1]], sgof)
    d.set_three_phase_scal_tables(swof, sgof)
    raw, keep = d.to_abi()
    assert raw.n_swof_rows == 3 and raw.n_sgof_rows == 2
    assert [raw.swof_rows[i] for i in range(9)] == list(np.ravel(swof))
    assert [raw.sgof_rows[i] for i in range(6)] == [0.0, 0.0, 1.0, 0.8, 0.9, 0.0]
    d.set_three_phase_rel_perm_props(0.1, 0.1, 0.05, 0.05, 0.15, 2.0, 2.0, 1.5, 1.0, 1.0, 1.0)
    assert d.scal_tables is None
    raw, keep = d.to_abi()
    assert raw.n_swof_rows == 0 and raw.n_sgof_rows == 0
