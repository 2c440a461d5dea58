"""The oracle pinned against the reference's own known-answer unit tests (restated, CPU only).

Each test cites the reference test it restates (paths inside the reference project).
"""
import math

import numpy as np
import pytest

from oracle.oracle_py import OracleSimulator, lib, ptr
from ressim_b200 import Deck, decks

TOL = 1e-12


def cnv_mb(residual, pv, fvf, final=False):
    r = np.ascontiguousarray(residual, dtype=float)
    p = np.ascontiguousarray(pv, dtype=float)
    f = np.ascontiguousarray(fvf, dtype=float).ravel()
    out = np.zeros(8)
    lib().orc_cnv_mb_from_parts(len(p), ptr(r), ptr(p), ptr(f), int(final), ptr(out))
    flags = int(out[7])
    return {"cnv": out[0:3], "mb": out[3:6], "viol": out[6], "pv_relax": bool(flags & 1),
            "strict": bool(flags & 2), "accept": bool(flags & 4)}


# fim/newton/tests.rs:294-329 cnv_mb_from_parts_matches_hand_computed_values
def test_cnv_mb_hand_values():
    d = cnv_mb([2.0, -0.6, 0.0, -1.0, 0.9, 0.0], [100.0, 300.0], [[1.0, 1.2, 0.01], [1.0, 1.4, 0.03]])
    assert abs(d["cnv"][0] - 0.02) < TOL
    assert abs(d["cnv"][1] - 1.3 * 0.006) < TOL
    assert d["cnv"][2] == 0.0
    assert abs(d["mb"][0] - 1.0 / 400.0) < TOL
    assert abs(d["mb"][1] - 1.3 * 0.3 / 400.0) < TOL
    assert abs(d["viol"] - 0.25) < TOL
    assert not d["pv_relax"] and not d["strict"] and not d["accept"]


# fim/newton/tests.rs:331-365 cnv_pv_rule_relaxes_when_violating_pv_below_three_percent
def test_cnv_pv_rule():
    d = cnv_mb([0.5, 0, 0, 0, 0, 0], [10.0, 990.0], [[1, 1, 1], [1, 1, 1]])
    assert abs(d["cnv"][0] - 0.05) < TOL
    assert abs(d["viol"] - 0.01) < TOL
    assert d["pv_relax"] and not d["strict"] and not d["accept"]
    d = cnv_mb([0.5, 0, 0, -0.5, 0, 0], [10.0, 990.0], [[1, 1, 1], [1, 1, 1]])
    assert d["mb"][0] == 0.0
    assert not d["strict"] and d["accept"]


# fim/newton/tests.rs:367-386 cnv_mb_relax_final_iteration_applies_relaxed_tiers_unconditionally
def test_cnv_final_iteration_tiers():
    r, pv, f = [25.0, 0, 0, -25.0, 0, 0], [500.0, 500.0], [[1, 1, 1], [1, 1, 1]]
    d = cnv_mb(r, pv, f, final=False)
    assert not d["pv_relax"] and not d["accept"]
    assert cnv_mb(r, pv, f, final=True)["accept"]


def chop(cells, bhp, update, relax):
    cells = np.ascontiguousarray(cells, dtype=float).ravel()
    b = np.ascontiguousarray(bhp, dtype=float)
    u = np.ascontiguousarray(update, dtype=float)
    out = np.zeros_like(u)
    lib().orc_opm_chop(len(cells) // 4, ptr(cells), len(b), ptr(b) if b.size else None, ptr(u), relax, ptr(out))
    return out


SAT = [[200.0, 0.3, 0.1, 0], [200.0, 0.3, 0.1, 0]]
UNDER = [[200.0, 0.3, 50.0, 1], [200.0, 0.3, 50.0, 1]]


# fim/newton/tests.rs:158-180 (two_cell_state_for_chop: p 200, sw 0.3, hc 0.1 | Rs 50)
def test_chop_implied_so():
    u = np.zeros(6)
    u[1], u[2], u[4], u[5] = 0.15, 0.15, 0.01, -0.02
    c = chop(SAT, [], u, 1.0)
    alpha = 0.2 / 0.3
    assert abs(c[1] - 0.15 * alpha) < TOL and abs(c[2] - 0.15 * alpha) < TOL
    assert c[4] == 0.01 and c[5] == -0.02


# fim/newton/tests.rs:182-200
def test_chop_pressure_relative():
    u = np.zeros(6)
    u[0], u[1], u[3] = -100.0, 0.5, 30.0
    c = chop(SAT, [], u, 1.0)
    assert abs(c[0] + 60.0) < TOL and abs(c[1] - 0.2) < TOL and c[3] == 30.0


# fim/newton/tests.rs:202-225
def test_chop_rs_guard():
    u = np.zeros(6)
    u[2], u[1], u[5] = -80.0, 0.25, -10.0
    c = chop(UNDER, [], u, 1.0)
    assert abs(c[2] + 50.0) < TOL and abs(c[1] - 0.2) < TOL and c[5] == -10.0


# fim/newton/tests.rs:227-239
def test_chop_relaxation_first():
    u = np.zeros(6)
    u[1] = 0.3
    assert abs(chop(SAT, [], u, 0.5)[1] - 0.15) < TOL


# fim/newton/tests.rs:241-290 (BHP 500 then 1.5; the cell block is irrelevant to the BHP entry)
def test_chop_bhp():
    cell = [[300.0, 0.3, 0.0, 0]]
    u = np.zeros(4)
    u[3] = 600.0
    assert abs(chop(cell, [500.0], u, 1.0)[3] - 500.0) < TOL
    u[3] = 200.0
    assert chop(cell, [500.0], u, 1.0)[3] == 200.0
    u[3] = -3.0
    assert abs(1.5 + chop(cell, [1.5], u, 1.0)[3] - 1.0) < TOL


# fim/timestep.rs:2081-2099 opm_relative_change_matches_hand_computed_sum_of_squares
def test_relative_change():
    a = np.array([[200.0, 0.3, 0.1, 0]])
    b = np.array([[220.0, 0.35, 0.12, 0]])
    delta = 20.0 ** 2 + 0.05 ** 2 + 0.02 ** 2 + 0.07 ** 2
    denom = 220.0 ** 2 + 0.35 ** 2 + 0.12 ** 2 + 0.53 ** 2
    got = lib().orc_relative_change(1, ptr(np.ascontiguousarray(a.ravel())), ptr(np.ascontiguousarray(b.ravel())))
    assert abs(got - delta / denom) < 1e-9
    assert lib().orc_relative_change(1, ptr(np.ascontiguousarray(a.ravel())),
                                     ptr(np.ascontiguousarray(a.ravel()))) == 0.0


def pid(dt, e):
    return lib().orc_pid_dt(dt, ptr(np.array(e, dtype=float)))


# fim/timestep.rs:2101-2125
def test_pid():
    assert abs(pid(1.0, [0.1, 0.1, 0.2]) - 0.5) < TOL
    assert pid(1.0, [0.0, 0.05, 0.05]) == np.finfo(float).max
    exp = (0.05 / 0.05) ** 0.075 * (0.1 / 0.05) ** 0.175 * (0.05 * 0.05 / (0.05 * 0.05)) ** 0.01
    got = pid(1.0, [0.05, 0.05, 0.05])
    assert abs(got - exp) < 1e-9 and got > 1.0


# fim/timestep.rs:2127-2135
def test_iteration_count_dt():
    f = lib().orc_iteration_count_dt
    assert abs(f(1.0, 2) - 3.4) < TOL and abs(f(1.0, 8) - 1.0) < TOL and abs(f(1.0, 16) - 0.5) < TOL


# fim/timestep.rs:2137-2161
def test_growth_decision():
    import ctypes as C
    e = np.array([1e-6, 1e-6, 1e-6])
    lim = C.c_int32()
    assert abs(lib().orc_growth_decision(1.0, 0, ptr(e), 0, C.byref(lim)) - 3.0) < 1e-9 and lim.value == 0
    assert abs(lib().orc_growth_decision(1.0, 16, ptr(e), 0, C.byref(lim)) - 0.5) < 1e-9 and lim.value == 2
    assert abs(lib().orc_growth_decision(1.0, 0, ptr(e), 1, C.byref(lim)) - 2.0) < 1e-9 and lim.value == 3


def ad(which, x, y=0.0):
    out = np.zeros(3)
    lib().orc_ad_probe(which, x, y, ptr(out))
    return out


def close(a, b):
    return abs(a - b) <= 1e-10 * (1 + max(abs(a), abs(b)))


# fim/ad.rs:432-500
def test_ad_rules():
    v = ad(0, 2.0, 3.0)
    assert close(v[0], 1.2) and close(v[1], 9 / 25) and close(v[2], 4 / 25)
    v = ad(1, 4.0)
    assert close(v[0], math.exp(2)) and close(v[1], math.exp(2) * 0.25)
    v = ad(2, 4.0)
    assert close(v[0], 8.0) and close(v[1], 3.0)
    v = ad(3, 2.0)
    assert close(v[0], 0.5) and close(v[1], -0.25)
    v = ad(4, 3.0)
    assert close(v[0], 10 - 4.5) and close(v[1], -1.5)
    v = ad(5, 1.0)
    assert v[0] == 2.0 and v[1] == 0.0
    v = ad(6, 1.0)
    assert v[0] == 1.0 and v[1] == 1.0


# relperm.rs:762-810 corey_table_derivatives_match_ad_derivative_of_the_table
@pytest.mark.parametrize("scal", [(0.1, 0.1, 2.0, 2.0, 1.0, 1.0), (0.15, 0.25, 3.0, 1.5, 0.4, 0.85)])
@pytest.mark.parametrize("points", [2, 3, 5, 21, 101 - 37])
def test_corey_table_slopes(scal, points):
    swc, sor, nw, no, krwm, krom = scal
    d = Deck(1, 1, 1, 0.2)
    d.set_rel_perm_props(*scal)
    d.set_fim_corey_table_points(points)
    abi, keep = d.to_abi()
    krw = lambda s: krwm * min(max((s - swc) / (1 - swc - sor), 0), 1) ** nw
    kro = lambda s: krom * min(max((1 - s - sor) / (1 - swc - sor), 0), 1) ** no
    lo, hi = swc, 1 - sor
    step = (hi - lo) / (points - 1)
    samples = [0.0, lo - 0.05, lo, hi, hi + 0.05, 1.0]
    for k in range(points):
        samples += [lo + k * step + f * step for f in (0.0, 0.25, 0.5)]
    import ctypes as C
    for s in samples:
        out = np.zeros(4)
        lib().orc_corey_table(C.byref(abi), s, ptr(out))
        if s <= lo or s >= hi:
            exp_d = (0.0, 0.0)
        else:
            seg = min(int(math.floor((s - lo) / step)), points - 2)
            x0, x1 = min(lo + seg * step, hi), min(lo + (seg + 1) * step, hi)
            w = max(x1 - x0, 1e-12)
            exp_d = ((krw(x1) - krw(x0)) / w, (kro(x1) - kro(x0)) / w)
        assert abs(out[2] - exp_d[0]) <= 1e-9 * max(abs(exp_d[0]), 1.0), (s, points)
        assert abs(out[3] - exp_d[1]) <= 1e-9 * max(abs(exp_d[1]), 1.0), (s, points)


# pvt.rs:1034-1046 pvtw_inverse_fvf_uses_reference_pressure_and_quadratic_compressibility
def test_pvtw():
    f = lib().orc_water_inverse_fvf
    assert abs(f(200.0, 200.0, 5e-5, 1.2) - 1 / 1.2) < 1e-14
    x = 5e-5 * 50.0
    assert abs(f(250.0, 200.0, 5e-5, 1.2) - (1 + x * (1 + x / 2)) / 1.2) < 1e-14


# fim/tests/wells.rs:13-50 peaceman_connection_law_matches_analytical_wi
def test_peaceman_wi():
    import ctypes as C
    d = Deck(1, 1, 1, 0.25)
    d.set_cell_dimensions_per_layer(400.0, 300.0, [20.0])
    d.set_permeability_per_layer([150.0], [60.0], [5.0])
    d.add_well(0, 0, 0, 100.0, 0.1, 1.5, False)
    abi, keep = d.to_abi()
    kx, ky = 150.0, 60.0
    r_eq = 0.28 * math.sqrt(math.sqrt(kx / ky) * 400.0 ** 2 + math.sqrt(ky / kx) * 300.0 ** 2) / (
        (kx / ky) ** 0.25 + (ky / kx) ** 0.25)
    wi = 8.5269888e-3 * 2 * math.pi * math.sqrt(kx * ky) * 20.0 / (math.log(r_eq / 0.1) + 1.5)
    assert abs(lib().orc_well_index(C.byref(abi), 0) - wi) <= 1e-12 * wi


def _fd_jacobian_check(deck, dt, perturb_seed=0):
    """AD Jacobian vs central differences h = 1e-6 (1 + |x|) (fim/numjac.rs:13-40)."""
    sim = OracleSimulator(deck)
    nw, npf = sim.topology()
    n = deck.n_cells
    rng = np.random.default_rng(perturb_seed)
    prev = np.stack([deck.pressure, deck.sat_water, np.zeros(n)], axis=1)
    cur = prev.copy()
    cur[:, 0] += rng.uniform(-5, 5, n)
    cur[:, 1] = np.clip(cur[:, 1] + rng.uniform(0.0, 0.3, n), 0.0, 0.9)
    # away from the max(hc, 0) kink at hc = 0, where a central difference averages two branches
    cur[:, 2] = 0.02
    bhp = np.array([w.bhp for w in deck.wells][:nw], dtype=float)
    q = rng.uniform(-20, 20, npf)
    for k, w in enumerate(deck.wells):
        q[k] = -abs(q[k]) if w.injector else abs(q[k])
    res, ptr_, col, val = sim.assemble_state(dt, prev, cur, bhp, q)
    J = np.zeros((len(res), len(res)))
    for r in range(len(res)):
        for k in range(ptr_[r], ptr_[r + 1]):
            J[r, col[k]] = val[k]
    x = np.concatenate([cur.ravel(), bhp, q])
    worst = 0.0
    for j in range(len(x)):
        h = 1e-6 * (1 + abs(x[j]))
        xp, xm = x.copy(), x.copy()
        xp[j] += h
        xm[j] -= h

        def resid(v):
            return sim.assemble_state(dt, prev, v[: 3 * n].reshape(n, 3), v[3 * n:3 * n + nw], v[3 * n + nw:])[0]
        fd = (resid(xp) - resid(xm)) / (2 * h)
        scale = np.maximum(np.abs(J[:, j]), np.max(np.abs(J[:, j])) * 1e-6 + 1e-8)
        worst = max(worst, float(np.max(np.abs(fd - J[:, j]) / scale)))
    return worst


def test_jacobian_matches_finite_differences_with_wells():
    d = Deck(4, 3, 2, 0.2)
    d.set_rel_perm_props(0.15, 0.15, 2.0, 2.5, 0.8, 1.0)
    d.set_fim_corey_table_points(0)  # smooth Corey so the central difference is well defined
    d.set_fluid_compressibilities(2e-5, 5e-6)
    d.set_rock_properties(3e-5, 0.0, 1.1, 1.02)
    d.set_capillary_params(0.0, 2.0)
    d.set_initial_pressure(250.0)
    d.set_initial_saturation(0.3)
    d.set_well_control_modes("rate", "rate")
    d.set_target_well_rates(30.0, 25.0)
    d.add_well(0, 0, 0, 400.0, 0.1, 0.0, True)
    d.add_well(3, 2, 1, 150.0, 0.1, 0.5, False)
    assert _fd_jacobian_check(d, 0.5) < 1e-4


def test_jacobian_matches_finite_differences_gravity_capillarity():
    d = Deck(3, 2, 3, 0.25)
    d.set_cell_dimensions(12.0, 9.0, 3.0)
    d.set_rel_perm_props(0.1, 0.2, 2.0, 2.0, 1.0, 1.0)
    d.set_fim_corey_table_points(0)
    d.set_capillary_params(2.0, 2.0)
    d.set_gravity_enabled(True)
    d.set_initial_pressure(200.0)
    d.set_initial_saturation(0.4)
    assert _fd_jacobian_check(d, 1.0, perturb_seed=3) < 1e-4


def test_waterflood_1d_material_balance_and_front():
    """Physics sanity of the oracle trajectory: water material balance closes to round-off
    and a saturation front has advanced from the injector."""
    deck, dt, _ = decks.waterflood_1d()
    sim = OracleSimulator(deck)
    for _ in range(10):
        rc, _ = sim.step(dt)
        assert rc == 0
    st = sim.state()
    sw = st["sat_water"]
    assert sw[0] > 0.5 and abs(sw[-1] - 0.2) < 1e-3
    front = int(np.argmax(sw < 0.25))
    assert 10 < front < 100
    assert sw[:front // 2].mean() > sw[front // 2:front].mean() > sw[front:].mean()
    last = sim.rate_history()[-1]
    assert last["material_balance_error_m3"] < 1e-6 * 20000.0


# tests/physics/wellbore_datum.rs: a 1x1x4 water column in hydrostatic equilibrium with a fully
# perforated producer; the completion heads carry the datum BHP down the wellbore.
GRAVITY_M_S2 = 9.80665


def _hydrostatic_water_column(gravity=True):
    layers, dz = 4, 10.0
    d = Deck(1, 1, layers, 0.2)
    d.set_cell_dimensions_per_layer(20.0, 20.0, [dz] * layers)
    d.set_fluid_densities(800.0, 1000.0)
    d.set_initial_pressure(300.0)
    d.set_initial_saturation(1.0)
    d.set_capillary_params(0.0, 2.0)
    d.set_gravity_enabled(gravity)
    rho_w = lib().orc_water_inverse_fvf(300.0, 300.0, d.c_w, d.b_w) * 1000.0
    depth = [d.depth_reference_m + dz * k + 0.5 * dz for k in range(layers)]
    d.pressure = np.array([300.0 + rho_w * GRAVITY_M_S2 * (depth[k] - depth[0]) * 1e-5 for k in range(layers)])
    for k in range(layers):
        d.add_well_with_id(0, 0, k, 290.0, 0.1, 0.0, False, "prod")
    return d, depth, rho_w


def test_wellbore_datum_defaults_to_shallowest_completion():
    d, depth, rho_w = _hydrostatic_water_column()
    h = OracleSimulator(d).head_offsets()
    assert h[0] == 0.0
    for k in range(1, 4):
        expected = rho_w * GRAVITY_M_S2 * (depth[k] - depth[0]) * 1e-5
        assert abs(h[k] - expected) < 1e-4, (k, h[k], expected)


def test_wellbore_datum_honours_explicit_datum_and_density():
    d, depth, _ = _hydrostatic_water_column()
    for w in d.wells:
        w.datum_depth_m = depth[-1]
        w.wellbore_density_kg_m3 = 500.0
    h = OracleSimulator(d).head_offsets()
    assert h[-1] == 0.0
    for k in range(4):
        assert abs(h[k] - 500.0 * GRAVITY_M_S2 * (depth[k] - depth[-1]) * 1e-5) < 1e-9
    assert h[0] < 0.0


def test_wellbore_datum_head_is_zero_without_gravity():
    d, _, _ = _hydrostatic_water_column(gravity=False)
    assert np.all(OracleSimulator(d).head_offsets() == 0.0)


def test_jacobian_matches_finite_differences_gravity_with_wells():
    """Gravity and wells together: the completion heads (refreshed on the assembled state, held
    fixed through the Newton step as in the reference) enter the connection rows."""
    d = Deck(3, 3, 4, 0.2)
    d.set_cell_dimensions(15.0, 15.0, 4.0)
    d.set_rel_perm_props(0.15, 0.15, 2.0, 2.0, 1.0, 1.0)
    d.set_fim_corey_table_points(0)
    d.set_capillary_params(0.0, 2.0)
    d.set_gravity_enabled(True)
    d.set_initial_pressure(250.0)
    d.set_initial_saturation(0.35)
    d.set_well_control_modes("rate", "pressure")
    d.set_target_well_rates(20.0, 0.0)
    for k in range(4):
        d.add_well_with_id(0, 0, k, 320.0, 0.1, 0.0, True, "INJ")
        d.add_well_with_id(2, 2, k, 200.0, 0.1, 0.0, False, "PROD")
    sim = OracleSimulator(d)
    h = sim.head_offsets()
    assert h[0] == 0.0 and h[1] == 0.0 and np.all(h[2:] > 0.0)  # datum at the top completions
    assert _fd_jacobian_check(d, 0.5, perturb_seed=5) < 1e-4
