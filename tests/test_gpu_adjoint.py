"""Discrete adjoint of the device FIM path against central finite differences (GPU tests).

Objective: cumulative surface oil produced over the report steps.  Parameters: the log of each
cell's permeability multiplier (kx, ky, kz together) and each physical well's active control.
The controller runs one substep per report step with Newton converged to tight CNV / MB
tolerances, so that the converged states are smooth functions of the parameters; central
differences use a step of 1e-4 in ln k.  The reference has no adjoint; the finite differences of
the device's own forward runs (which match the oracle to 1e-13 on these decks) are the check.
"""
import copy

import numpy as np
import pytest

from ressim_b200 import ReservoirSimulator, decks

pytestmark = pytest.mark.gpu

CNV, MB = 1e-10, 1e-12


def forward(deck, steps, dt, record=False):
    sim = ReservoirSimulator.from_deck(deck)
    sim.set_controller_options(True, CNV, MB)
    if record:
        sim.adjoint_record(True)
    for _ in range(steps):
        r = sim.step(dt)
        assert r["warning"] == 0, r
    hist = sim.get_rate_history()
    t0, J = 0.0, 0.0
    for h in hist:
        J += (h["time"] - t0) * h["total_production_oil"]
        t0 = h["time"]
    return sim, J


def perturbed(deck, weights):
    d = copy.deepcopy(deck)
    m = np.exp(weights)
    d.perm_x = np.asarray(d.perm_x) * m
    d.perm_y = np.asarray(d.perm_y) * m
    d.perm_z = np.asarray(d.perm_z) * m
    return d


def fd_lnk(deck, direction, steps, dt, h=1e-4):
    _, jp = forward(perturbed(deck, h * direction), steps, dt)
    _, jm = forward(perturbed(deck, -h * direction), steps, dt)
    return (jp - jm) / (2 * h)


def oracle_objective(deck, steps, dt):
    """The oracle's cumulative oil over the same report steps with the same controller options."""
    from oracle.oracle_py import OracleSimulator, lib

    lib().orc_set_controller_options(1, CNV, MB)
    try:
        o = OracleSimulator(deck)
        for _ in range(steps):
            rc, _ = o.step(dt)
            assert rc == 0
        t0, J = 0.0, 0.0
        for h in o.rate_history():
            J += (h["time"] - t0) * h["total_production_oil"]
            t0 = h["time"]
        o.close()
    finally:
        lib().orc_set_controller_options(0, 0.0, 0.0)
    return J


@pytest.mark.parametrize("kind", ["waterflood", "black_oil"])
def test_adjoint_gradient_matches_finite_differences(kind):
    if kind == "waterflood":
        deck = decks.waterflood_3d(6, 5, 2, seed=3, rate_per_perf=20.0)
        steps, dt = 3, 5.0
    else:
        deck = decks.black_oil_3d(5, 5, 2, seed=4, rate_per_perf=10.0)
        steps, dt = 3, 5.0
    n = deck.n_cells
    sim, J = forward(deck, steps, dt, record=True)
    value, g, gc = sim.backward()
    print(f"{kind}: J {J:.10e} adjoint objective {value:.10e}; |g| max {np.max(np.abs(g)):.3e}")
    assert abs(value - J) <= 1e-9 * abs(J)
    # the backward pass leaves the simulator where it was
    _, J_again = forward(deck, steps, dt)
    assert J_again == J
    rng = np.random.default_rng(17)
    cells = rng.choice(n, size=6, replace=False)
    gscale = np.max(np.abs(g))
    worst = 0.0
    for i in cells:
        e = np.zeros(n)
        e[i] = 1.0
        fd = fd_lnk(deck, e, steps, dt)
        fd2 = fd_lnk(deck, e, steps, dt, h=1e-5)
        err = abs(g[i] - fd) / max(abs(fd), 1e-3 * gscale)
        print(f"cell {i}: adjoint {g[i]:.8e} fd {fd:.8e} (h 1e-5: {fd2:.8e}) rel {err:.2e}")
        worst = max(worst, err)
    # the reference gradient: central differences of the oracle's forward runs on two cells
    for i in cells[:2]:
        e = np.zeros(n)
        e[i] = 1.0
        h = 1e-4
        fo = (oracle_objective(perturbed(deck, h * e), steps, dt) -
              oracle_objective(perturbed(deck, -h * e), steps, dt)) / (2 * h)
        ref_err = abs(g[i] - fo) / max(abs(fo), 1e-3 * gscale)
        print(f"cell {i}: oracle fd {fo:.8e}, adjoint rel {ref_err:.2e}")
        assert ref_err < 1e-4, (int(i), g[i], fo)
    v = rng.standard_normal(n)
    fd = fd_lnk(deck, v, steps, dt)
    dd = float(g @ v)
    err_dir = abs(dd - fd) / abs(fd)
    print(f"direction: adjoint {dd:.8e} fd {fd:.8e} rel {err_dir:.2e}")
    assert err_dir < 1e-4
    # controls: the producer's BHP target (one physical well) and the injectors' common rate target
    dp = copy.deepcopy(deck)
    dm = copy.deepcopy(deck)
    hb = 1e-3
    for dd_, s in ((dp, 1.0), (dm, -1.0)):
        for w in dd_.wells:
            if not w.injector:
                w.bhp += s * hb
    fd_bhp = (forward(dp, steps, dt)[1] - forward(dm, steps, dt)[1]) / (2 * hb)
    adj_bhp = gc[-1]  # physical wells: the injectors first, the producer last
    print(f"producer BHP: adjoint {adj_bhp:.8e} fd {fd_bhp:.8e}")
    assert abs(adj_bhp - fd_bhp) <= 1e-4 * max(abs(fd_bhp), 1e-8)
    # the injectors' common rate target moves every injector's control together
    dp, dm = copy.deepcopy(deck), copy.deepcopy(deck)
    q0 = deck.target_injector_rate_m3_day
    hq = 1e-5 * q0
    dp.target_injector_rate_m3_day = q0 + hq
    dm.target_injector_rate_m3_day = q0 - hq
    fd_q = (forward(dp, steps, dt)[1] - forward(dm, steps, dt)[1]) / (2 * hq)
    adj_q = float(np.sum(gc[:-1]))
    print(f"injector rate target: adjoint {adj_q:.8e} fd {fd_q:.8e}")
    assert abs(adj_q - fd_q) <= 1e-4 * max(abs(fd_q), 1e-8)
    assert worst < 1e-4
