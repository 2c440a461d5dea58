"""Seeded synthetic decks for the FIM benchmark configurations.

No reservoir dataset is involved: every deck is generated from a seed, with the grid sizes,
statistics and controls of the benchmark configurations.  `deck_digest` hashes every array so a
run can state exactly which deck it used.
"""
from __future__ import annotations

import hashlib
import math

import numpy as np

from .deck import Deck


def lognormal_field(shape_zyx, seed: int, ln_mean: float, sigma: float, corr_cells: float):
    """ln k = ln_mean + sigma * z, where z is seeded white noise smoothed with a Gaussian of
    `corr_cells` cells and re-standardised to zero mean and unit variance.  Returns (k, z) in
    natural cell order (x fastest)."""
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape_zyx)
    sm = gaussian_filter(noise, sigma=corr_cells, mode="wrap") if corr_cells > 0 else noise
    z = (sm - sm.mean()) / max(sm.std(), 1e-12)
    k = np.exp(ln_mean + sigma * z)
    return k.ravel(), z.ravel()


def waterflood_1d(n_cells: int = 200, steps: int = 100, total_days: float = 1000.0) -> tuple[Deck, float, int]:
    """1D two-phase waterflood: n x 1 x 1, dx=5 m, dy=dz=10 m, k=100 mD, phi=0.2, Corey n=2,
    Swc=Sor=0.2, mu_w=0.5 cP, mu_o=2 cP, c_w=c_o=1e-5/bar, no gravity or capillarity.  Rate
    injector in cell 0 delivering 0.5 pore volumes over the run, BHP producer (250 bar) in the
    last cell, initial pressure 300 bar.  Returns (deck, dt_days, steps)."""
    d = Deck(n_cells, 1, 1, 0.2)
    d.set_cell_dimensions(5.0, 10.0, 10.0)
    d.set_permeability_per_layer([100.0], [100.0], [100.0])
    d.set_rel_perm_props(0.2, 0.2, 2.0, 2.0, 1.0, 1.0)
    d.set_fluid_properties(2.0, 0.5)
    d.set_fluid_compressibilities(1e-5, 1e-5)
    d.set_rock_properties(0.0, 0.0, 1.0, 1.0)
    d.set_capillary_params(0.0, 2.0)
    d.set_gravity_enabled(False)
    d.set_initial_pressure(300.0)
    d.set_initial_saturation(0.2)
    pv_total = float(np.sum(d.porosity) * d.dx * d.dy * d.dz[0])
    rate = 0.5 * pv_total / total_days
    d.set_well_control_modes("rate", "pressure")
    d.set_target_well_rates(rate, 0.0)
    d.set_well_bhp_limits(50.0, 600.0)
    d.add_well(0, 0, 0, 500.0, 0.1, 0.0, True)
    d.add_well(n_cells - 1, 0, 0, 250.0, 0.1, 0.0, False)
    return d, total_days / steps, steps


def waterflood_3d(nx: int, ny: int, nz: int, seed: int = 7, dx: float = 20.0, dz: float = 2.0,
                  sigma: float = 1.0, corr_cells: float = 5.0, kv_kh: float = 0.1,
                  rate_per_perf: float = 50.0, gravity: bool = False) -> Deck:
    """Two-phase waterflood on an nx x ny x nz grid with the 1D deck's fluid and SCAL: ln kh ~
    N(ln 100 mD, sigma) smoothed to `corr_cells` correlation length, kv = kv_kh * kh,
    phi = clip(0.1 + 0.02 z, 0.05, 0.3), inverted five-spot (four corner rate injectors, one
    centre BHP producer at 250 bar), every layer perforated, initial pressure 300 bar.  With
    `gravity`, the BHPs are quoted at the shallowest completion and carried down each wellbore."""
    d = Deck(nx, ny, nz, 0.2)
    d.set_cell_dimensions(dx, dx, dz)
    kh, z = lognormal_field((nz, ny, nx), seed, math.log(100.0), sigma, corr_cells)
    d.set_permeability_field(kh, kh, kv_kh * kh)
    d.set_porosity_field(np.clip(0.1 + 0.02 * z, 0.05, 0.3))
    d.set_rel_perm_props(0.2, 0.2, 2.0, 2.0, 1.0, 1.0)
    d.set_fluid_properties(2.0, 0.5)
    d.set_fluid_compressibilities(1e-5, 1e-5)
    d.set_rock_properties(0.0, 0.0, 1.0, 1.0)
    d.set_capillary_params(0.0, 2.0)
    d.set_gravity_enabled(gravity)
    d.set_initial_pressure(300.0)
    d.set_initial_saturation(0.2)
    d.set_well_control_modes("rate", "pressure")
    d.set_target_well_rates(rate_per_perf * nz, 0.0)
    d.set_well_bhp_limits(50.0, 600.0)
    corners = [(0, 0), (nx - 1, 0), (0, ny - 1), (nx - 1, ny - 1)]
    for n, (i, j) in enumerate(corners):
        for k in range(nz):
            d.add_well_with_id(i, j, k, 500.0, 0.1, 0.0, True, f"INJ{n + 1}")
    for k in range(nz):
        d.add_well_with_id(nx // 2, ny // 2, k, 250.0, 0.1, 0.0, False, "PROD")
    return d


def ensemble_variant(index: int, seed: int = 1000, steps: int = 40, dt_days: float = 10.0) -> Deck:
    """One variant of the sensitivity ensemble: nx, ny ~ U{20..64}, nz ~ U{5..16}, ln kh with
    sigma ~ U[0.5, 1.5] (5-cell correlation), mobility ratio mu_o/mu_w ~ U[0.5, 10] (mu_w 0.5 cP),
    Corey n_w, n_o ~ U[1.5, 4], kv/kh ~ U[0.01, 1]; quarter five-spot: a rate injector in the
    (0, 0) column delivering 0.5 pore volumes over `steps` x `dt_days`, a 250-bar BHP producer in
    the opposite column, every layer perforated.  Variant `index` draws from seed + index."""
    rng = np.random.default_rng(seed + index)
    nx, ny = (int(v) for v in rng.integers(20, 65, size=2))
    nz = int(rng.integers(5, 17))
    sigma = float(rng.uniform(0.5, 1.5))
    mob = float(rng.uniform(0.5, 10.0))
    n_w, n_o = (float(v) for v in rng.uniform(1.5, 4.0, size=2))
    kv_kh = float(rng.uniform(0.01, 1.0))
    d = Deck(nx, ny, nz, 0.2)
    d.set_cell_dimensions(20.0, 20.0, 2.0)
    kh, z = lognormal_field((nz, ny, nx), seed + index, math.log(100.0), sigma, 5.0)
    d.set_permeability_field(kh, kh, kv_kh * kh)
    d.set_porosity_field(np.clip(0.1 + 0.02 * z, 0.05, 0.3))
    d.set_rel_perm_props(0.2, 0.2, n_w, n_o, 1.0, 1.0)
    d.set_fluid_properties(0.5 * mob, 0.5)
    d.set_fluid_compressibilities(1e-5, 1e-5)
    d.set_rock_properties(0.0, 0.0, 1.0, 1.0)
    d.set_capillary_params(0.0, 2.0)
    d.set_gravity_enabled(False)
    d.set_initial_pressure(300.0)
    d.set_initial_saturation(0.2)
    pv_total = float(np.sum(d.porosity) * 20.0 * 20.0 * 2.0)
    d.set_well_control_modes("rate", "pressure")
    d.set_target_well_rates(0.5 * pv_total / (steps * dt_days), 0.0)
    d.set_well_bhp_limits(50.0, 600.0)
    for k in range(nz):
        d.add_well_with_id(0, 0, k, 500.0, 0.1, 0.0, True, "INJ")
    for k in range(nz):
        d.add_well_with_id(nx - 1, ny - 1, k, 250.0, 0.1, 0.0, False, "PROD")
    return d


def black_oil_3d(nx: int, ny: int, nz: int, seed: int = 7, dx: float = 20.0, dz: float = 2.0, sigma: float = 1.0,
                 corr_cells: float = 5.0, kv_kh: float = 0.1, rate_per_perf: float = 20.0,
                 producer_bhp: float = 150.0, pb_bar: float = 200.0, p_init: float = 250.0,
                 gravity: bool = True, pc_og: bool = False, injected_fluid: str = "water") -> Deck:
    """Three-phase black-oil inverted five-spot: the 3D deck's seeded field statistics (ln kh ~
    N(ln 100 mD, sigma), kv = kv_kh kh, phi = clip(0.1 + 0.02 z, 0.05, 0.3)); a correlation PVT
    table (API 35, gas gravity 0.75, 80 C, bubble point `pb_bar`, 20 rows to 300 bar, c_o 1e-4/bar);
    Corey three-phase SCAL with Stone II (Swc = Sor = 0.1, Sgc = Sgr = 0.05, Sorg = 0.15, nw = no = 2,
    ng = 1.5); initial pressure `p_init` with the saturated Rs and no free gas; gravity on; four
    corner rate injectors of `injected_fluid` and a centre BHP producer at `producer_bhp`, every
    layer perforated."""
    from .pvt import black_oil_table

    d = Deck(nx, ny, nz, 0.2)
    d.set_cell_dimensions(dx, dx, dz)
    kh, z = lognormal_field((nz, ny, nx), seed, math.log(100.0), sigma, corr_cells)
    d.set_permeability_field(kh, kh, kv_kh * kh)
    d.set_porosity_field(np.clip(0.1 + 0.02 * z, 0.05, 0.3))
    d.set_rel_perm_props(0.1, 0.1, 2.0, 2.0, 1.0, 1.0)
    d.set_fluid_properties(1.0, 0.5)
    d.set_fluid_compressibilities(1e-4, 3e-6)
    d.set_fluid_densities(800.0, 1000.0)
    d.set_rock_properties(1e-6, 0.0, 1.1, 1.0)
    d.set_capillary_params(0.0, 2.0)
    d.set_gravity_enabled(gravity)
    d.set_initial_pressure(p_init)
    d.set_initial_saturation(0.1)
    d.set_three_phase_mode_enabled(True)
    d.set_three_phase_rel_perm_props(0.1, 0.1, 0.05, 0.05, 0.15, 2.0, 2.0, 1.5, 1.0, 1.0, 1.0)
    d.set_gas_fluid_properties(0.02, 1e-4, 10.0)
    if pc_og:
        d.set_gas_oil_capillary_params(0.5, 2.0)
    d.set_pvt_table(black_oil_table(35.0, 0.75, 80.0, pb_bar, 300.0, 20, 1e-4))
    d.set_initial_gas_saturation(0.0)
    d.set_injected_fluid(injected_fluid)
    d.set_well_control_modes("rate", "pressure")
    d.set_target_well_rates(rate_per_perf * nz, 0.0)
    d.set_well_bhp_limits(50.0, 600.0)
    corners = [(0, 0), (nx - 1, 0), (0, ny - 1), (nx - 1, ny - 1)]
    for n, (i, j) in enumerate(corners):
        for k in range(nz):
            d.add_well_with_id(i, j, k, 400.0, 0.1, 0.0, True, f"INJ{n + 1}")
    for k in range(nz):
        d.add_well_with_id(nx // 2, ny // 2, k, producer_bhp, 0.1, 0.0, False, "PROD")
    return d


def mixed_precision_deck(seed: int = 7) -> Deck:
    """The 2M-cell waterflood (200 x 200 x 50) of the mixed-precision configuration."""
    return waterflood_3d(200, 200, 50, seed=seed)


def deck_digest(d: Deck) -> str:
    h = hashlib.sha256()
    for a in (d.dz, d.porosity, d.perm_x, d.perm_y, d.perm_z, d.pressure, d.sat_water, d.sat_gas, d.rs):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    for w in d.wells:
        h.update(repr((w.i, w.j, w.k, w.bhp, w.injector, w.physical_well_id)).encode())
    return h.hexdigest()[:16]
