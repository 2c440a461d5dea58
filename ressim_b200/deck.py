"""Host-side mirror of the reference simulator's construction API.

`Deck` reproduces the setters, argument validation and defaults of the reference's
`ReservoirSimulator` (src/lib/ressim/src/frontend.rs:36-123 and the setters below it) for the
fields the fully implicit path reads, and serialises them into the C ABI's `RfDeck`.  Errors are
raised as `ValueError` with the reference's messages (the Rust API returns `Err(String)`).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

DEFAULT_FIM_COREY_TABLE_POINTS = 21  # src/lib/ressim/src/lib.rs:87


@dataclass
class Well:
    """One completion entry (src/lib/ressim/src/well.rs:64-90)."""
    i: int
    j: int
    k: int
    bhp: float
    well_radius: float
    skin: float
    injector: bool
    physical_well_id: str | None = None
    schedule_control: str | None = None
    schedule_target_rate: float | None = None
    schedule_target_surface_rate: float | None = None
    schedule_bhp_limit: float | None = None
    schedule_enabled: bool = True
    datum_depth_m: float | None = None
    wellbore_density_kg_m3: float | None = None


def _nan(x):
    return math.nan if x is None else float(x)


@dataclass
class Deck:
    """Static deck plus the initial state, built with the reference's setter API."""
    nx: int
    ny: int
    nz: int
    porosity_val: float
    dx: float = 10.0
    dy: float = 10.0
    dz: np.ndarray = None
    porosity: np.ndarray = None
    perm_x: np.ndarray = None
    perm_y: np.ndarray = None
    perm_z: np.ndarray = None
    pressure: np.ndarray = None
    sat_water: np.ndarray = None
    mu_o: float = 1.0
    mu_w: float = 0.5
    c_o: float = 1e-5
    c_w: float = 3e-6
    rho_o: float = 800.0
    rho_w: float = 1000.0
    b_o: float = 1.0
    b_w: float = 1.0
    water_pvt_reference_pressure_bar: float = 300.0
    rock_reference_pressure_bar: float = 300.0
    rock_compressibility: float = 0.0
    depth_reference_m: float = 0.0
    gravity_enabled: bool = False
    s_wc: float = 0.1
    s_or: float = 0.1
    n_w: float = 2.0
    n_o: float = 2.0
    k_rw_max: float = 1.0
    k_ro_max: float = 1.0
    corey_table_points: int = DEFAULT_FIM_COREY_TABLE_POINTS
    pc_entry: float = 5.0
    pc_lambda: float = 2.0
    wells: list = field(default_factory=list)
    injector_rate_controlled: bool = False
    producer_rate_controlled: bool = False
    injector_enabled: bool = True
    target_injector_rate_m3_day: float = 0.0
    target_producer_rate_m3_day: float = 0.0
    target_injector_surface_rate_m3_day: float | None = None
    target_producer_surface_rate_m3_day: float | None = None
    well_bhp_min: float = -100.0
    well_bhp_max: float = 2000.0
    three_phase_mode: bool = False
    # three-phase black-oil (frontend.rs:1011-1241)
    injected_fluid: str = "gas"  # InjectedFluid::Gas is the reference's default
    pvt_rows: list = None
    pvt_c_o: float = 0.0
    scal_3p: tuple = None
    scal_tables: tuple = None  # (swof rows (sw, krw, krow), sgof rows (sg, krg, krog))
    pc_og: tuple = None
    mu_g: float = 0.02
    c_g: float = 1e-4
    rho_g: float = 10.0
    gas_redissolution_enabled: bool = True
    sat_gas: np.ndarray = None
    rs: np.ndarray = None

    def __post_init__(self):
        n = self.nx * self.ny * self.nz
        if self.dz is None:
            self.dz = np.ones(self.nz)
        if self.porosity is None:
            self.porosity = np.full(n, float(self.porosity_val))
        if self.perm_x is None:
            self.perm_x = np.full(n, 100.0)
        if self.perm_y is None:
            self.perm_y = np.full(n, 100.0)
        if self.perm_z is None:
            self.perm_z = np.full(n, 10.0)
        if self.pressure is None:
            self.pressure = np.full(n, 300.0)
        if self.sat_water is None:
            self.sat_water = np.full(n, 0.3)
        if self.sat_gas is None:
            self.sat_gas = np.zeros(n)
        if self.rs is None:
            self.rs = np.zeros(n)

    # ---- geometry / rock (frontend.rs:573-640, 1291-1324) ----
    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    def idx(self, i, j, k) -> int:
        return (k * self.nx * self.ny) + (j * self.nx) + i

    def set_cell_dimensions(self, dx, dy, dz):
        for v in (dx, dy, dz):
            if not math.isfinite(v):
                raise ValueError("Cell dimensions must be finite numbers")
        if dx <= 0 or dy <= 0 or dz <= 0:
            raise ValueError(f"Cell dimensions must be positive, got dx={dx}, dy={dy}, dz={dz}")
        self.dx, self.dy = float(dx), float(dy)
        self.dz = np.full(self.nz, float(dz))

    def set_cell_dimensions_per_layer(self, dx, dy, dz_per_layer):
        if not (math.isfinite(dx) and math.isfinite(dy)):
            raise ValueError("Cell dimensions must be finite numbers")
        if dx <= 0 or dy <= 0:
            raise ValueError(f"Cell dimensions must be positive, got dx={dx}, dy={dy}")
        dz = np.asarray(dz_per_layer, dtype=np.float64)
        if dz.shape != (self.nz,):
            raise ValueError(f"dz_per_layer must have length equal to nz ({self.nz}), got {dz.size}")
        if not np.all(np.isfinite(dz) & (dz > 0)):
            raise ValueError("dz for every layer must be positive and finite")
        self.dx, self.dy, self.dz = float(dx), float(dy), dz.copy()

    def set_permeability_per_layer(self, kx, ky, kz):
        kx, ky, kz = (np.asarray(a, dtype=np.float64) for a in (kx, ky, kz))
        if kx.size != self.nz or ky.size != self.nz or kz.size != self.nz:
            raise ValueError(f"Permeability vectors must have length equal to nz ({self.nz})")
        layer = np.arange(self.n_cells) // (self.nx * self.ny)
        self.perm_x, self.perm_y, self.perm_z = kx[layer], ky[layer], kz[layer]

    def set_permeability_field(self, kx, ky, kz):
        arrs = [np.asarray(a, dtype=np.float64).ravel() for a in (kx, ky, kz)]
        for a in arrs:
            if a.size != self.n_cells:
                raise ValueError(f"Permeability fields must have length {self.n_cells}")
            if not np.all(np.isfinite(a) & (a > 0)):
                raise ValueError("Permeability values must be positive and finite")
        self.perm_x, self.perm_y, self.perm_z = (a.copy() for a in arrs)

    def set_porosity_field(self, phi):
        """Per-cell porosity.  The reference only takes a uniform porosity in its constructor;
        heterogeneous decks write the private porosity array directly."""
        phi = np.asarray(phi, dtype=np.float64).ravel()
        if phi.size != self.n_cells or not np.all(np.isfinite(phi) & (phi > 0)):
            raise ValueError(f"Porosity field must have {self.n_cells} positive finite values")
        self.porosity = phi.copy()

    def set_rock_properties(self, c_r, depth_reference_m, b_o, b_w):
        if not all(math.isfinite(v) for v in (c_r, depth_reference_m, b_o, b_w)):
            raise ValueError("Rock properties must be finite numbers")
        if c_r < 0:
            raise ValueError(f"Rock compressibility must be non-negative, got {c_r}")
        if b_o <= 0 or b_w <= 0:
            raise ValueError(f"Volume expansion factors must be positive, got b_o={b_o}, b_w={b_w}")
        self.rock_compressibility, self.depth_reference_m = float(c_r), float(depth_reference_m)
        self.b_o, self.b_w = float(b_o), float(b_w)

    # ---- initial state ----
    def set_initial_pressure(self, p):
        self.pressure = np.full(self.n_cells, float(p))
        self.water_pvt_reference_pressure_bar = float(p)
        self.rock_reference_pressure_bar = float(p)

    def set_initial_saturation(self, sw):
        self.sat_water = np.full(self.n_cells, min(max(float(sw), 0.0), 1.0))

    def set_initial_saturation_per_layer(self, sw):
        sw = np.asarray(sw, dtype=np.float64)
        if sw.size != self.nz:
            raise ValueError(f"Initial saturation vector must have length equal to nz ({self.nz})")
        if not np.all(np.isfinite(sw)) or np.any((sw < 0) | (sw > 1)):
            raise ValueError("Initial saturation must be finite and within [0, 1]")
        self.sat_water = sw[np.arange(self.n_cells) // (self.nx * self.ny)].copy()

    # ---- fluid / SCAL ----
    def set_rel_perm_props(self, s_wc, s_or, n_w, n_o, k_rw_max, k_ro_max):
        vals = (s_wc, s_or, n_w, n_o, k_rw_max, k_ro_max)
        if not all(math.isfinite(v) for v in vals):
            raise ValueError("Relative permeability parameters must be finite numbers")
        if s_wc < 0 or s_wc >= 1:
            raise ValueError(f"S_wc must be in [0, 1), got {s_wc}")
        if s_or < 0 or s_or >= 1:
            raise ValueError(f"S_or must be in [0, 1), got {s_or}")
        if s_wc + s_or >= 1:
            raise ValueError(f"Invalid saturation endpoints: S_wc + S_or must be < 1.0, got {s_wc + s_or}")
        if n_w <= 0 or n_o <= 0:
            raise ValueError(f"Corey exponents must be positive, got n_w={n_w}, n_o={n_o}")
        if k_rw_max < 0 or k_rw_max > 1:
            raise ValueError(f"k_rw_max must be in [0, 1], got {k_rw_max}")
        if k_ro_max <= 0 or k_ro_max > 1:
            raise ValueError(f"k_ro_max must be in (0, 1], got {k_ro_max}")
        self.s_wc, self.s_or, self.n_w, self.n_o = map(float, (s_wc, s_or, n_w, n_o))
        self.k_rw_max, self.k_ro_max = float(k_rw_max), float(k_ro_max)

    def set_fluid_properties(self, mu_o, mu_w):
        if not (math.isfinite(mu_o) and math.isfinite(mu_w)):
            raise ValueError("Fluid viscosities must be finite numbers")
        if mu_o <= 0 or mu_w <= 0:
            raise ValueError(f"Fluid viscosities must be positive, got mu_o={mu_o}, mu_w={mu_w}")
        self.mu_o, self.mu_w = float(mu_o), float(mu_w)

    def set_fluid_compressibilities(self, c_o, c_w):
        if not (math.isfinite(c_o) and math.isfinite(c_w)):
            raise ValueError("Fluid compressibilities must be finite numbers")
        if c_o < 0 or c_w < 0:
            raise ValueError(f"Fluid compressibilities must be non-negative, got c_o={c_o}, c_w={c_w}")
        self.c_o, self.c_w = float(c_o), float(c_w)

    def set_fluid_densities(self, rho_o, rho_w):
        if not (math.isfinite(rho_o) and math.isfinite(rho_w)):
            raise ValueError("Fluid densities must be finite numbers")
        if rho_o <= 0 or rho_w <= 0:
            raise ValueError(f"Fluid densities must be positive, got rho_o={rho_o}, rho_w={rho_w}")
        self.rho_o, self.rho_w = float(rho_o), float(rho_w)

    def set_capillary_params(self, p_entry, lam):
        if not (math.isfinite(p_entry) and math.isfinite(lam)):
            raise ValueError("Capillary parameters must be finite numbers")
        if p_entry < 0:
            raise ValueError(f"Capillary entry pressure must be non-negative, got {p_entry}")
        if lam <= 0:
            raise ValueError(f"Capillary lambda must be positive, got {lam}")
        self.pc_entry, self.pc_lambda = float(p_entry), float(lam)

    def set_gravity_enabled(self, enabled):
        self.gravity_enabled = bool(enabled)

    def set_fim_corey_table_points(self, points):
        self.corey_table_points = int(points)

    # ---- three-phase black-oil (frontend.rs:1011-1241) ----
    def set_three_phase_mode_enabled(self, enabled):
        self.three_phase_mode = bool(enabled)

    def set_three_phase_rel_perm_props(self, s_wc, s_or, s_gc, s_gr, s_org, n_w, n_o, n_g, k_rw_max, k_ro_max,
                                       k_rg_max):
        if s_wc + s_or + s_gc + s_gr >= 1.0:
            raise ValueError("Invalid saturation endpoints: S_wc + S_or + S_gc + S_gr must be < 1.0, got "
                             f"{s_wc + s_or + s_gc + s_gr}")
        if s_wc + s_org >= 1.0:
            raise ValueError(f"Invalid saturation endpoints: S_wc + S_org must be < 1.0, got {s_wc + s_org}")
        if n_w <= 0.0 or n_o <= 0.0 or n_g <= 0.0:
            raise ValueError(f"Corey exponents must be positive, got n_w={n_w}, n_o={n_o}, n_g={n_g}")
        self.scal_3p = tuple(float(v) for v in (s_wc, s_or, n_w, n_o, k_rw_max, k_ro_max, s_gc, s_gr, s_org, n_g,
                                                 k_rg_max))
        self.scal_tables = None  # new Corey props drop the tables, as the reference's setter does

    def set_three_phase_scal_tables(self, swof, sgof):
        """setThreePhaseScalTables (frontend.rs:1145-1158, checks relperm.rs:65-122): SWOF rows
        (sw, krw, krow[, pcow]) and SGOF rows (sg, krg, krog[, pcog]), as tuples or as dicts with
        those keys; the capillary columns are accepted and not used by the FIM path."""

        def rows(table, name, keys):
            out = []
            for r in table:
                v = [r[k] for k in keys] if isinstance(r, dict) else list(r)[:3]
                out.append([float(x) for x in v])
            if len(out) < 2:
                raise ValueError(f"{name} table must contain at least two rows")
            prev = -math.inf
            for i, (s, kr, kro) in enumerate(out):
                if not (math.isfinite(s) and math.isfinite(kr) and math.isfinite(kro)):
                    raise ValueError(f"{name} row {i} must contain finite values")
                if not (0.0 <= s <= 1.0 and 0.0 <= kr <= 1.0 and 0.0 <= kro <= 1.0):
                    raise ValueError(f"{name} row {i} must stay within [0, 1]")
                if s <= prev:
                    raise ValueError(f"{name} saturation must be strictly increasing at row {i}")
                prev = s
            return np.array(out, dtype=np.float64)

        w = rows(swof, "SWOF", ("sw", "krw", "krow"))
        g = rows(sgof, "SGOF", ("sg", "krg", "krog"))
        if self.scal_3p is None:
            raise ValueError("Three-phase relperm props must be configured before SWOF/SGOF tables")
        self.scal_tables = (w, g)

    def set_gas_oil_capillary_params(self, p_entry, lam):
        if p_entry < 0.0:
            raise ValueError(f"Gas-oil capillary entry pressure must be non-negative, got {p_entry}")
        if lam <= 0.0:
            raise ValueError(f"Gas-oil capillary lambda must be positive, got {lam}")
        self.pc_og = (float(p_entry), float(lam))

    def set_gas_fluid_properties(self, mu_g, c_g, rho_g):
        if mu_g <= 0.0:
            raise ValueError(f"Gas viscosity must be positive, got {mu_g}")
        if c_g < 0.0:
            raise ValueError(f"Gas compressibility must be non-negative, got {c_g}")
        if rho_g <= 0.0:
            raise ValueError(f"Gas density must be positive, got {rho_g}")
        self.mu_g, self.c_g, self.rho_g = float(mu_g), float(c_g), float(rho_g)

    def set_gas_redissolution_enabled(self, enabled):
        self.gas_redissolution_enabled = bool(enabled)

    def set_injected_fluid(self, fluid):
        f = fluid.lower()
        if f not in ("water", "gas"):
            raise ValueError(f"Unknown injected fluid '{f}'; expected 'water' or 'gas'")
        self.injected_fluid = f

    def set_pvt_table(self, rows):
        """setPvtTable: the table takes the current oil compressibility, and every cell gets the
        saturated Rs at its pressure."""
        from .pvt import PvtTable

        table = PvtTable(rows, self.c_o)
        self.pvt_rows = [r.as_tuple() for r in table.rows]
        self.pvt_c_o = table.c_o
        self.rs = np.array([table.interpolate(float(p)).rs_m3m3 for p in self.pressure])

    def set_initial_rs(self, rs):
        self.rs = np.full(self.n_cells, float(rs))

    def set_initial_gas_saturation(self, sat_gas):
        sg = min(max(float(sat_gas), 0.0), 1.0)
        self.sat_gas = np.minimum(sg, 1.0 - np.asarray(self.sat_water, dtype=np.float64))

    # ---- wells and controls (frontend.rs:125-345, 430-520) ----
    def add_well(self, i, j, k, bhp, well_radius, skin, injector, physical_well_id=None):
        if not (0 <= i < self.nx and 0 <= j < self.ny and 0 <= k < self.nz):
            raise ValueError(
                f"Well indices out of bounds: (i={i}, j={j}, k={k}) for grid ({self.nx}, {self.ny}, {self.nz})")
        if not math.isfinite(bhp):
            raise ValueError(f"BHP must be finite, got: {bhp}")
        if well_radius <= 0 or not math.isfinite(well_radius):
            raise ValueError(f"Well radius must be positive and finite, got: {well_radius}")
        if not math.isfinite(skin):
            raise ValueError(f"Skin factor must be finite, got: {skin}")
        if any(w.i == i and w.j == j and w.k == k for w in self.wells):
            raise ValueError(f"Multiple well completions in the same cell are not supported: ({i}, {j}, {k})")
        if bhp < -100.0 or bhp > 2000.0:
            raise ValueError(f"BHP out of reasonable range [-100, 2000] bar, got: {bhp}")
        self.wells.append(Well(int(i), int(j), int(k), float(bhp), float(well_radius), float(skin),
                               bool(injector), physical_well_id))

    def add_well_with_id(self, i, j, k, bhp, well_radius, skin, injector, physical_well_id):
        self.add_well(i, j, k, bhp, well_radius, skin, injector, physical_well_id)

    def set_well_schedule(self, physical_well_id, control_mode, target_rate_m3_day,
                          target_surface_rate_m3_day, bhp_limit, enabled):
        wid = physical_well_id.strip()
        if not wid:
            raise ValueError("Physical well id must not be empty")
        mode = control_mode.strip().lower()
        if mode in ("pressure", ""):
            mode = "pressure"
        elif mode != "rate":
            raise ValueError(f"Well control mode must be 'pressure' or 'rate', got: {mode}")
        tr = target_rate_m3_day if math.isfinite(target_rate_m3_day) and target_rate_m3_day >= 0 else None
        ts = (target_surface_rate_m3_day
              if math.isfinite(target_surface_rate_m3_day) and target_surface_rate_m3_day >= 0 else None)
        bl = bhp_limit if math.isfinite(bhp_limit) else None
        hit = False
        for w in self.wells:
            if w.physical_well_id == wid:
                w.schedule_control, w.schedule_target_rate = mode, tr
                w.schedule_target_surface_rate, w.schedule_bhp_limit = ts, bl
                w.schedule_enabled = bool(enabled)
                hit = True
        if not hit:
            raise ValueError(f"No well found for physical well id '{wid}'")

    def set_rate_controlled_wells(self, enabled):
        self.injector_rate_controlled = self.producer_rate_controlled = bool(enabled)

    def set_well_control_modes(self, injector_mode, producer_mode):
        self.injector_rate_controlled = injector_mode.lower() == "rate"
        self.producer_rate_controlled = producer_mode.lower() == "rate"

    def set_injector_enabled(self, enabled):
        self.injector_enabled = bool(enabled)

    def set_target_well_rates(self, injector_rate_m3_day, producer_rate_m3_day):
        if not (math.isfinite(injector_rate_m3_day) and math.isfinite(producer_rate_m3_day)):
            raise ValueError("Target well rates must be finite numbers")
        if injector_rate_m3_day < 0 or producer_rate_m3_day < 0:
            raise ValueError("Target well rates must be non-negative, got "
                             f"injector={injector_rate_m3_day}, producer={producer_rate_m3_day}")
        self.target_injector_rate_m3_day = float(injector_rate_m3_day)
        self.target_producer_rate_m3_day = float(producer_rate_m3_day)

    def set_target_well_surface_rates(self, injector_rate_m3_day, producer_rate_m3_day):
        if not (math.isfinite(injector_rate_m3_day) and math.isfinite(producer_rate_m3_day)):
            raise ValueError("Target well surface rates must be finite numbers")
        if injector_rate_m3_day < 0 or producer_rate_m3_day < 0:
            raise ValueError("Target well surface rates must be non-negative")
        self.target_injector_surface_rate_m3_day = float(injector_rate_m3_day) if injector_rate_m3_day > 0 else None
        self.target_producer_surface_rate_m3_day = float(producer_rate_m3_day) if producer_rate_m3_day > 0 else None

    def set_well_bhp_limits(self, bhp_min, bhp_max):
        if not (math.isfinite(bhp_min) and math.isfinite(bhp_max)):
            raise ValueError("Well BHP limits must be finite numbers")
        if bhp_min > bhp_max:
            raise ValueError(f"Invalid BHP limits: bhp_min ({bhp_min}) must be <= bhp_max ({bhp_max})")
        self.well_bhp_min, self.well_bhp_max = float(bhp_min), float(bhp_max)

    # ---- serialisation ----
    def to_abi(self):
        """Return an `RfDeck` plus the list of buffers that must stay alive while it is used."""
        keep = []

        def arr(a, n):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
            if a.size != n:
                raise ValueError(f"array has {a.size} values, expected {n}")
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        ids: dict[str, int] = {}
        wells = (_abi.RfWell * max(len(self.wells), 1))()
        for n, w in enumerate(self.wells):
            pid = -1
            if w.physical_well_id is not None:
                pid = ids.setdefault(w.physical_well_id, len(ids))
            has_sched = int(w.schedule_control is not None or w.schedule_target_rate is not None
                            or w.schedule_target_surface_rate is not None
                            or w.schedule_bhp_limit is not None or not w.schedule_enabled)
            ctl = {None: 0, "pressure": 1, "rate": 2}[w.schedule_control]
            wells[n] = _abi.RfWell(
                w.i, w.j, w.k, int(w.injector), pid, has_sched, int(w.schedule_enabled), ctl,
                w.bhp, w.well_radius, w.skin, _nan(w.schedule_target_rate),
                _nan(w.schedule_target_surface_rate), _nan(w.schedule_bhp_limit),
                _nan(w.datum_depth_m), _nan(w.wellbore_density_kg_m3))
        keep.append(wells)
        n = self.n_cells
        d = _abi.RfDeck()
        d.abi_version = _abi.RF_ABI_VERSION
        d.nx, d.ny, d.nz = self.nx, self.ny, self.nz
        d.dx, d.dy = self.dx, self.dy
        d.dz = arr(self.dz, self.nz)
        d.porosity = arr(self.porosity, n)
        d.perm_x, d.perm_y, d.perm_z = arr(self.perm_x, n), arr(self.perm_y, n), arr(self.perm_z, n)
        for name in ("mu_o", "mu_w", "c_o", "c_w", "rho_o", "rho_w", "b_o", "b_w",
                     "water_pvt_reference_pressure_bar", "rock_compressibility",
                     "rock_reference_pressure_bar", "depth_reference_m", "s_wc", "s_or", "n_w", "n_o",
                     "k_rw_max", "k_ro_max", "pc_entry", "pc_lambda", "target_injector_rate_m3_day",
                     "target_producer_rate_m3_day", "well_bhp_min", "well_bhp_max"):
            setattr(d, name, float(getattr(self, name)))
        d.gravity_enabled = int(self.gravity_enabled)
        d.corey_table_points = int(self.corey_table_points)
        d.n_wells = len(self.wells)
        d.wells = C.cast(wells, C.POINTER(_abi.RfWell))
        d.injector_rate_controlled = int(self.injector_rate_controlled)
        d.producer_rate_controlled = int(self.producer_rate_controlled)
        d.injector_enabled = int(self.injector_enabled)
        d.target_injector_surface_rate_m3_day = _nan(self.target_injector_surface_rate_m3_day)
        d.target_producer_surface_rate_m3_day = _nan(self.target_producer_surface_rate_m3_day)
        d.three_phase_mode = int(self.three_phase_mode)
        d.injected_fluid = 1 if self.injected_fluid == "gas" else 0
        if self.pvt_rows:
            d.n_pvt_rows = len(self.pvt_rows)
            d.pvt_rows = arr(np.array(self.pvt_rows, dtype=np.float64), 6 * len(self.pvt_rows))
            d.pvt_c_o = float(self.pvt_c_o)
        if self.scal_3p is not None:
            d.has_scal_3p = 1
            (d.s_wc_3p, d.s_or_3p, d.n_w_3p, d.n_o_3p, d.k_rw_max_3p, d.k_ro_max_3p, d.s_gc, d.s_gr, d.s_org,
             d.n_g, d.k_rg_max) = self.scal_3p
        if self.pc_og is not None:
            d.has_pc_og = 1
            d.pc_og_entry, d.pc_og_lambda = self.pc_og
        d.mu_g, d.c_g, d.rho_g = self.mu_g, self.c_g, self.rho_g
        d.gas_redissolution_enabled = int(self.gas_redissolution_enabled)
        if self.scal_tables is not None:
            w, g = (np.ascontiguousarray(t, dtype=np.float64) for t in self.scal_tables)
            d.n_swof_rows, d.swof_rows = len(w), arr(w, 3 * len(w))
            d.n_sgof_rows, d.sgof_rows = len(g), arr(g, 3 * len(g))
        return d, keep
