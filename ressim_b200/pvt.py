"""Black-oil PVT tables on the host: the reference's table layout and saturated-curve lookup, and
the correlation generator its scenarios build tables with.

`PvtTable` follows src/lib/ressim/src/pvt.rs:36-186: rows in input order, oil branches of equal
Rs (PVTO style), the saturated curve made of each branch's first row, and `interpolate(p)` over
that curve (linear in 1/B and 1/(B mu) inside a segment, the first row below it, exponential Bo
and Boyle-law Bg above it).  `setPvtTable` uses the lookup to give every cell the saturated Rs
at its pressure (frontend.rs:1011-1020).

`black_oil_table` restates src/lib/physics/pvt.ts:195-292, which tabulates published
correlations: Standing (1947) bubble point, Rs and Bo; Beggs-Robinson (1975) dead and saturated
oil viscosity; Vasquez-Beggs undersaturated viscosity; Sutton (1985) pseudo-criticals;
Hall-Yarborough (1973) z-factor by Newton iteration; Lee-Gonzalez-Eakin gas viscosity.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

PVTO_RS_TOLERANCE = 1e-6
PSI_PER_BAR = 14.5037738
SCF_PER_BBL_TO_M3_PER_M3 = 0.1781076
DEFAULT_UNDERSATURATED_OIL_COMPRESSIBILITY_PER_BAR = 1e-5


@dataclass
class PvtRow:
    p_bar: float
    rs_m3m3: float
    bo_m3m3: float
    mu_o_cp: float
    bg_m3m3: float
    mu_g_cp: float

    def as_tuple(self):
        return (self.p_bar, self.rs_m3m3, self.bo_m3m3, self.mu_o_cp, self.bg_m3m3, self.mu_g_cp)


def _row(r) -> PvtRow:
    if isinstance(r, PvtRow):
        return r
    if isinstance(r, dict):
        return PvtRow(*(float(r[k]) for k in ("p_bar", "rs_m3m3", "bo_m3m3", "mu_o_cp", "bg_m3m3", "mu_g_cp")))
    return PvtRow(*(float(v) for v in r))


class PvtTable:
    """PvtTable::new (pvt.rs:86-135) and its saturated-curve lookup."""

    def __init__(self, rows, c_o: float):
        self.rows = [_row(r) for r in rows]
        self.c_o = float(c_o)
        branches: list[tuple[float, list[PvtRow]]] = []
        for row in self.rows:
            if branches:
                rs, brow = branches[-1]
                same_rs = abs(row.rs_m3m3 - rs) <= PVTO_RS_TOLERANCE
                higher = row.p_bar >= brow[-1].p_bar - 1e-9 if brow else True
                if same_rs and higher:
                    brow.append(row)
                    continue
            branches.append((row.rs_m3m3, [row]))
        for _, brow in branches:
            brow.sort(key=lambda r: r.p_bar)
        branches.sort(key=lambda b: b[0])
        self.branches = branches
        self.saturated = sorted((b[1][0] for b in branches if b[1]), key=lambda r: r.p_bar)

    def interpolate(self, p: float) -> PvtRow:
        """interpolate_rows over the saturated curve (pvt.rs:137-186)."""
        rows = self.saturated
        if not rows:
            return PvtRow(p, 0.0, 1.0, 1.0, 1.0, 0.02)
        if p <= rows[0].p_bar:
            return rows[0]
        last = rows[-1]
        if p >= last.p_bar:
            return PvtRow(p, last.rs_m3m3, last.bo_m3m3 * math.exp(-self.c_o * (p - last.p_bar)), last.mu_o_cp,
                          last.bg_m3m3 * (last.p_bar / p), last.mu_g_cp)
        for r0, r1 in zip(rows, rows[1:]):
            if r0.p_bar <= p <= r1.p_bar:
                dp = r1.p_bar - r0.p_bar
                if dp < 1e-6:
                    return r0
                t = (p - r0.p_bar) / dp
                inv_bo = (1.0 / r0.bo_m3m3) + t * (1.0 / r1.bo_m3m3 - 1.0 / r0.bo_m3m3)
                inv_bo_mu = (1.0 / (r0.bo_m3m3 * r0.mu_o_cp)) + t * (
                    1.0 / (r1.bo_m3m3 * r1.mu_o_cp) - 1.0 / (r0.bo_m3m3 * r0.mu_o_cp))
                inv_bg = (1.0 / r0.bg_m3m3) + t * (1.0 / r1.bg_m3m3 - 1.0 / r0.bg_m3m3)
                inv_bg_mu = (1.0 / (r0.bg_m3m3 * r0.mu_g_cp)) + t * (
                    1.0 / (r1.bg_m3m3 * r1.mu_g_cp) - 1.0 / (r0.bg_m3m3 * r0.mu_g_cp))
                return PvtRow(p, r0.rs_m3m3 + t * (r1.rs_m3m3 - r0.rs_m3m3), 1.0 / inv_bo, inv_bo / inv_bo_mu,
                              1.0 / inv_bg, inv_bg / inv_bg_mu)
        return last


# ---- correlations (pvt.ts:17-192) ----
def c_to_f(c):
    return c * 1.8 + 32.0


def c_to_r(c):
    return c * 1.8 + 491.67


def standing_rs(p_psia, sg_gas, api, temp_f):
    return sg_gas * math.pow(p_psia / (18.0 * math.pow(10, 0.0125 * api - 0.00091 * temp_f)), 1.0 / 0.83)


def standing_bo(rs_scf, sg_gas, sg_oil, temp_f):
    factor = rs_scf * math.pow(sg_gas / sg_oil, 0.5) + 1.25 * temp_f
    return 0.9759 + 0.000120 * math.pow(factor, 1.2)


def beggs_robinson_dead_oil_viscosity(api, temp_f):
    z = 3.0324 - 0.02023 * api - 1.163 * math.log10(temp_f)
    return math.pow(10, math.pow(10, z)) - 1.0


def beggs_robinson_saturated_oil_viscosity(mu_od, rs_scf):
    a = 10.715 * math.pow(rs_scf + 100.0, -0.515)
    b = 5.44 * math.pow(rs_scf + 150.0, -0.338)
    return a * math.pow(mu_od, b)


def vasquez_beggs_undersaturated_viscosity(mu_ob, p_psia, pb_psia):
    m = 2.6 * math.pow(p_psia, 1.187) * math.exp(-11.513 - 8.98e-5 * p_psia)
    return mu_ob * math.pow(p_psia / pb_psia, m)


def sutton_pseudo_criticals(sg_gas):
    return 169.2 + 349.5 * sg_gas - 74.0 * sg_gas * sg_gas, 756.8 - 131.0 * sg_gas - 3.6 * sg_gas * sg_gas


def hall_yarborough_z(p_psia, temp_r, tpc, ppc):
    ppr, tpr = p_psia / ppc, temp_r / tpc
    t = 1.0 / tpr
    if ppr < 0.05:
        return 1.0
    a = 0.06125 * t * math.exp(-1.2 * (1.0 - t) ** 2)
    b = t * (14.76 - 9.76 * t + 4.58 * t * t)
    c = t * (90.7 - 242.2 * t + 42.4 * t * t)
    d = 2.18 + 2.82 * t
    y = 0.001
    for _ in range(50):
        y2, y3 = y * y, y * y * y
        y4 = y3 * y
        om = 1.0 - y
        fy = (y + y2 + y3 - y4) / om ** 3 - a * ppr - b * y2 + c * math.pow(y, d)
        dfy = (1.0 + 4.0 * y + 4.0 * y2 - 4.0 * y3 + y4) / om ** 4 - 2.0 * b * y + c * d * math.pow(y, d - 1.0)
        dy = fy / dfy
        y -= dy
        if abs(dy) < 1e-6:
            break
    return a * ppr / y if y > 0 else 1.0


def lee_gonzalez_eakin_viscosity(p_psia, z, temp_r, sg_gas):
    mg = 28.96 * sg_gas
    rho = (p_psia * mg) / (z * 10.732 * temp_r) * 0.01601846
    k = (9.4 + 0.02 * mg) * math.pow(temp_r, 1.5) / (209.0 + 19.0 * mg + temp_r) * 1e-4
    x = 3.5 + 986.0 / temp_r + 0.01 * mg
    y = 2.4 - 0.2 * x
    return k * math.exp(x * math.pow(rho, y))


def black_oil_table(api: float, sg_gas: float, temp_c: float, pb_bar: float, p_max_bar: float, points: int = 30,
                    c_o_per_bar: float = DEFAULT_UNDERSATURATED_OIL_COMPRESSIBILITY_PER_BAR) -> list[PvtRow]:
    """generateBlackOilTable (pvt.ts:195-292): saturated rows up to the bubble point, then the
    bubble-point Rs with Bo shrinking as exp(-c_o (p - pb)) and Vasquez-Beggs viscosity."""
    temp_f, temp_r = c_to_f(temp_c), c_to_r(temp_c)
    pb_psia = pb_bar * PSI_PER_BAR
    sg_oil = 141.5 / (131.5 + api)
    tpc, ppc = sutton_pseudo_criticals(sg_gas)
    rs_max_scf = standing_rs(pb_psia, sg_gas, api, temp_f)
    mu_od = beggs_robinson_dead_oil_viscosity(api, temp_f)
    bo_pb = standing_bo(rs_max_scf, sg_gas, sg_oil, temp_f)
    mu_o_pb = beggs_robinson_saturated_oil_viscosity(mu_od, rs_max_scf)
    pressures = [1.0]
    dp = p_max_bar / (points - 1)
    for i in range(1, points):
        p = i * dp
        if abs(p - pb_bar) < dp * 0.5:
            p = pb_bar
        if p not in pressures:
            pressures.append(p)
    if pb_bar not in pressures:
        pressures.append(pb_bar)
    pressures.sort()
    rows = []
    for p_bar in pressures:
        p_psia = p_bar * PSI_PER_BAR
        if p_bar <= pb_bar:
            rs_scf = standing_rs(p_psia, sg_gas, api, temp_f)
            bo = standing_bo(rs_scf, sg_gas, sg_oil, temp_f)
            mu_o = beggs_robinson_saturated_oil_viscosity(mu_od, rs_scf)
        else:
            rs_scf = rs_max_scf
            mu_o = vasquez_beggs_undersaturated_viscosity(mu_o_pb, p_psia, pb_psia)
            bo = bo_pb * math.exp(-c_o_per_bar * (p_bar - pb_bar))
        z = hall_yarborough_z(p_psia, temp_r, tpc, ppc)
        mu_g = lee_gonzalez_eakin_viscosity(p_psia, z, temp_r, sg_gas)
        bg = (14.7 / 519.67) * (z * temp_r / p_psia)
        rows.append(PvtRow(p_bar, rs_scf * SCF_PER_BBL_TO_M3_PER_M3, bo, mu_o, bg, mu_g))
    return rows
