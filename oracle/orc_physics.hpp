// ORACLE — test infrastructure only (see orc_core.hpp).  Physics of the reference FIM path:
// PVT, relative permeability, capillary pressure, cell properties (two-phase oil-water and the
// three-phase black-oil regimes), accumulation, face flux and the AD well model.
#pragma once

#include <map>
#include <string>
#include <tuple>

#include "../include/ressim_fim.h"
#include "orc_blackoil.hpp"
#include "orc_core.hpp"

namespace orc {

constexpr double DARCY_METRIC_FACTOR = 8.5269888e-3;  // fim/assembly.rs:29, fim/wells.rs:9
constexpr double GRAVITY = 9.80665;
constexpr double FB_EPSILON = 1e-6;  // fim/wells.rs:1582

struct Perf {
  int entry, well, cell, i, j, k;
  bool injector;
  bool has_wi;
  double wi;  // geometric well index (Peaceman)
};
struct PWell {
  int rep_entry;
  bool injector;
  std::vector<int> perfs;
};
struct Topo {
  std::vector<PWell> wells;
  std::vector<Perf> perfs;
};

struct Control {
  bool enabled, rate_controlled, uses_surface_target, has_target;
  double target_rate, bhp_limit, bhp_target;
};

struct Cell {
  double p, sw, hc;
  int regime;  // 0 saturated, 1 undersaturated
  // gas redissolution off (DRSDT0): the simulator's Rs of the cell at the substep start, which
  // caps Rs in the flash, the regime test and the properties; NaN when redissolution is on
  double base_rs = NAN;
};
struct State {
  std::vector<Cell> cells;
  std::vector<double> bhp;  // per physical well
  std::vector<double> q;    // per perforation (reservoir connection rate primary)
  int n_cells() const { return int(cells.size()); }
  int n_unknowns() const { return 3 * n_cells() + int(bhp.size()) + int(q.size()); }
  int bhp_off(int w) const { return 3 * n_cells() + w; }
  int q_off(int p) const { return 3 * n_cells() + int(bhp.size()) + p; }
};

struct Sim {
  int nx = 0, ny = 0, nz = 0;
  double dx = 0, dy = 0;
  std::vector<double> dz, porosity, kx, ky, kz;
  double mu_o = 1, mu_w = 0.5, c_o = 1e-5, c_w = 3e-6, rho_o = 800, rho_w = 1000;
  double b_o = 1, b_w = 1, p_wref = 300, c_r = 0, p_rref = 300, depth_ref = 0;
  double rho_g = 10.0;  // surface gas density [kg/m3] (frontend.rs:117)
  // three-phase black-oil (frontend.rs:1011-1241); absent parts keep the reference's defaults
  bool three_phase = false;
  bool has_pvt = false;
  PvtTable pvt;
  bool has_scal3 = false;
  Scal3 scal3{};
  bool has_pc_og = false;
  double pcog_entry = 0.0, pcog_lambda = 2.0;
  double mu_g = 0.02, c_g = 1e-4;
  int injected_fluid = 1;  // 0 water, 1 gas (InjectedFluid::Gas is the reference default)
  bool gas_redissolution = true;
  bool gravity = false;
  double s_wc = 0.1, s_or = 0.1, n_w = 2, n_o = 2, krw_max = 1, kro_max = 1;
  int table_points = 21;
  double pc_entry = 5, pc_lambda = 2;
  std::vector<RfWell> wells;
  std::vector<double> head_offset;
  bool inj_rate_ctl = false, prod_rate_ctl = false, inj_enabled = true;
  double tgt_inj = 0, tgt_prod = 0, tgt_inj_surf = NAN, tgt_prod_surf = NAN;
  double bhp_min = -100, bhp_max = 2000;
  // simulator state
  std::vector<double> pressure, sat_water, sat_oil, sat_gas, rs;
  double time_days = 0;
  std::vector<RfTimePointRates> rate_history;
  double cum_inj = 0, cum_prod = 0, cum_mb = 0, cum_mb_oil = 0, cum_mb_gas = 0;
  std::string last_warning;
  Topo topo;

  int n() const { return nx * ny * nz; }
  int idx(int i, int j, int k) const { return k * nx * ny + j * nx + i; }
  double dz_at(int id) const { return dz[id / (nx * ny)]; }
  double pore_volume_m3(int id) const { return dx * dy * dz_at(id) * porosity[id]; }
  double depth_at_k(int k) const {
    double d = depth_ref;
    for (int l = 0; l < k; ++l) d += dz[l];
    return d + dz[k] * 0.5;
  }
};

// grid.rs:3-9
inline double harmonic_mean(double a, double b) { return a + b == 0.0 ? 0.0 : 2.0 * a * b / (a + b); }

// grid.rs:47-80
inline double geometric_transmissibility(const Sim& s, int id1, int id2, char dim) {
  const int k1 = id1 / (s.nx * s.ny), k2 = id2 / (s.nx * s.ny);
  const double dz1 = s.dz[k1], dz2 = s.dz[k2];
  if (dim == 'x') return harmonic_mean(s.kx[id1], s.kx[id2]) * (s.dy * dz1) / s.dx;
  if (dim == 'y') return harmonic_mean(s.ky[id1], s.ky[id2]) * (s.dx * dz1) / s.dy;
  const double p1 = s.kz[id1], p2 = s.kz[id2];
  const double denom = p2 * dz1 + p1 * dz2;
  if (denom <= 0.0) return 0.0;
  return 2.0 * p1 * p2 * (s.dx * s.dy) / denom;
}

// ---- PVT (pvt.rs:603-618, 620-626, 988-1009) ----
template <class S>
inline S water_inverse_fvf_g(const Sim& s, const S& p) {
  S x = (p - s.p_wref) * s.c_w;
  return (sc<S>(1.0) + x * (sc<S>(1.0) + x * 0.5)) / rmax(s.b_w, 1e-9);
}
inline double water_fvf(const Sim& s, double p) { return 1.0 / rmax(water_inverse_fvf_g(s, p), 1e-9); }
template <class S>
inline S water_density_g(const Sim& s, const S& p) {
  return water_inverse_fvf_g(s, p) * s.rho_w;
}
template <class S>
inline S base_oil_fvf_g(const Sim& s, const S& p) {
  return max_floor(sc<S>(s.b_o) * s_exp(p * (-s.c_o)), 1e-9);
}
inline double base_oil_fvf(const Sim& s, double p) { return rmax(s.b_o * std::exp(-s.c_o * p), 1e-9); }
// ---- simulator-level black-oil accessors (pvt.rs:628-1009) ----
// get_b_g (pvt.rs:835-841)
inline double get_b_g(const Sim& s, double p) { return s.has_pvt ? pvt_interpolate(s.pvt, p).bg : 1.0; }
// get_mu_g (pvt.rs:665-671)
inline double get_mu_g(const Sim& s, double p) { return s.has_pvt ? pvt_interpolate(s.pvt, p).mu_g : s.mu_g; }
// get_b_o_for_rs (pvt.rs:792-803)
inline double get_b_o_for_rs(const Sim& s, double p, double rs) {
  if (!s.has_pvt) return base_oil_fvf(s, p);
  if (!s.three_phase) return pvt_interpolate(s.pvt, p).bo;
  double bo, mu;
  pvt_interpolate_oil(s.pvt, p, rs, bo, mu);
  return bo;
}
// get_mu_o_for_rs (pvt.rs:649-659)
inline double get_mu_o_for_rs(const Sim& s, double p, double rs) {
  if (!s.has_pvt) return s.mu_o;
  if (!s.three_phase) return pvt_interpolate(s.pvt, p).mu_o;
  double bo, mu;
  pvt_interpolate_oil(s.pvt, p, rs, bo, mu);
  return mu;
}
// get_b_o_cell / get_mu_o_cell (pvt.rs:636-647, 769-779): the simulator's Rs of the cell
inline double get_b_o_cell(const Sim& s, int id, double p) { return get_b_o_for_rs(s, p, s.rs[id]); }
inline double get_mu_o_cell(const Sim& s, int id, double p) { return get_mu_o_for_rs(s, p, s.rs[id]); }
// get_mu_o_for_rs_generic / get_mu_g_generic (pvt.rs:674-693)
template <class S>
inline S mu_o_for_rs_g(const Sim& s, const S& p, const S& rs) {
  if (!s.has_pvt) return sc<S>(s.mu_o);
  if (!s.three_phase) return pvt_saturated_g(s.pvt, p).mu_o;
  S bo, mu;
  pvt_oil_g(s.pvt, p, rs, bo, mu);
  return mu;
}
template <class S>
inline S mu_g_g(const Sim& s, const S& p) {
  return s.has_pvt ? pvt_saturated_g(s.pvt, p).mu_g : sc<S>(s.mu_g);
}
// oil_density_generic / gas_density_generic (pvt.rs:988-1009)
template <class S>
inline S oil_density_g(const Sim& s, const S& p, const S& rs) {
  if (s.has_pvt) {
    S bo, mu;
    pvt_oil_g(s.pvt, p, rs, bo, mu);
    return (sc<S>(s.rho_o) + rs * s.rho_g) / max_floor(bo, 1e-9);
  }
  S bo = max_floor(sc<S>(s.b_o) * s_exp(p * (-s.c_o)), 1e-9);
  return sc<S>(s.rho_o) / bo;
}
template <class S>
inline S gas_density_g(const Sim& s, const S& p) {
  if (s.has_pvt) return sc<S>(s.rho_g) / max_floor(pvt_saturated_g(s.pvt, p).bg, 1e-9);
  return sc<S>(s.rho_g);
}

// ---- relperm (relperm.rs:491-629) ----
inline double k_rw(const Sim& s, double sw) {
  const double e = rclamp((sw - s.s_wc) / (1.0 - s.s_wc - s.s_or), 0.0, 1.0);
  return s.krw_max * std::pow(e, s.n_w);
}
inline double k_ro(const Sim& s, double sw) {
  const double e = rclamp((1.0 - sw - s.s_or) / (1.0 - s.s_wc - s.s_or), 0.0, 1.0);
  return s.kro_max * std::pow(e, s.n_o);
}
template <class S>
inline void corey_table_g(const Sim& s, const S& sw, S& krw, S& kro) {
  const int points = std::max(s.table_points, 2);
  const double lo = s.s_wc, hi = 1.0 - s.s_or;
  const double span = rmax(hi - lo, 1e-12);
  const double step = span / double(points - 1);
  auto knot_x = [&](int i) { return rmin(lo + double(i) * step, hi); };
  const double v = val(sw);
  if (v <= lo) {
    const double x = knot_x(0);
    krw = sc<S>(k_rw(s, x));
    kro = sc<S>(k_ro(s, x));
    return;
  }
  if (v >= hi) {
    const double x = knot_x(points - 1);
    krw = sc<S>(k_rw(s, x));
    kro = sc<S>(k_ro(s, x));
    return;
  }
  const int seg = std::min(int(std::floor((v - lo) / step)), points - 2);
  const double x0 = knot_x(seg), x1 = knot_x(seg + 1);
  const double krw0 = k_rw(s, x0), kro0 = k_ro(s, x0), krw1 = k_rw(s, x1), kro1 = k_ro(s, x1);
  S t = min_ceil(max_floor((sw - x0) / (x1 - x0), 0.0), 1.0);
  krw = t * (krw1 - krw0) + krw0;
  kro = t * (kro1 - kro0) + kro0;
}
// analytic Corey generic mirrors, used when the table is switched off (points == 0)
template <class S>
inline void corey_analytic_g(const Sim& s, const S& sw, S& krw, S& kro) {
  const double denom = 1.0 - s.s_wc - s.s_or;
  S ew = min_ceil(max_floor((sw - s.s_wc) / denom, 0.0), 1.0);
  krw = s_powf(ew, s.n_w) * s.krw_max;
  S eo = min_ceil(max_floor((sc<S>(1.0 - s.s_or) - sw) / denom, 0.0), 1.0);
  kro = s_powf(eo, s.n_o) * s.kro_max;
}
template <class S>
inline void two_phase_relperm_g(const Sim& s, const S& sw, S& krw, S& kro) {
  if (s.table_points > 0)
    corey_table_g(s, sw, krw, kro);
  else
    corey_analytic_g(s, sw, krw, kro);
}

// ---- capillary (capillary.rs:73-97) ----
template <class S>
inline S capillary_pressure_g(const Sim& s, const S& sw) {
  const double denom = 1.0 - s.s_wc - s.s_or;
  S e = min_ceil(max_floor((sw - s.s_wc) / denom, 0.0), 1.0);
  if (val(e) >= 1.0) return sc<S>(0.0);
  const double pc_max = s.pc_entry * 20.0;
  if (val(e) <= 0.0) return sc<S>(pc_max);
  S pc = s_powf(e, -1.0 / s.pc_lambda) * s.pc_entry;
  return min_ceil(max_floor(pc, 0.0), pc_max);
}

// ---- mobility (mobility.rs:114-149 f64; 196-249 generic) ----
template <class S>
struct Mob {
  S w, o, g;
};
template <class S>
inline Mob<S> phase_mobilities_g(const Sim& s, const S& sw, const S& sg, const S& p, const S& rs) {
  const S mu_w = sc<S>(s.mu_w);
  Mob<S> m;
  if (s.three_phase) {
    if (!s.has_scal3) {
      S krw, kro;
      corey_analytic_g(s, sw, krw, kro);
      m.w = krw / mu_w;
      m.o = kro / mu_o_for_rs_g(s, p, rs);
      m.g = sc<S>(0.0);
      return m;
    }
    m.w = k_rw3_g(s.scal3, sw) / mu_w;
    m.o = k_ro_stone2_g(s.scal3, sw, sg) / mu_o_for_rs_g(s, p, rs);
    m.g = k_rg3_g(s.scal3, sg) / mu_g_g(s, p);
    return m;
  }
  S krw, kro;
  two_phase_relperm_g(s, sw, krw, kro);
  m.w = krw / mu_w;
  m.o = kro / mu_o_for_rs_g(s, p, rs);
  m.g = sc<S>(0.0);
  return m;
}
inline Mob<double> phase_mobilities_f64(const Sim& s, double sw, double sg, double p, double rs) {
  if (s.three_phase) {
    if (!s.has_scal3) return Mob<double>{k_rw(s, sw) / s.mu_w, k_ro(s, sw) / get_mu_o_for_rs(s, p, rs), 0.0};
    return Mob<double>{k_rw3(s.scal3, sw) / s.mu_w, k_ro_stone2(s.scal3, sw, sg) / get_mu_o_for_rs(s, p, rs),
                       k_rg3(s.scal3, sg) / get_mu_g(s, p)};
  }
  double krw, kro;
  two_phase_relperm_g(s, sw, krw, kro);
  return Mob<double>{krw / s.mu_w, kro / get_mu_o_for_rs(s, p, rs), 0.0};
}

// ---- the gas flash (step.rs:65-200, fim/flash_ad.rs:25-207, fim/flash.rs:13-160) ----
// solve_rs_for_dissolved_gas: 64 bisection steps on dissolved(rs) = So PV rs / Bo(p, rs)
inline double solve_rs_plain(const Sim& s, double p, double sw, double sg, double pv, double dissolved,
                             double rs_upper) {
  if (!s.has_pvt) return 0.0;
  const double target = rmax(dissolved, 0.0);
  if (target <= 0.0 || rs_upper <= 0.0) return 0.0;
  const double so = rmax(1.0 - sw - sg, 0.0);
  if (so <= 1e-12 || pv <= 0.0) return 0.0;
  double lo = 0.0, hi = rmax(rs_upper, 0.0);
  for (int i = 0; i < 64; ++i) {
    const double mid = 0.5 * (lo + hi);
    double bo, mu;
    pvt_interpolate_oil(s.pvt, p, mid, bo, mu);
    const double d = (so * pv / rmax(bo, 1e-9)) * mid;
    if (d < target)
      lo = mid;
    else
      hi = mid;
  }
  return 0.5 * (lo + hi);
}

// split_gas_inventory_after_transport (step.rs:106-200); base_rs: the DRSDT0 cap (NaN: none)
inline void split_gas_plain(const Sim& s, double p, double pv, double sw, double free_sc, double dissolved_sc,
                            double base_rs, double& sg, double& so, double& rs) {
  const double total_hc = rmax(1.0 - sw, 0.0);
  const double bg = rmax(get_b_g(s, p), 1e-9);
  const double free_t = rmax(free_sc, 0.0);
  const double sg_t = rclamp((free_t * bg) / rmax(pv, 1e-9), 0.0, total_hc);
  const double so_t = rmax(total_hc - sg_t, 0.0);
  const double dissolved = rmax(dissolved_sc, 0.0);
  const double rs_max = rmax(pvt_interpolate(s.pvt, p).rs, 0.0);
  const bool redis = s.gas_redissolution;
  const double cap = redis ? rs_max : (std::isnan(base_rs) ? rs_max : rmin(rmax(base_rs, 0.0), rs_max));
  double bo_cap, mu;
  pvt_interpolate_oil(s.pvt, p, cap, bo_cap, mu);
  bo_cap = rmax(bo_cap, 1e-9);
  if (!redis) {
    const double max_t = (so_t * pv / bo_cap) * cap;
    if (dissolved <= max_t + 1e-9) {
      rs = solve_rs_plain(s, p, sw, sg_t, pv, dissolved, cap);
      sg = sg_t;
      so = so_t;
      return;
    }
  }
  const double total_gas = free_t + dissolved;
  double rs_sat, bo_sat;
  if (redis) {
    double bo_sat_raw;
    pvt_interpolate_oil(s.pvt, p, rs_max, bo_sat_raw, mu);
    rs_sat = rs_max;
    bo_sat = rmax(bo_sat_raw, 1e-9);
  } else {
    rs_sat = cap;
    bo_sat = bo_cap;
  }
  const double max_all = (total_hc * pv / bo_sat) * rs_sat;
  if (redis && total_gas <= max_all + 1e-9) {
    rs = solve_rs_plain(s, p, sw, 0.0, pv, total_gas, rs_sat);
    sg = 0.0;
    so = total_hc;
    return;
  }
  const double denom = (1.0 / bg) - (rs_sat / bo_sat);
  const double sg_sat = std::fabs(denom) > 1e-12 ? ((total_gas / pv) - (total_hc * rs_sat / bo_sat)) / denom : sg_t;
  sg = rclamp(sg_sat, redis ? 0.0 : sg_t, total_hc);
  so = rmax(total_hc - sg, 0.0);
  rs = rs_sat;
}

// dissolved_gas_value_generic (flash_ad.rs:29-43)
template <class S>
inline S dissolved_gas_g(const Sim& s, const S& p, const S& rs, const S& so, const S& pv) {
  S bo = sc<S>(1.0), mu;
  if (s.has_pvt) pvt_oil_g(s.pvt, p, rs, bo, mu);
  return (so * pv / max_floor(bo, 1e-9)) * rs;
}
// solve_rs_for_dissolved_gas_generic (flash_ad.rs:46-100): the plain bisection's root, with its
// derivative from one implicit-function Newton step
template <class S>
inline S solve_rs_g(const Sim& s, const S& p, const S& sw, const S& sg, const S& pv, const S& dissolved,
                    double rs_upper) {
  const double rs_star = solve_rs_plain(s, val(p), val(sw), val(sg), val(pv), val(dissolved), rs_upper);
  S so = max_floor(sc<S>(1.0) - sw - sg, 0.0);
  S target = max_floor(dissolved, 0.0);
  const double dgdrs = dissolved_gas_g<Ad<1>>(s, ad_const<1>(val(p)), ad_var<1>(rs_star, 0),
                                              ad_const<1>(val(so)), ad_const<1>(val(pv)))
                           .d[0];
  if (std::fabs(dgdrs) < 1e-14) return sc<S>(rs_star);
  S g = dissolved_gas_g<S>(s, p, sc<S>(rs_star), so, pv) - target;
  return sc<S>(rs_star) - g / dgdrs;
}
// split_gas_inventory_after_transport_generic (flash_ad.rs:104-207); base_rs: the DRSDT0 cap
template <class S>
inline void split_gas_g(const Sim& s, const S& p, const S& pv, const S& sw, const S& free_sc, const S& dissolved_sc,
                        double base_rs, S& sg, S& so, S& rs) {
  const PvtTable& t = s.pvt;
  S total_hc = max_floor(sc<S>(1.0) - sw, 0.0);
  S bg = max_floor(pvt_saturated_g(t, p).bg, 1e-9);
  S free_t = max_floor(free_sc, 0.0);
  S sg_t = min_of(max_floor((free_t * bg) / max_floor(pv, 1e-9), 0.0), total_hc);
  S so_t = max_floor(total_hc - sg_t, 0.0);
  S dissolved = max_floor(dissolved_sc, 0.0);
  S rs_max = max_floor(pvt_saturated_g(t, p).rs, 0.0);
  const bool redis = s.gas_redissolution;
  S cap = (redis || std::isnan(base_rs)) ? rs_max : min_of(sc<S>(rmax(base_rs, 0.0)), rs_max);
  S bo_cap, mu;
  pvt_oil_g(t, p, cap, bo_cap, mu);
  bo_cap = max_floor(bo_cap, 1e-9);
  if (!redis) {
    S max_t = (so_t * pv / bo_cap) * cap;
    if (val(dissolved) <= val(max_t) + 1e-9) {
      rs = solve_rs_g(s, p, sw, sg_t, pv, dissolved, val(cap));
      sg = sg_t;
      so = so_t;
      return;
    }
  }
  S total_gas = free_t + dissolved;
  S rs_sat, bo_sat;
  if (redis) {
    S bo_sat_raw;
    pvt_oil_g(t, p, rs_max, bo_sat_raw, mu);
    rs_sat = rs_max;
    bo_sat = max_floor(bo_sat_raw, 1e-9);
  } else {
    rs_sat = cap;
    bo_sat = bo_cap;
  }
  S max_all = (total_hc * pv / bo_sat) * rs_sat;
  if (redis && val(total_gas) <= val(max_all) + 1e-9) {
    rs = solve_rs_g(s, p, sw, sc<S>(0.0), pv, total_gas, val(rs_sat));
    sg = sc<S>(0.0);
    so = total_hc;
    return;
  }
  S denom = s_recip(bg) - (rs_sat / bo_sat);
  S sg_sat = std::fabs(val(denom)) > 1e-12 ? ((total_gas / pv) - (total_hc * rs_sat / bo_sat)) / denom : sg_t;
  sg = min_of(max_of(sg_sat, redis ? sc<S>(0.0) : sg_t), total_hc);
  so = max_floor(total_hc - sg, 0.0);
  rs = rs_sat;
}

// classify_cell_regime (flash.rs:13-40): 0 saturated, 1 undersaturated; base_rs: DRSDT0 cap
inline int classify_cell_regime(const Sim& s, double p, double sg, double rs, double base_rs = NAN) {
  if (!s.three_phase || !s.has_pvt) return 0;
  if (sg > 1e-9) return 0;
  double rs_sat = pvt_interpolate(s.pvt, p).rs;
  if (!std::isnan(base_rs)) rs_sat = rmin(rs_sat, base_rs);
  return rs < rs_sat - 1e-6 ? 1 : 0;
}

// ---- cell properties (properties.rs:37-133) ----
template <class S>
struct Props {
  S so, sg, rs, bo, bg;
};
template <class S>
inline Props<S> cell_props_g(const Sim& s, int regime, const S& p, const S& sw, const S& hc, double base_rs = NAN) {
  const S one = sc<S>(1.0);
  const S raw_total = one - sw;
  Props<S> pr;
  if (!s.three_phase || !s.has_pvt) {
    const S total = max_floor(raw_total, 0.0);
    pr.sg = min_of(max_floor(hc, 0.0), total);
    pr.so = max_floor(one - sw - pr.sg, 0.0);
    pr.bo = base_oil_fvf_g(s, p);
    pr.rs = sc<S>(0.0);
    pr.bg = sc<S>(1.0);
    return pr;
  }
  const PvtTable& t = s.pvt;
  S mu;
  if (regime == 0) {
    pr.sg = hc;
    pr.rs = pvt_saturated_g(t, p).rs;
    if (!std::isnan(base_rs)) pr.rs = min_ceil(pr.rs, base_rs);
    pr.so = raw_total - pr.sg;
    pvt_oil_g(t, p, pr.rs, pr.bo, mu);
    pr.bg = pvt_saturated_g(t, p).bg;
    return pr;
  }
  S rs_cap = max_floor(pvt_saturated_g(t, p).rs, 0.0);
  if (!std::isnan(base_rs)) rs_cap = min_of(rs_cap, sc<S>(rmax(base_rs, 0.0)));
  const S& rs_trial = hc;
  if (val(rs_trial) <= val(rs_cap) + 1e-6) {
    pr.sg = sc<S>(0.0);
    pr.so = raw_total;
    pr.rs = rs_trial;
  } else {
    S bo_t;
    pvt_oil_g(t, p, rs_trial, bo_t, mu);
    bo_t = max_floor(bo_t, 1e-9);
    S dissolved = raw_total * rs_trial / bo_t;
    split_gas_g(s, p, sc<S>(1.0), sw, sc<S>(0.0), dissolved, base_rs, pr.sg, pr.so, pr.rs);
  }
  pvt_oil_g(t, p, pr.rs, pr.bo, mu);
  pr.bg = pvt_saturated_g(t, p).bg;
  return pr;
}

template <class S>
inline S pore_volume_g(const Sim& s, int cell, const S& p) {
  return sc<S>(s.pore_volume_m3(cell)) * s_exp((p - s.p_rref) * s.c_r);
}

template <class S>
inline void component_inventory_g(const Sim& s, const S& pv, const S& p, const S& sw,
                                  const Props<S>& pr, S out[3]) {
  out[0] = pv * sw * water_inverse_fvf_g(s, p);
  out[1] = pv * pr.so / max_floor(pr.bo, 1e-9);
  out[2] = pv * pr.sg / max_floor(pr.bg, 1e-9) + out[1] * pr.rs;
}

// properties.rs:171-212: the previous inventory is evaluated with the previous regime
template <class S>
inline void cell_accumulation_g(const Sim& s, int cell, int regime, const S& p, const S& sw, const S& hc,
                                double pp, double psw, double phc, int pregime, S out[3], double base_rs = NAN) {
  Props<S> pr = cell_props_g(s, regime, p, sw, hc, base_rs);
  S pv = pore_volume_g(s, cell, p);
  S cur[3];
  component_inventory_g(s, pv, p, sw, pr, cur);
  Props<double> ppr = cell_props_g<double>(s, pregime, pp, psw, phc, base_rs);
  double ppv = pore_volume_g<double>(s, cell, pp);
  double prev[3];
  component_inventory_g<double>(s, ppv, pp, psw, ppr, prev);
  for (int c = 0; c < 3; ++c) out[c] = cur[c] - prev[c];
}

// ---- face flux (flux.rs:42-191) ----
template <class S>
struct FaceIn {
  S p, sw, hc;
  double depth;
  int regime;
  double base_rs = NAN;  // DRSDT0 cap
};
template <class S>
inline S gravity_head_g(const Sim& s, double di, double dj, const S& ri, const S& rj) {
  if (!s.gravity) return sc<S>(0.0);
  S avg = (ri + rj) * 0.5;
  return avg * (GRAVITY * (di - dj) * 1e-5);
}
// gas_oil_capillary_pressure_generic (flux.rs:137-142)
template <class S>
inline S gas_oil_pc_g(const Sim& s, const S& sg) {
  if (s.has_pc_og && s.has_scal3) return pc_og_g(s.scal3, s.pcog_entry, s.pcog_lambda, sg);
  return sc<S>(0.0);
}
template <class S>
inline void face_flux_g(const Sim& s, double geom_t, const FaceIn<S>& i, const FaceIn<S>& j,
                        S flux[3]) {
  Props<S> pi = cell_props_g(s, i.regime, i.p, i.sw, i.hc, i.base_rs);
  Props<S> pj = cell_props_g(s, j.regime, j.p, j.sw, j.hc, j.base_rs);
  S rwi = water_density_g(s, i.p), rwj = water_density_g(s, j.p);
  S roi = oil_density_g(s, i.p, pi.rs), roj = oil_density_g(s, j.p, pj.rs);
  S rgi = gas_density_g(s, i.p), rgj = gas_density_g(s, j.p);
  S pcwi = capillary_pressure_g(s, i.sw), pcwj = capillary_pressure_g(s, j.sw);
  S pcogi = gas_oil_pc_g(s, pi.sg), pcogj = gas_oil_pc_g(s, pj.sg);
  S gw = gravity_head_g(s, i.depth, j.depth, rwi, rwj);
  S go = gravity_head_g(s, i.depth, j.depth, roi, roj);
  S gg = gravity_head_g(s, i.depth, j.depth, rgi, rgj);
  S dphi_w = (i.p - j.p) - (pcwi - pcwj) - gw;
  S dphi_o = (i.p - j.p) - go;
  S dphi_g = (i.p - j.p) + (pcogi - pcogj) - gg;
  Mob<S> mi = phase_mobilities_g(s, i.sw, pi.sg, i.p, pi.rs), mj = phase_mobilities_g(s, j.sw, pj.sg, j.p, pj.rs);
  S mob_w, p_w, mob_o, bo_o, rs_o, mob_g, bg_g;
  if (val(dphi_w) >= 0.0) {
    mob_w = mi.w;
    p_w = i.p;
  } else {
    mob_w = mj.w;
    p_w = j.p;
  }
  if (val(dphi_o) >= 0.0) {
    mob_o = mi.o;
    bo_o = pi.bo;
    rs_o = pi.rs;
  } else {
    mob_o = mj.o;
    bo_o = pj.bo;
    rs_o = pj.rs;
  }
  if (val(dphi_g) >= 0.0) {
    mob_g = mi.g;
    bg_g = pi.bg;
  } else {
    mob_g = mj.g;
    bg_g = pj.bg;
  }
  S qw = mob_w * dphi_w * geom_t * water_inverse_fvf_g(s, p_w);
  S qo_res = mob_o * dphi_o * geom_t;
  S qo = qo_res / max_floor(bo_o, 1e-9);
  S qg_free = mob_g * dphi_g * geom_t / max_floor(bg_g, 1e-9);
  S qg_dis = qo * rs_o;
  flux[0] = qw;
  flux[1] = qo;
  flux[2] = qg_free + qg_dis;
}

// ---- wells ----
// fim/wells.rs:800-832
inline bool geometric_well_index(const Sim& s, const RfWell& w, int id, double& out) {
  const double kx = s.kx[id], ky = s.ky[id];
  if (!std::isfinite(kx) || !std::isfinite(ky) || kx <= 0.0 || ky <= 0.0) return false;
  const double r_eq = 0.28 * std::sqrt(std::sqrt(kx / ky) * s.dx * s.dx + std::sqrt(ky / kx) * s.dy * s.dy) /
                      (std::pow(kx / ky, 0.25) + std::pow(ky / kx, 0.25));
  if (!std::isfinite(r_eq) || r_eq <= w.well_radius) return false;
  const double k_avg = std::sqrt(kx * ky);
  const double denom = std::log(r_eq / w.well_radius) + w.skin;
  if (!std::isfinite(k_avg) || k_avg <= 0.0 || !std::isfinite(denom) || std::fabs(denom) <= F64_EPS)
    return false;
  out = DARCY_METRIC_FACTOR * 2.0 * M_PI * k_avg * s.dz_at(id) / denom;
  return true;
}

// fim/wells.rs:544-594
inline Topo build_well_topology(const Sim& s) {
  Topo t;
  std::map<std::tuple<int, int, int, int, uint64_t, uint64_t, uint64_t>, int> groups;
  for (int e = 0; e < int(s.wells.size()); ++e) {
    const RfWell& w = s.wells[e];
    std::tuple<int, int, int, int, uint64_t, uint64_t, uint64_t> key;
    if (w.physical_well_id >= 0) {
      key = std::make_tuple(0, w.physical_well_id, 0, 0, 0, 0, 0);
    } else {
      uint64_t b, r, k;
      std::memcpy(&b, &w.bhp, 8);
      std::memcpy(&r, &w.well_radius, 8);
      std::memcpy(&k, &w.skin, 8);
      key = std::make_tuple(1, w.injector, w.i, w.j, b, r, k);
    }
    auto it = groups.find(key);
    int pw;
    if (it == groups.end()) {
      pw = int(t.wells.size());
      groups[key] = pw;
      t.wells.push_back(PWell{e, w.injector != 0, {}});
    } else {
      pw = it->second;
    }
    Perf p;
    p.entry = e;
    p.well = pw;
    p.cell = s.idx(w.i, w.j, w.k);
    p.i = w.i;
    p.j = w.j;
    p.k = w.k;
    p.injector = w.injector != 0;
    p.has_wi = geometric_well_index(s, w, p.cell, p.wi);
    t.wells[pw].perfs.push_back(int(t.perfs.size()));
    t.perfs.push_back(p);
  }
  return t;
}

// fim/wells.rs:691-798
inline Control physical_well_control(const Sim& s, int w) {
  const RfWell& rep = s.wells[s.topo.wells[w].rep_entry];
  const bool injector = s.topo.wells[w].injector;
  const bool explicit_schedule =
      rep.has_schedule && (rep.schedule_control != 0 || !std::isnan(rep.schedule_target_rate) ||
                           !std::isnan(rep.schedule_target_surface_rate) ||
                           !std::isnan(rep.schedule_bhp_limit) || !rep.schedule_enabled);
  Control c;
  c.enabled = explicit_schedule ? rep.schedule_enabled != 0 : (injector ? s.inj_enabled : true);
  const bool fam_rate = injector ? (s.inj_rate_ctl && s.inj_enabled) : s.prod_rate_ctl;
  if (!c.enabled)
    c.rate_controlled = false;
  else if (explicit_schedule)
    c.rate_controlled = rep.schedule_control == 2;
  else
    c.rate_controlled = fam_rate;
  c.uses_surface_target = explicit_schedule ? !std::isnan(rep.schedule_target_surface_rate)
                                            : !std::isnan(injector ? s.tgt_inj_surf : s.tgt_prod_surf);
  c.has_target = false;
  c.target_rate = 0.0;
  if (c.rate_controlled) {
    if (explicit_schedule) {
      double t = !std::isnan(rep.schedule_target_surface_rate)
                     ? rep.schedule_target_surface_rate
                     : (!std::isnan(rep.schedule_target_rate) ? rep.schedule_target_rate : 0.0);
      c.has_target = true;
      c.target_rate = rmax(t, 0.0);
    } else if (fam_rate) {
      double t = injector ? (!std::isnan(s.tgt_inj_surf) ? s.tgt_inj_surf : s.tgt_inj)
                          : (!std::isnan(s.tgt_prod_surf) ? s.tgt_prod_surf : s.tgt_prod);
      c.has_target = true;
      c.target_rate = rmax(t, 0.0);
    }
  }
  const double fam_limit = injector ? s.bhp_max : s.bhp_min;
  c.bhp_limit = explicit_schedule ? (!std::isnan(rep.schedule_bhp_limit) ? rep.schedule_bhp_limit : fam_limit)
                                  : fam_limit;
  c.bhp_target = rep.bhp;
  return c;
}

// resolve_cell_flash (flash.rs:43-160), gas redissolution enabled
struct Flash {
  int regime;
  double so, sg, rs;
};
inline Flash resolve_cell_flash(const Sim& s, double p, double sw, double hc, int regime, double base_rs = NAN) {
  const double raw_total = 1.0 - sw;
  const double bounded_total = rmax(raw_total, 0.0);
  if (!s.three_phase || !s.has_pvt) return Flash{regime, bounded_total, 0.0, 0.0};
  if (regime == 0) {
    const double sg = hc;
    double rs = pvt_interpolate(s.pvt, p).rs;
    if (!std::isnan(base_rs)) rs = rmin(rs, base_rs);
    return Flash{regime, raw_total - sg, sg, rs};
  }
  double rs_cap = rmax(pvt_interpolate(s.pvt, p).rs, 0.0);
  if (!std::isnan(base_rs)) rs_cap = rmin(rs_cap, rmax(base_rs, 0.0));
  const double rs_trial = hc;
  if (rs_trial <= rs_cap + 1e-6) return Flash{regime, raw_total, 0.0, rs_trial};
  const double bo_trial = rmax(get_b_o_for_rs(s, p, rs_trial), 1e-9);
  const double dissolved = raw_total * rs_trial / bo_trial;
  Flash f;
  split_gas_plain(s, p, 1.0, sw, 0.0, dissolved, base_rs, f.sg, f.so, f.rs);
  f.regime = f.sg > 1e-12 ? 0 : 1;
  return f;
}

// derive_cell (state.rs:823-854)
struct Derived {
  double so, sg, rs, bo, bg;
};
inline Derived derive_cell(const Sim& s, const Cell& c) {
  const Flash f = resolve_cell_flash(s, c.p, c.sw, c.hc, c.regime, c.base_rs);
  Derived d;
  d.so = f.so;
  d.sg = f.sg;
  d.rs = f.rs;
  if (s.has_pvt) {
    double mu;
    pvt_interpolate_oil(s.pvt, c.p, f.rs, d.bo, mu);
    d.bg = pvt_interpolate(s.pvt, c.p).bg;
  } else {
    d.bo = base_oil_fvf(s, c.p);
    d.bg = 1.0;
  }
  return d;
}

// effective_injected_fluid (fim/wells.rs:618-624): 1 when the injectors inject gas
inline int injected_fluid(const Sim& s) { return s.three_phase ? s.injected_fluid : 0; }

// fim/wells.rs:1098-1129
inline bool connection_rate_for_bhp(const Sim& s, const State& st, int perf, double bhp, double& q) {
  const Perf& pf = s.topo.perfs[perf];
  const Cell& c = st.cells[pf.cell];
  const Derived d = derive_cell(s, c);
  Mob<double> m = phase_mobilities_f64(s, c.sw, d.sg, c.p, d.rs);
  if (!pf.has_wi) return false;
  const double mob = rmax(m.w + m.o + m.g, 0.0);
  const double raw = pf.wi * mob * (c.p - (bhp + s.head_offset[pf.entry]));
  if (!std::isfinite(raw)) return false;
  q = pf.injector ? rmin(raw, 0.0) : rmax(raw, 0.0);
  return true;
}

// producer_control_state (fim/wells.rs:834-859)
struct ProducerState {
  double wf, of, gf, bo, bg, rs;
};
inline ProducerState producer_control_state(const Sim& s, const Cell& c) {
  const Derived d = derive_cell(s, c);
  Mob<double> m = phase_mobilities_f64(s, c.sw, d.sg, c.p, d.rs);
  const double lw = rmax(m.w, 0.0), lo = rmax(m.o, 0.0), lg = rmax(m.g, 0.0);
  const double lt = rmax(lw + lo + lg, F64_EPS);
  ProducerState p;
  p.wf = rclamp(lw / lt, 0.0, 1.0);
  p.of = rclamp(lo / lt, 0.0, 1.0);
  p.gf = rclamp(lg / lt, 0.0, 1.0);
  p.bo = rmax(d.bo, 1e-9);
  p.bg = rmax(d.bg, 1e-9);
  p.rs = rmax(d.rs, 0.0);
  return p;
}

// fim/wells.rs:1147-1170
inline double perforation_surface_rate_sc_day(const Sim& s, const State& st, int perf, double q) {
  const Perf& pf = s.topo.perfs[perf];
  const Cell& c = st.cells[pf.cell];
  if (pf.injector) {
    if (injected_fluid(s) == 1) return rmax(-q, 0.0) / rmax(derive_cell(s, c).bg, 1e-9);
    return rmax(-q, 0.0) * water_inverse_fvf_g(s, c.p);
  }
  ProducerState ps = producer_control_state(s, c);
  return rmax(q, 0.0) * ps.of / rmax(ps.bo, 1e-9);
}

// fim/wells.rs:389-408
inline double total_rate_for_bhp(const Sim& s, const State& st, int w, double bhp) {
  const Control c = physical_well_control(s, w);
  const bool inj = s.topo.wells[w].injector;
  double total = 0.0;
  for (int perf : s.topo.wells[w].perfs) {
    double q;
    if (!connection_rate_for_bhp(s, st, perf, bhp, q)) continue;
    if (c.uses_surface_target)
      total += perforation_surface_rate_sc_day(s, st, perf, q);
    else
      total += inj ? rmax(-q, 0.0) : rmax(q, 0.0);
  }
  return total;
}

// fim/wells.rs:431-504
inline bool solve_bhp_from_target(const Sim& s, const State& st, int w, double& bhp_out) {
  const Control c = physical_well_control(s, w);
  if (!c.enabled || !c.rate_controlled) return false;
  const auto& perfs = s.topo.wells[w].perfs;
  if (perfs.empty() || !c.has_target) return false;
  double minp = INFINITY, maxp = -INFINITY;
  for (int perf : perfs) {
    const Perf& pf = s.topo.perfs[perf];
    const double z = st.cells[pf.cell].p - s.head_offset[pf.entry];
    minp = rmin(minp, z);
    maxp = rmax(maxp, z);
  }
  if (!std::isfinite(minp) || !std::isfinite(maxp)) return false;
  const double target = c.target_rate;
  const double limit = c.bhp_limit;
  const double max_rate = total_rate_for_bhp(s, st, w, limit);
  if (target >= max_rate - 1e-9) {
    bhp_out = limit;
    return true;
  }
  if (s.topo.wells[w].injector) {
    double lo = rmin(minp, limit), hi = limit;
    for (int it = 0; it < 64; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (total_rate_for_bhp(s, st, w, mid) < target)
        lo = mid;
      else
        hi = mid;
    }
    bhp_out = 0.5 * (lo + hi);
  } else {
    double lo = limit, hi = rmax(maxp, limit);
    for (int it = 0; it < 64; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (total_rate_for_bhp(s, st, w, mid) > target)
        lo = mid;
      else
        hi = mid;
    }
    bhp_out = 0.5 * (lo + hi);
  }
  return true;
}

// ---- AD well model (fim/wells_ad.rs) ----
template <class S>
struct WellCell {
  S p, sw, hc;
  int regime;
  double base_rs = NAN;  // DRSDT0 cap
};
template <class S>
struct Fractions {
  S wf, of, gf;
};
// producer_fractions_generic (wells_ad.rs:44-72) over the one-cell neighbourhood
template <class S>
inline Fractions<S> producer_fractions_g(const Sim& s, const WellCell<S>& c) {
  S lw = sc<S>(0.0), lo = sc<S>(0.0), lg = sc<S>(0.0);
  Props<S> pr = cell_props_g(s, c.regime, c.p, c.sw, c.hc, c.base_rs);
  Mob<S> m = phase_mobilities_g(s, c.sw, pr.sg, c.p, pr.rs);
  lw = lw + max_floor(m.w, 0.0);
  lo = lo + max_floor(m.o, 0.0);
  lg = lg + max_floor(m.g, 0.0);
  S lt = max_floor(lw + lo + lg, F64_EPS);
  Fractions<S> f;
  f.wf = min_ceil(max_floor(lw / lt, 0.0), 1.0);
  f.of = min_ceil(max_floor(lo / lt, 0.0), 1.0);
  f.gf = min_ceil(max_floor(lg / lt, 0.0), 1.0);
  return f;
}
// connection_rate_generic (wells_ad.rs:119-159)
template <class S>
inline S connection_rate_g(const Sim& s, double wi, double head, bool injector, const WellCell<S>& c,
                           const S& bhp) {
  Props<S> pr = cell_props_g(s, c.regime, c.p, c.sw, c.hc, c.base_rs);
  Mob<S> m = phase_mobilities_g(s, c.sw, pr.sg, c.p, pr.rs);
  S cm = max_floor(m.w + m.o + m.g, 0.0);
  S raw = (cm * (c.p - bhp - sc<S>(head))) * wi;
  if (injector) return val(raw) < 0.0 ? raw : sc<S>(0.0);
  return val(raw) > 0.0 ? raw : sc<S>(0.0);
}
// component_rate_coefficients_generic (wells_ad.rs:161-201)
template <class S>
inline void component_coefficients_g(const Sim& s, bool injector, const WellCell<S>& c,
                                     const Fractions<S>* f, S out[3]) {
  Props<S> pr = cell_props_g(s, c.regime, c.p, c.sw, c.hc, c.base_rs);
  if (injector) {
    if (injected_fluid(s) == 1) {
      out[0] = sc<S>(0.0);
      out[1] = sc<S>(0.0);
      out[2] = s_recip(max_floor(pr.bg, 1e-9));
      return;
    }
    out[0] = water_inverse_fvf_g(s, c.p);
    out[1] = sc<S>(0.0);
    out[2] = sc<S>(0.0);
    return;
  }
  S bo = max_floor(pr.bo, 1e-9), bg = max_floor(pr.bg, 1e-9);
  S oc = f->of / bo;
  out[0] = f->wf * water_inverse_fvf_g(s, c.p);
  out[1] = oc;
  out[2] = f->gf / bg + oc * pr.rs;
}
// perforation_surface_rate_generic (wells_ad.rs:203-229)
template <class S>
inline S perforation_surface_rate_g(const Sim& s, bool injector, const WellCell<S>& c,
                                    const Fractions<S>* f, const S& q) {
  Props<S> pr = cell_props_g(s, c.regime, c.p, c.sw, c.hc, c.base_rs);
  if (injector) {
    S clamped = max_floor(-q, 0.0);
    if (injected_fluid(s) == 1) return clamped / max_floor(pr.bg, 1e-9);
    return clamped * water_inverse_fvf_g(s, c.p);
  }
  return max_floor(q, 0.0) * f->of / max_floor(pr.bo, 1e-9);
}
template <class S>
inline S perforation_reservoir_rate_g(bool injector, const S& q) {
  return injector ? max_floor(-q, 0.0) : max_floor(q, 0.0);
}
template <class S>
inline S fischer_burmeister_g(const S& a, const S& b) {
  const double e = 2.0 * FB_EPSILON * FB_EPSILON;
  S norm = s_sqrt((a * a + b * b) + e);
  return norm - a - b;
}
inline void fischer_burmeister_gradient(double a, double b, double& da, double& db) {
  const double norm = std::sqrt(a * a + b * b + 2.0 * FB_EPSILON * FB_EPSILON);
  da = a / norm - 1.0;
  db = b / norm - 1.0;
}

}  // namespace orc
