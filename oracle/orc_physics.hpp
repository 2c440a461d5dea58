// ORACLE — test infrastructure only (see orc_core.hpp).  Two-phase oil-water physics of the
// reference FIM path: PVT, Corey relperm (tabulated), capillary pressure, cell properties,
// accumulation, face flux and the AD well model.
#pragma once

#include <map>
#include <string>
#include <tuple>

#include "../include/ressim_fim.h"
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
  double rho_g = 10.0;  // default gas density; the gas phase carries no flow in two-phase mode
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
  double cum_inj = 0, cum_prod = 0, cum_mb = 0, cum_mb_oil = 0;
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
template <class S>
inline S oil_density_g(const Sim& s, const S& p) {
  S bo = max_floor(sc<S>(s.b_o) * s_exp(p * (-s.c_o)), 1e-9);
  return sc<S>(s.rho_o) / bo;
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

// ---- mobility (mobility.rs:196-249 generic; 114-149 f64) ----
template <class S>
struct Mob {
  S w, o, g;
};
template <class S>
inline Mob<S> phase_mobilities_g(const Sim& s, const S& sw) {
  S krw, kro;
  two_phase_relperm_g(s, sw, krw, kro);
  Mob<S> m;
  m.w = krw / sc<S>(s.mu_w);
  m.o = kro / sc<S>(s.mu_o);
  m.g = sc<S>(0.0);
  return m;
}
inline Mob<double> phase_mobilities_f64(const Sim& s, double sw) {
  double krw, kro;
  two_phase_relperm_g(s, sw, krw, kro);
  return Mob<double>{krw / s.mu_w, kro / s.mu_o, 0.0};
}

// ---- cell properties (properties.rs:37-73, two-phase branch) ----
template <class S>
struct Props {
  S so, sg, rs, bo, bg;
};
template <class S>
inline Props<S> cell_props_g(const Sim& s, const S& p, const S& sw, const S& hc) {
  const S one = sc<S>(1.0);
  const S raw_total = one - sw;
  const S total = max_floor(raw_total, 0.0);
  Props<S> pr;
  pr.sg = min_of(max_floor(hc, 0.0), total);
  pr.so = max_floor(one - sw - pr.sg, 0.0);
  pr.bo = base_oil_fvf_g(s, p);
  pr.rs = sc<S>(0.0);
  pr.bg = sc<S>(1.0);
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

// properties.rs:171-212
template <class S>
inline void cell_accumulation_g(const Sim& s, int cell, const S& p, const S& sw, const S& hc,
                                double pp, double psw, double phc, S out[3]) {
  Props<S> pr = cell_props_g(s, p, sw, hc);
  S pv = pore_volume_g(s, cell, p);
  S cur[3];
  component_inventory_g(s, pv, p, sw, pr, cur);
  Props<double> ppr = cell_props_g<double>(s, pp, psw, phc);
  double ppv = pore_volume_g<double>(s, cell, pp);
  double prev[3];
  component_inventory_g<double>(s, ppv, pp, psw, ppr, prev);
  for (int c = 0; c < 3; ++c) out[c] = cur[c] - prev[c];
}

// ---- face flux (flux.rs:42-118) ----
template <class S>
struct FaceIn {
  S p, sw, hc;
  double depth;
};
template <class S>
inline S gravity_head_g(const Sim& s, double di, double dj, const S& ri, const S& rj) {
  if (!s.gravity) return sc<S>(0.0);
  S avg = (ri + rj) * 0.5;
  return avg * (GRAVITY * (di - dj) * 1e-5);
}
template <class S>
inline void face_flux_g(const Sim& s, double geom_t, const FaceIn<S>& i, const FaceIn<S>& j,
                        S flux[3]) {
  Props<S> pi = cell_props_g(s, i.p, i.sw, i.hc);
  Props<S> pj = cell_props_g(s, j.p, j.sw, j.hc);
  S rwi = water_density_g(s, i.p), rwj = water_density_g(s, j.p);
  S roi = oil_density_g(s, i.p), roj = oil_density_g(s, j.p);
  S rgi = sc<S>(s.rho_g), rgj = sc<S>(s.rho_g);
  S pcwi = capillary_pressure_g(s, i.sw), pcwj = capillary_pressure_g(s, j.sw);
  S pcogi = sc<S>(0.0), pcogj = sc<S>(0.0);
  S gw = gravity_head_g(s, i.depth, j.depth, rwi, rwj);
  S go = gravity_head_g(s, i.depth, j.depth, roi, roj);
  S gg = gravity_head_g(s, i.depth, j.depth, rgi, rgj);
  S dphi_w = (i.p - j.p) - (pcwi - pcwj) - gw;
  S dphi_o = (i.p - j.p) - go;
  S dphi_g = (i.p - j.p) + (pcogi - pcogj) - gg;
  Mob<S> mi = phase_mobilities_g(s, i.sw), mj = phase_mobilities_g(s, j.sw);
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

// derive_cell two-phase (state.rs:823-854, flash.rs:43-72)
struct Derived {
  double so, sg, rs, bo;
};
inline Derived derive_cell(const Sim& s, const Cell& c) {
  Derived d;
  d.so = rmax(1.0 - c.sw, 0.0);
  d.sg = 0.0;
  d.rs = 0.0;
  d.bo = base_oil_fvf(s, c.p);
  return d;
}

// fim/wells.rs:1098-1129
inline bool connection_rate_for_bhp(const Sim& s, const State& st, int perf, double bhp, double& q) {
  const Perf& pf = s.topo.perfs[perf];
  const RfWell& w = s.wells[pf.entry];
  const Cell& c = st.cells[pf.cell];
  Mob<double> m = phase_mobilities_f64(s, c.sw);
  if (!pf.has_wi) return false;
  const double mob = rmax(m.w + m.o + m.g, 0.0);
  const double raw = pf.wi * mob * (c.p - (bhp + s.head_offset[pf.entry]));
  (void)w;
  if (!std::isfinite(raw)) return false;
  q = pf.injector ? rmin(raw, 0.0) : rmax(raw, 0.0);
  return true;
}

// producer_control_state (fim/wells.rs:834-859), two-phase
struct ProducerState {
  double wf, of, gf, bo;
};
inline ProducerState producer_control_state(const Sim& s, const Cell& c) {
  Mob<double> m = phase_mobilities_f64(s, c.sw);
  const double lw = rmax(m.w, 0.0), lo = rmax(m.o, 0.0), lg = rmax(m.g, 0.0);
  const double lt = rmax(lw + lo + lg, F64_EPS);
  ProducerState p;
  p.wf = rclamp(lw / lt, 0.0, 1.0);
  p.of = rclamp(lo / lt, 0.0, 1.0);
  p.gf = rclamp(lg / lt, 0.0, 1.0);
  p.bo = rmax(base_oil_fvf(s, c.p), 1e-9);
  return p;
}

// fim/wells.rs:1147-1170 (injected fluid is water in two-phase mode)
inline double perforation_surface_rate_sc_day(const Sim& s, const State& st, int perf, double q) {
  const Perf& pf = s.topo.perfs[perf];
  const Cell& c = st.cells[pf.cell];
  if (pf.injector) return rmax(-q, 0.0) * water_inverse_fvf_g(s, c.p);
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
};
template <class S>
struct Fractions {
  S wf, of, gf;
};
// producer_fractions_generic (wells_ad.rs:44-72) over the one-cell neighbourhood
template <class S>
inline Fractions<S> producer_fractions_g(const Sim& s, const WellCell<S>& c) {
  S lw = sc<S>(0.0), lo = sc<S>(0.0), lg = sc<S>(0.0);
  Mob<S> m = phase_mobilities_g(s, c.sw);
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
  Mob<S> m = phase_mobilities_g(s, c.sw);
  S cm = max_floor(m.w + m.o + m.g, 0.0);
  S raw = (cm * (c.p - bhp - sc<S>(head))) * wi;
  if (injector) return val(raw) < 0.0 ? raw : sc<S>(0.0);
  return val(raw) > 0.0 ? raw : sc<S>(0.0);
}
// component_rate_coefficients_generic (wells_ad.rs:161-201), water injection
template <class S>
inline void component_coefficients_g(const Sim& s, bool injector, const WellCell<S>& c,
                                     const Fractions<S>* f, S out[3]) {
  Props<S> pr = cell_props_g(s, c.p, c.sw, c.hc);
  if (injector) {
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
  Props<S> pr = cell_props_g(s, c.p, c.sw, c.hc);
  if (injector) return max_floor(-q, 0.0) * water_inverse_fvf_g(s, c.p);
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
