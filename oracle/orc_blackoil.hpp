// ORACLE — test infrastructure only (see orc_core.hpp).  The three-phase black-oil pieces of the
// reference FIM path, each in the operation order of the reference function it cites:
//   pvt.rs:46-500                 PVTO/PVDG-style table (saturated curve, undersaturated oil
//                                 branches), plain and generic interpolation, bubble point
//   relperm.rs:199-458            three-phase Corey relative permeability with Stone II
//   capillary.rs:100-172          gas-oil capillary pressure (Brooks-Corey, capped at 20x entry)
//   step.rs:65-200                Rs bisection and the gas-inventory split of a cell
//   fim/flash_ad.rs:25-207        the same split, differentiated through the implicit function
// Where the reference keeps a plain f64 routine beside its generic mirror (their roundings
// differ), both are restated.
#pragma once

#include <algorithm>
#include <vector>

#include "orc_core.hpp"

namespace orc {

constexpr double PVTO_RS_TOLERANCE = 1e-6;  // pvt.rs:17

struct PvtRow {
  double p, rs, bo, mu_o, bg, mu_g;
};
struct OilBranch {
  double rs;
  std::vector<PvtRow> rows;
};
struct PvtTable {
  std::vector<PvtRow> rows, saturated;
  std::vector<OilBranch> branches;
  double c_o = 0.0;
};

// PvtTable::new + build_oil_branches (pvt.rs:86-135); the sorts are stable, as Rust's sort_by
inline PvtTable make_pvt_table(const std::vector<PvtRow>& rows, double c_o) {
  PvtTable t;
  t.rows = rows;
  t.c_o = c_o;
  std::vector<OilBranch> br;
  for (const PvtRow& r : rows) {
    if (!br.empty()) {
      OilBranch& b = br.back();
      const bool same_rs = std::fabs(r.rs - b.rs) <= PVTO_RS_TOLERANCE;
      const bool higher = b.rows.empty() ? true : r.p >= b.rows.back().p - 1e-9;
      if (same_rs && higher) {
        b.rows.push_back(r);
        continue;
      }
    }
    br.push_back(OilBranch{r.rs, {r}});
  }
  for (OilBranch& b : br)
    std::stable_sort(b.rows.begin(), b.rows.end(), [](const PvtRow& a, const PvtRow& c) { return a.p < c.p; });
  std::stable_sort(br.begin(), br.end(), [](const OilBranch& a, const OilBranch& c) { return a.rs < c.rs; });
  for (const OilBranch& b : br)
    if (!b.rows.empty()) t.saturated.push_back(b.rows.front());
  std::stable_sort(t.saturated.begin(), t.saturated.end(),
                   [](const PvtRow& a, const PvtRow& c) { return a.p < c.p; });
  t.branches = br;
  return t;
}

// ---- plain interpolation ----
// interpolate_oil_segment / interpolate_gas_segment (pvt.rs:64-77): linear in 1/B and 1/(B mu)
inline void oil_segment(const PvtRow& r0, const PvtRow& r1, double t, double& bo, double& mu) {
  const double inv_bo = (1.0 / r0.bo) + t * (1.0 / r1.bo - 1.0 / r0.bo);
  const double inv_bo_mu = (1.0 / (r0.bo * r0.mu_o)) + t * (1.0 / (r1.bo * r1.mu_o) - 1.0 / (r0.bo * r0.mu_o));
  bo = 1.0 / inv_bo;
  mu = inv_bo / inv_bo_mu;
}
inline void gas_segment(const PvtRow& r0, const PvtRow& r1, double t, double& bg, double& mu) {
  const double inv_bg = (1.0 / r0.bg) + t * (1.0 / r1.bg - 1.0 / r0.bg);
  const double inv_bg_mu = (1.0 / (r0.bg * r0.mu_g)) + t * (1.0 / (r1.bg * r1.mu_g) - 1.0 / (r0.bg * r0.mu_g));
  bg = 1.0 / inv_bg;
  mu = inv_bg / inv_bg_mu;
}

// interpolate_rows over the saturated curve (pvt.rs:137-186, 250-252)
inline PvtRow pvt_interpolate(const PvtTable& t, double p) {
  const std::vector<PvtRow>& rows = t.saturated;
  if (rows.empty()) return PvtRow{p, 0.0, 1.0, 1.0, 1.0, 0.02};
  if (p <= rows[0].p) return rows[0];
  const size_t last = rows.size() - 1;
  if (p >= rows[last].p) {
    const PvtRow& l = rows[last];
    PvtRow e = l;
    e.p = p;
    e.bo = l.bo * std::exp(-t.c_o * (p - l.p));
    e.bg = l.bg * (l.p / p);
    return e;
  }
  for (size_t i = 0; i < last; ++i) {
    const PvtRow& r0 = rows[i];
    const PvtRow& r1 = rows[i + 1];
    if (p >= r0.p && p <= r1.p) {
      const double dp = r1.p - r0.p;
      if (dp < 1e-6) return r0;
      const double tt = (p - r0.p) / dp;
      PvtRow r;
      r.p = p;
      r.rs = r0.rs + tt * (r1.rs - r0.rs);
      oil_segment(r0, r1, tt, r.bo, r.mu_o);
      gas_segment(r0, r1, tt, r.bg, r.mu_g);
      return r;
    }
  }
  return rows[last];
}

// branch_props (pvt.rs:188-225)
inline void branch_props(const OilBranch& b, double p, double c_o, double& bo, double& mu) {
  const std::vector<PvtRow>& rows = b.rows;
  if (rows.empty()) {
    bo = 1.0;
    mu = 1.0;
    return;
  }
  if (rows.size() == 1) {
    bo = rows[0].bo * std::exp(-c_o * (p - rows[0].p));
    mu = rows[0].mu_o * std::exp(c_o * (p - rows[0].p));
    return;
  }
  if (p <= rows[0].p) {
    bo = rows[0].bo;
    mu = rows[0].mu_o;
    return;
  }
  for (size_t i = 0; i + 1 < rows.size(); ++i) {
    const PvtRow& r0 = rows[i];
    const PvtRow& r1 = rows[i + 1];
    if (p >= r0.p && p <= r1.p) {
      const double dp = r1.p - r0.p;
      if (std::fabs(dp) < 1e-9) {
        bo = r0.bo;
        mu = r0.mu_o;
        return;
      }
      oil_segment(r0, r1, (p - r0.p) / dp, bo, mu);
      return;
    }
  }
  const PvtRow& l = rows.back();
  const double excess = p - l.p;
  bo = rmax(l.bo * std::exp(-c_o * excess), 1e-9);
  mu = l.mu_o * std::exp(c_o * excess);
}

// branch_bounds (pvt.rs:227-248): indices of the lower and upper branch
inline bool branch_bounds(const PvtTable& t, double rs, int& lo, int& hi) {
  if (t.branches.empty()) return false;
  const int last = int(t.branches.size()) - 1;
  if (rs <= t.branches[0].rs + PVTO_RS_TOLERANCE) {
    lo = hi = 0;
    return true;
  }
  if (rs >= t.branches[last].rs - PVTO_RS_TOLERANCE) {
    lo = hi = last;
    return true;
  }
  for (int i = 0; i < last; ++i)
    if (rs >= t.branches[i].rs - PVTO_RS_TOLERANCE && rs <= t.branches[i + 1].rs + PVTO_RS_TOLERANCE) {
      lo = i;
      hi = i + 1;
      return true;
    }
  lo = hi = last;
  return true;
}

// interpolate_oil (pvt.rs:458-488): undersaturation-aware Bo and mu_o
inline void pvt_interpolate_oil(const PvtTable& t, double p, double rs, double& bo, double& mu) {
  if (t.saturated.empty()) {
    bo = 1.0;
    mu = 1.0;
    return;
  }
  const PvtRow sat = pvt_interpolate(t, p);
  if (rs >= sat.rs - 1e-6) {
    bo = sat.bo;
    mu = sat.mu_o;
    return;
  }
  int lo, hi;
  if (branch_bounds(t, rs, lo, hi)) {
    const OilBranch& low = t.branches[lo];
    const OilBranch& high = t.branches[hi];
    double bo_low, mu_low;
    branch_props(low, p, t.c_o, bo_low, mu_low);
    if (std::fabs(high.rs - low.rs) <= PVTO_RS_TOLERANCE) {
      bo = bo_low;
      mu = mu_low;
      return;
    }
    const double tt = (rs - low.rs) / (high.rs - low.rs);
    const double shift = high.rows[0].p - low.rows[0].p;
    const double p_low = p - tt * shift;
    const double p_high = p + (1.0 - tt) * shift;
    double bo_high, mu_high;
    branch_props(low, p_low, t.c_o, bo_low, mu_low);
    branch_props(high, p_high, t.c_o, bo_high, mu_high);
    const double inv_bo = 1.0 / bo_low + tt * (1.0 / bo_high - 1.0 / bo_low);
    const double inv_bo_mu = 1.0 / (bo_low * mu_low) + tt * (1.0 / (bo_high * mu_high) - 1.0 / (bo_low * mu_low));
    bo = 1.0 / inv_bo;
    mu = inv_bo / inv_bo_mu;
    return;
  }
  bo = sat.bo;
  mu = sat.mu_o;
}

// bubble_point_pressure (pvt.rs:427-456)
inline double pvt_bubble_point(const PvtTable& t, double rs) {
  if (t.saturated.empty()) return 0.0;
  if (rs <= t.branches[0].rs) return t.branches[0].rows[0].p;
  const size_t last = t.branches.size() - 1;
  if (rs >= t.branches[last].rs) return t.branches[last].rows[0].p;
  for (size_t i = 0; i < last; ++i) {
    const OilBranch& r0 = t.branches[i];
    const OilBranch& r1 = t.branches[i + 1];
    if (rs >= r0.rs && rs <= r1.rs) {
      const double drs = r1.rs - r0.rs;
      if (drs < 1e-12) return r0.rows[0].p;
      const double tt = (rs - r0.rs) / drs;
      return r0.rows[0].p + tt * (r1.rows[0].p - r0.rows[0].p);
    }
  }
  return t.branches[last].rows[0].p;
}

// ---- generic interpolation ----
template <class S>
struct SatProps {
  S rs, bo, bg, mu_o, mu_g;
};

// interpolate_oil_segment_generic (pvt.rs:79-84)
template <class S>
inline void oil_segment_g(const PvtRow& r0, const PvtRow& r1, const S& t, S& bo, S& mu) {
  S inv_bo = t * (1.0 / r1.bo - 1.0 / r0.bo) + 1.0 / r0.bo;
  S inv_bo_mu = t * (1.0 / (r1.bo * r1.mu_o) - 1.0 / (r0.bo * r0.mu_o)) + 1.0 / (r0.bo * r0.mu_o);
  bo = s_recip(inv_bo);
  mu = inv_bo / inv_bo_mu;
}

// interpolate_saturated_generic (pvt.rs:259-342): the segment is chosen on the value of p
template <class S>
inline SatProps<S> pvt_saturated_g(const PvtTable& t, const S& p) {
  const std::vector<PvtRow>& rows = t.saturated;
  SatProps<S> o;
  if (rows.empty()) {
    o.rs = sc<S>(0.0);
    o.bo = sc<S>(1.0);
    o.bg = sc<S>(1.0);
    o.mu_o = sc<S>(1.0);
    o.mu_g = sc<S>(0.02);
    return o;
  }
  const double pv = val(p);
  auto constant_row = [&](const PvtRow& r) {
    o.rs = sc<S>(r.rs);
    o.bo = sc<S>(r.bo);
    o.bg = sc<S>(r.bg);
    o.mu_o = sc<S>(r.mu_o);
    o.mu_g = sc<S>(r.mu_g);
    return o;
  };
  if (pv <= rows[0].p) return constant_row(rows[0]);
  const size_t last = rows.size() - 1;
  if (pv >= rows[last].p) {
    const PvtRow& r = rows[last];
    o.bo = sc<S>(r.bo) * s_exp((p * (-t.c_o)) + (t.c_o * r.p));
    o.bg = sc<S>(r.bg * r.p) / p;
    o.rs = sc<S>(r.rs);
    o.mu_o = sc<S>(r.mu_o);
    o.mu_g = sc<S>(r.mu_g);
    return o;
  }
  for (size_t i = 0; i < last; ++i) {
    const PvtRow& r0 = rows[i];
    const PvtRow& r1 = rows[i + 1];
    if (pv >= r0.p && pv <= r1.p) {
      const double dp = r1.p - r0.p;
      if (dp < 1e-6) return constant_row(r0);
      S tt = (p - r0.p) / dp;
      auto lerp = [&](double a, double b) { return tt * (b - a) + a; };
      S inv_bg = lerp(1.0 / r0.bg, 1.0 / r1.bg);
      S inv_bg_mu = lerp(1.0 / (r0.bg * r0.mu_g), 1.0 / (r1.bg * r1.mu_g));
      o.rs = lerp(r0.rs, r1.rs);
      S bo, mu;
      oil_segment_g(r0, r1, tt, bo, mu);
      o.bo = bo;
      o.bg = sc<S>(1.0) / inv_bg;
      o.mu_o = mu;
      o.mu_g = inv_bg / inv_bg_mu;
      return o;
    }
  }
  return constant_row(rows[last]);
}

// branch_props_generic (pvt.rs:344-382)
template <class S>
inline void branch_props_g(const OilBranch& b, const S& p, double c_o, S& bo, S& mu) {
  const std::vector<PvtRow>& rows = b.rows;
  if (rows.empty()) {
    bo = sc<S>(1.0);
    mu = sc<S>(1.0);
    return;
  }
  if (rows.size() == 1) {
    S excess = p - rows[0].p;
    bo = sc<S>(rows[0].bo) * s_exp(excess * (-c_o));
    mu = sc<S>(rows[0].mu_o) * s_exp(excess * c_o);
    return;
  }
  const double pv = val(p);
  if (pv <= rows[0].p) {
    bo = sc<S>(rows[0].bo);
    mu = sc<S>(rows[0].mu_o);
    return;
  }
  for (size_t i = 0; i + 1 < rows.size(); ++i) {
    const PvtRow& r0 = rows[i];
    const PvtRow& r1 = rows[i + 1];
    if (pv >= r0.p && pv <= r1.p) {
      const double dp = r1.p - r0.p;
      if (std::fabs(dp) < 1e-9) {
        bo = sc<S>(r0.bo);
        mu = sc<S>(r0.mu_o);
        return;
      }
      S tt = (p - r0.p) / dp;
      oil_segment_g(r0, r1, tt, bo, mu);
      return;
    }
  }
  const PvtRow& l = rows.back();
  S excess = p - l.p;
  bo = max_floor(sc<S>(l.bo) * s_exp(excess * (-c_o)), 1e-9);
  mu = sc<S>(l.mu_o) * s_exp(excess * c_o);
}

// interpolate_oil_generic (pvt.rs:384-425)
template <class S>
inline void pvt_oil_g(const PvtTable& t, const S& p, const S& rs, S& bo, S& mu) {
  if (t.saturated.empty()) {
    bo = sc<S>(1.0);
    mu = sc<S>(1.0);
    return;
  }
  const SatProps<S> sat = pvt_saturated_g(t, p);
  const double rs_sat = val(sat.rs);
  if (val(rs) >= rs_sat - 1e-6) {
    bo = sat.bo;
    mu = sat.mu_o;
    return;
  }
  int lo, hi;
  if (branch_bounds(t, val(rs), lo, hi)) {
    const OilBranch& low = t.branches[lo];
    const OilBranch& high = t.branches[hi];
    S bo_low, mu_low;
    branch_props_g(low, p, t.c_o, bo_low, mu_low);
    if (std::fabs(high.rs - low.rs) <= PVTO_RS_TOLERANCE) {
      bo = bo_low;
      mu = mu_low;
      return;
    }
    S tt = (rs - low.rs) / (high.rs - low.rs);
    const double shift = high.rows[0].p - low.rows[0].p;
    S p_low = p - tt * shift;
    S p_high = p + (sc<S>(1.0) - tt) * shift;
    S bo_high, mu_high;
    branch_props_g(low, p_low, t.c_o, bo_low, mu_low);
    branch_props_g(high, p_high, t.c_o, bo_high, mu_high);
    S inv_bo = tt * (s_recip(bo_high) - s_recip(bo_low)) + s_recip(bo_low);
    S inv_bo_mu = tt * (s_recip(bo_high * mu_high) - s_recip(bo_low * mu_low)) + s_recip(bo_low * mu_low);
    bo = s_recip(inv_bo);
    mu = inv_bo / inv_bo_mu;
    return;
  }
  bo = sat.bo;
  mu = sat.mu_o;
}

// ---- three-phase relative permeability (relperm.rs:199-458): Corey, or the SWOF/SGOF tables ----
struct Scal3 {
  double s_wc, s_or, n_w, n_o, krw_max, kro_max, s_gc, s_gr, s_org, n_g, krg_max;
  // SWOF rows (sw, krw, krow) and SGOF rows (sg, krg, krog); empty: the Corey curves
  std::vector<double> swof, sgof;
};

// interpolate_piecewise (relperm.rs:124-147) on column `y` of rows of three doubles (x first)
inline double table_interp(const std::vector<double>& t, int y, double x) {
  const int n = int(t.size() / 3);
  if (n == 0) return 0.0;
  if (x <= t[0]) return t[y];
  for (int r = 0; r + 1 < n; ++r) {
    const double x0 = t[3 * r], x1 = t[3 * r + 3];
    if (x <= x1) {
      if (std::fabs(x1 - x0) <= 2.220446049250313e-16) return t[3 * r + 3 + y];
      const double f = rclamp((x - x0) / (x1 - x0), 0.0, 1.0);
      return t[3 * r + y] + f * (t[3 * r + 3 + y] - t[3 * r + y]);
    }
  }
  return t[3 * (n - 1) + y];
}
// interpolate_piecewise_generic (relperm.rs:9-40): the segment from the value, the derivative of
// the active segment
template <class S>
inline S table_interp_g(const std::vector<double>& t, int y, const S& x) {
  const int n = int(t.size() / 3);
  if (n == 0) return sc<S>(0.0);
  const double xv = val(x);
  if (xv <= t[0]) return sc<S>(t[y]);
  for (int r = 0; r + 1 < n; ++r) {
    const double x0 = t[3 * r], x1 = t[3 * r + 3];
    if (xv <= x1) {
      if (std::fabs(x1 - x0) <= 2.220446049250313e-16) return sc<S>(t[3 * r + 3 + y]);
      S f = min_ceil(max_floor((x - x0) / (x1 - x0), 0.0), 1.0);
      const double y0 = t[3 * r + y], y1 = t[3 * r + 3 + y];
      return f * (y1 - y0) + y0;
    }
  }
  return sc<S>(t[3 * (n - 1) + y]);
}

inline double k_rw3(const Scal3& s, double sw) {
  if (!s.swof.empty()) return table_interp(s.swof, 1, sw);
  const double e = rclamp((sw - s.s_wc) / (1.0 - s.s_wc - s.s_or), 0.0, 1.0);
  return s.krw_max * std::pow(e, s.n_w);
}
inline double k_rg3(const Scal3& s, double sg) {
  if (!s.sgof.empty()) return table_interp(s.sgof, 1, sg);
  const double denom = 1.0 - s.s_wc - s.s_gc - s.s_gr;
  if (denom <= 0.0) return 0.0;
  const double e = rclamp((sg - s.s_gc) / denom, 0.0, 1.0);
  return s.krg_max * std::pow(e, s.n_g);
}
inline double k_ro_water3(const Scal3& s, double sw) {
  if (!s.swof.empty()) return table_interp(s.swof, 2, sw);
  const double e = rclamp((1.0 - sw - s.s_or) / (1.0 - s.s_wc - s.s_or), 0.0, 1.0);
  return s.kro_max * std::pow(e, s.n_o);
}
inline double k_ro_gas3(const Scal3& s, double sg) {
  if (!s.sgof.empty()) return table_interp(s.sgof, 2, sg);
  const double denom = 1.0 - s.s_wc - s.s_org;
  if (denom <= 0.0) return 0.0;
  const double e = rclamp((1.0 - s.s_wc - sg - s.s_org) / denom, 0.0, 1.0);
  return s.kro_max * std::pow(e, s.n_o);
}
inline double k_ro_stone2(const Scal3& s, double sw, double sg) {
  const double kro_max = s.kro_max;
  const double kro_w = k_ro_water3(s, sw), kro_g = k_ro_gas3(s, sg);
  const double krw = k_rw3(s, sw), krg = k_rg3(s, sg);
  const double v = kro_max * ((kro_w / kro_max + krw) * (kro_g / kro_max + krg) - krw - krg);
  return rclamp(v, 0.0, kro_max);
}

template <class S>
inline S k_rw3_g(const Scal3& s, const S& sw) {
  if (!s.swof.empty()) return table_interp_g(s.swof, 1, sw);
  const double denom = 1.0 - s.s_wc - s.s_or;
  S e = min_ceil(max_floor((sw - s.s_wc) / denom, 0.0), 1.0);
  return s_powf(e, s.n_w) * s.krw_max;
}
template <class S>
inline S k_rg3_g(const Scal3& s, const S& sg) {
  if (!s.sgof.empty()) return table_interp_g(s.sgof, 1, sg);
  const double denom = 1.0 - s.s_wc - s.s_gc - s.s_gr;
  S e = min_ceil(max_floor((sg - s.s_gc) / denom, 0.0), 1.0);
  return s_powf(e, s.n_g) * s.krg_max;
}
template <class S>
inline S k_ro_water3_g(const Scal3& s, const S& sw) {
  if (!s.swof.empty()) return table_interp_g(s.swof, 2, sw);
  const double denom = 1.0 - s.s_wc - s.s_or;
  S e = min_ceil(max_floor((sc<S>(1.0 - s.s_or) - sw) / denom, 0.0), 1.0);
  return s_powf(e, s.n_o) * s.kro_max;
}
template <class S>
inline S k_ro_gas3_g(const Scal3& s, const S& sg) {
  if (!s.sgof.empty()) return table_interp_g(s.sgof, 2, sg);
  const double denom = 1.0 - s.s_wc - s.s_org;
  S e = min_ceil(max_floor((sc<S>(1.0 - s.s_wc - s.s_org) - sg) / denom, 0.0), 1.0);
  return s_powf(e, s.n_o) * s.kro_max;
}
// k_ro_stone2_generic: zero derivative at and beyond either clamp bound (relperm.rs:431-457)
template <class S>
inline S k_ro_stone2_g(const Scal3& s, const S& sw, const S& sg) {
  const double kro_max = s.kro_max;
  S kro_w = k_ro_water3_g(s, sw), kro_g = k_ro_gas3_g(s, sg);
  S krw = k_rw3_g(s, sw), krg = k_rg3_g(s, sg);
  S v = ((kro_w / kro_max + krw) * (kro_g / kro_max + krg) - krw - krg) * kro_max;
  if (val(v) <= 0.0 || val(v) >= kro_max) return sc<S>(rclamp(val(v), 0.0, kro_max));
  return v;
}

// capillary_pressure_og_generic (capillary.rs:130-153)
template <class S>
inline S pc_og_g(const Scal3& rock, double entry, double lambda, const S& sg) {
  const double denom = 1.0 - rock.s_wc - rock.s_org;
  if (denom <= 0.0) return sc<S>(entry * 20.0);
  S so = sc<S>(1.0 - rock.s_wc) - sg;
  S e = min_ceil(max_floor((so - rock.s_org) / denom, 0.0), 1.0);
  const double pc_max = entry * 20.0;
  if (val(e) <= 0.0) return sc<S>(pc_max);
  S pc = s_powf(e, -1.0 / lambda) * entry;
  return min_ceil(max_floor(pc, 0.0), pc_max);
}

}  // namespace orc
