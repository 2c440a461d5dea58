// rf_blackoil.cuh — three-phase black-oil physics of the fully implicit step, as __host__
// __device__ templates over `double` and `Dual<N>` (the same pattern as rf_physics.cuh).  Kernels
// instantiate them with Dual<3>/Dual<4>/Dual<6> for exact Jacobian blocks; the host controller
// uses the plain routines for the per-well logic, reading the PVT table from its host copy.
//
// Reference semantics kept (src/lib/ressim/src/…):
//   pvt.rs:46-500                PVTO/PVDG-style table: saturated curve, undersaturated oil
//                                branches, plain and generic interpolation (linear in 1/B and
//                                1/(B mu)); the segment is chosen on the value of p
//   pvt.rs:636-693, 769-841,     simulator-level accessors (Bo/mu_o for a given Rs, Bg, mu_g)
//   988-1009                     and phase densities
//   relperm.rs:199-458           three-phase Corey with Stone II (zero derivative at the clamps)
//   capillary.rs:100-172         gas-oil capillary pressure, capped at 20x entry
//   mobility.rs:114-249          phase mobilities
//   step.rs:65-200,              Rs bisection and the gas-inventory split (gas redissolution on),
//   fim/flash_ad.rs:25-207       differentiated through one implicit-function Newton step
//   fim/flash.rs:13-160          regime classification and the cell flash
//   fim/properties.rs:37-212     cell properties per regime (0 saturated: hc = Sg; 1
//                                undersaturated: hc = Rs), component inventory
//   fim/flux.rs:42-191           three-phase face flux, dissolved gas carried with the oil
//   fim/wells_ad.rs:44-229       producer fractions, connection rate, component coefficients and
//                                surface rates, gas injection
// Where the reference keeps a plain f64 routine beside its generic mirror, both appear here, and
// each caller uses the one the reference's caller uses (their roundings differ).
#pragma once

#include "rf_physics.cuh"

namespace rf {

constexpr double kPvtoRsTol = 1e-6;  // pvt.rs:17

// ---- Dual helpers the black-oil expressions need ----
template <int N>
RF_HD Dual<N> operator-(double a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -b.d[i];
  return r;
}
RF_HD double srecip(double x) { return 1.0 / x; }
template <int N>
RF_HD Dual<N> srecip(const Dual<N>& a) {
  Dual<N> r;
  r.v = 1.0 / a.v;
  const double coef = -r.v * r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * coef;
  return r;
}
RF_HD double smax(double a, double b) { return fmax(a, b); }
template <int N>
RF_HD Dual<N> smax(const Dual<N>& a, const Dual<N>& b) {
  return a.v >= b.v ? a : b;
}
RF_HD double clamp01(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

// ---------------------------------------------------------------------------------------------
// PVT table
// ---------------------------------------------------------------------------------------------
struct PvtRowV {
  double p, rs, bo, mu_o, bg, mu_g;
};
RF_HD PvtRowV pvt_row(const double* r) { return PvtRowV{r[0], r[1], r[2], r[3], r[4], r[5]}; }
RF_HD PvtRowV sat_row(const Fluid& f, int i) { return pvt_row(f.pvt + 6 * i); }
RF_HD double br_rs(const Fluid& f, int b) { return f.pvt[f.pvt_hdr + 3 * b]; }
RF_HD int br_first(const Fluid& f, int b) { return int(f.pvt[f.pvt_hdr + 3 * b + 1]); }
RF_HD int br_count(const Fluid& f, int b) { return int(f.pvt[f.pvt_hdr + 3 * b + 2]); }
RF_HD PvtRowV br_row(const Fluid& f, int b, int r) { return pvt_row(f.pvt + f.pvt_rows + 6 * (br_first(f, b) + r)); }

// interpolate_oil_segment / interpolate_gas_segment (pvt.rs:64-77)
RF_HD void oil_segment(const PvtRowV& r0, const PvtRowV& r1, double t, double& bo, double& mu) {
  const double inv_bo = (1.0 / r0.bo) + t * (1.0 / r1.bo - 1.0 / r0.bo);
  const double inv_bo_mu = (1.0 / (r0.bo * r0.mu_o)) + t * (1.0 / (r1.bo * r1.mu_o) - 1.0 / (r0.bo * r0.mu_o));
  bo = 1.0 / inv_bo;
  mu = inv_bo / inv_bo_mu;
}
RF_HD void gas_segment(const PvtRowV& r0, const PvtRowV& r1, double t, double& bg, double& mu) {
  const double inv_bg = (1.0 / r0.bg) + t * (1.0 / r1.bg - 1.0 / r0.bg);
  const double inv_bg_mu = (1.0 / (r0.bg * r0.mu_g)) + t * (1.0 / (r1.bg * r1.mu_g) - 1.0 / (r0.bg * r0.mu_g));
  bg = 1.0 / inv_bg;
  mu = inv_bg / inv_bg_mu;
}

// interpolate_rows over the saturated curve (pvt.rs:137-186, 250-252)
RF_HD_CALL PvtRowV pvt_interpolate(const Fluid& f, double p) {
  const int n = f.pvt_n_sat;
  if (n == 0) return PvtRowV{p, 0.0, 1.0, 1.0, 1.0, 0.02};
  const PvtRowV first = sat_row(f, 0);
  if (p <= first.p) return first;
  const int last = n - 1;
  const PvtRowV l = sat_row(f, last);
  if (p >= l.p) {
    PvtRowV e = l;
    e.p = p;
    e.bo = l.bo * exp(-f.pvt_c_o * (p - l.p));
    e.bg = l.bg * (l.p / p);
    return e;
  }
  for (int i = 0; i < last; ++i) {
    const PvtRowV r0 = sat_row(f, i), r1 = sat_row(f, i + 1);
    if (p >= r0.p && p <= r1.p) {
      const double dp = r1.p - r0.p;
      if (dp < 1e-6) return r0;
      const double tt = (p - r0.p) / dp;
      PvtRowV r;
      r.p = p;
      r.rs = r0.rs + tt * (r1.rs - r0.rs);
      oil_segment(r0, r1, tt, r.bo, r.mu_o);
      gas_segment(r0, r1, tt, r.bg, r.mu_g);
      return r;
    }
  }
  return l;
}

// branch_props (pvt.rs:188-225)
RF_HD void branch_props(const Fluid& f, int b, double p, double& bo, double& mu) {
  const int n = br_count(f, b);
  const double c_o = f.pvt_c_o;
  if (n == 0) {
    bo = 1.0;
    mu = 1.0;
    return;
  }
  const PvtRowV r0f = br_row(f, b, 0);
  if (n == 1) {
    bo = r0f.bo * exp(-c_o * (p - r0f.p));
    mu = r0f.mu_o * exp(c_o * (p - r0f.p));
    return;
  }
  if (p <= r0f.p) {
    bo = r0f.bo;
    mu = r0f.mu_o;
    return;
  }
  for (int i = 0; i + 1 < n; ++i) {
    const PvtRowV r0 = br_row(f, b, i), r1 = br_row(f, b, i + 1);
    if (p >= r0.p && p <= r1.p) {
      const double dp = r1.p - r0.p;
      if (fabs(dp) < 1e-9) {
        bo = r0.bo;
        mu = r0.mu_o;
        return;
      }
      oil_segment(r0, r1, (p - r0.p) / dp, bo, mu);
      return;
    }
  }
  const PvtRowV l = br_row(f, b, n - 1);
  const double excess = p - l.p;
  bo = fmax(l.bo * exp(-c_o * excess), 1e-9);
  mu = l.mu_o * exp(c_o * excess);
}

// branch_bounds (pvt.rs:227-248)
RF_HD bool branch_bounds(const Fluid& f, double rs, int& lo, int& hi) {
  if (f.pvt_n_br == 0) return false;
  const int last = f.pvt_n_br - 1;
  if (rs <= br_rs(f, 0) + kPvtoRsTol) {
    lo = hi = 0;
    return true;
  }
  if (rs >= br_rs(f, last) - kPvtoRsTol) {
    lo = hi = last;
    return true;
  }
  for (int i = 0; i < last; ++i)
    if (rs >= br_rs(f, i) - kPvtoRsTol && rs <= br_rs(f, i + 1) + kPvtoRsTol) {
      lo = i;
      hi = i + 1;
      return true;
    }
  lo = hi = last;
  return true;
}

// interpolate_oil (pvt.rs:458-488)
RF_HD_CALL void pvt_interpolate_oil(const Fluid& f, double p, double rs, double& bo, double& mu) {
  if (f.pvt_n_sat == 0) {
    bo = 1.0;
    mu = 1.0;
    return;
  }
  const PvtRowV sat = pvt_interpolate(f, p);
  if (rs >= sat.rs - 1e-6) {
    bo = sat.bo;
    mu = sat.mu_o;
    return;
  }
  int lo, hi;
  if (branch_bounds(f, rs, lo, hi)) {
    double bo_low, mu_low;
    branch_props(f, lo, p, bo_low, mu_low);
    const double rs_lo = br_rs(f, lo), rs_hi = br_rs(f, hi);
    if (fabs(rs_hi - rs_lo) <= kPvtoRsTol) {
      bo = bo_low;
      mu = mu_low;
      return;
    }
    const double tt = (rs - rs_lo) / (rs_hi - rs_lo);
    const double shift = br_row(f, hi, 0).p - br_row(f, lo, 0).p;
    const double p_low = p - tt * shift;
    const double p_high = p + (1.0 - tt) * shift;
    double bo_high, mu_high;
    branch_props(f, lo, p_low, bo_low, mu_low);
    branch_props(f, hi, p_high, bo_high, mu_high);
    const double inv_bo = 1.0 / bo_low + tt * (1.0 / bo_high - 1.0 / bo_low);
    const double inv_bo_mu = 1.0 / (bo_low * mu_low) + tt * (1.0 / (bo_high * mu_high) - 1.0 / (bo_low * mu_low));
    bo = 1.0 / inv_bo;
    mu = inv_bo / inv_bo_mu;
    return;
  }
  bo = sat.bo;
  mu = sat.mu_o;
}

// ---- generic interpolation ----
template <class S>
struct SatProps {
  S rs, bo, bg, mu_o, mu_g;
};

// interpolate_oil_segment_generic (pvt.rs:79-84)
template <class S>
RF_HD void oil_segment_g(const PvtRowV& r0, const PvtRowV& r1, const S& t, S& bo, S& mu) {
  S inv_bo = t * (1.0 / r1.bo - 1.0 / r0.bo) + 1.0 / r0.bo;
  S inv_bo_mu = t * (1.0 / (r1.bo * r1.mu_o) - 1.0 / (r0.bo * r0.mu_o)) + 1.0 / (r0.bo * r0.mu_o);
  bo = srecip(inv_bo);
  mu = inv_bo / inv_bo_mu;
}

// interpolate_saturated_generic (pvt.rs:259-342)
template <class S>
RF_HD_CALL SatProps<S> pvt_saturated_g(const Fluid& f, const S& p) {
  SatProps<S> o;
  const int n = f.pvt_n_sat;
  if (n == 0) {
    o.rs = lift<S>(0.0);
    o.bo = lift<S>(1.0);
    o.bg = lift<S>(1.0);
    o.mu_o = lift<S>(1.0);
    o.mu_g = lift<S>(0.02);
    return o;
  }
  const double pv = value(p);
  const int last = n - 1;
  int seg = -1;
  PvtRowV r0 = sat_row(f, 0), r1 = r0;
  if (pv <= r0.p) {
    seg = -2;
  } else if (pv >= sat_row(f, last).p) {
    const PvtRowV r = sat_row(f, last);
    o.bo = lift<S>(r.bo) * sexp((p * (-f.pvt_c_o)) + (f.pvt_c_o * r.p));
    o.bg = lift<S>(r.bg * r.p) / p;
    o.rs = lift<S>(r.rs);
    o.mu_o = lift<S>(r.mu_o);
    o.mu_g = lift<S>(r.mu_g);
    return o;
  } else {
    for (int i = 0; i < last; ++i) {
      r0 = sat_row(f, i);
      r1 = sat_row(f, i + 1);
      if (pv >= r0.p && pv <= r1.p) {
        seg = i;
        break;
      }
    }
  }
  if (seg >= 0 && !(r1.p - r0.p < 1e-6)) {
    const double dp = r1.p - r0.p;
    S tt = (p - r0.p) / dp;
    S inv_bg = tt * (1.0 / r1.bg - 1.0 / r0.bg) + 1.0 / r0.bg;
    S inv_bg_mu = tt * (1.0 / (r1.bg * r1.mu_g) - 1.0 / (r0.bg * r0.mu_g)) + 1.0 / (r0.bg * r0.mu_g);
    o.rs = tt * (r1.rs - r0.rs) + r0.rs;
    S bo, mu;
    oil_segment_g(r0, r1, tt, bo, mu);
    o.bo = bo;
    o.bg = lift<S>(1.0) / inv_bg;
    o.mu_o = mu;
    o.mu_g = inv_bg / inv_bg_mu;
    return o;
  }
  // constant row: the first row (p at or below it), a degenerate segment's left row, or the last
  const PvtRowV c = seg == -2 ? sat_row(f, 0) : (seg >= 0 ? r0 : sat_row(f, last));
  o.rs = lift<S>(c.rs);
  o.bo = lift<S>(c.bo);
  o.bg = lift<S>(c.bg);
  o.mu_o = lift<S>(c.mu_o);
  o.mu_g = lift<S>(c.mu_g);
  return o;
}

// branch_props_generic (pvt.rs:344-382)
template <class S>
RF_HD_CALL void branch_props_g(const Fluid& f, int b, const S& p, S& bo, S& mu) {
  const int n = br_count(f, b);
  const double c_o = f.pvt_c_o;
  if (n == 0) {
    bo = lift<S>(1.0);
    mu = lift<S>(1.0);
    return;
  }
  const PvtRowV r0f = br_row(f, b, 0);
  if (n == 1) {
    S excess = p - r0f.p;
    bo = lift<S>(r0f.bo) * sexp(excess * (-c_o));
    mu = lift<S>(r0f.mu_o) * sexp(excess * c_o);
    return;
  }
  const double pv = value(p);
  if (pv <= r0f.p) {
    bo = lift<S>(r0f.bo);
    mu = lift<S>(r0f.mu_o);
    return;
  }
  for (int i = 0; i + 1 < n; ++i) {
    const PvtRowV r0 = br_row(f, b, i), r1 = br_row(f, b, i + 1);
    if (pv >= r0.p && pv <= r1.p) {
      const double dp = r1.p - r0.p;
      if (fabs(dp) < 1e-9) {
        bo = lift<S>(r0.bo);
        mu = lift<S>(r0.mu_o);
        return;
      }
      S tt = (p - r0.p) / dp;
      oil_segment_g(r0, r1, tt, bo, mu);
      return;
    }
  }
  const PvtRowV l = br_row(f, b, n - 1);
  S excess = p - l.p;
  bo = floor_at(lift<S>(l.bo) * sexp(excess * (-c_o)), 1e-9);
  mu = lift<S>(l.mu_o) * sexp(excess * c_o);
}

// interpolate_oil_generic (pvt.rs:384-425); `sat` is the saturated curve at p
template <class S>
RF_HD_CALL void pvt_oil_sat_g(const Fluid& f, const SatProps<S>& sat, const S& p, const S& rs, S& bo, S& mu) {
  if (f.pvt_n_sat == 0) {
    bo = lift<S>(1.0);
    mu = lift<S>(1.0);
    return;
  }
  const double rs_sat = value(sat.rs);
  if (value(rs) >= rs_sat - 1e-6) {
    bo = sat.bo;
    mu = sat.mu_o;
    return;
  }
  int lo, hi;
  if (branch_bounds(f, value(rs), lo, hi)) {
    S bo_low, mu_low;
    branch_props_g(f, lo, p, bo_low, mu_low);
    const double rs_lo = br_rs(f, lo), rs_hi = br_rs(f, hi);
    if (fabs(rs_hi - rs_lo) <= kPvtoRsTol) {
      bo = bo_low;
      mu = mu_low;
      return;
    }
    S tt = (rs - rs_lo) / (rs_hi - rs_lo);
    const double shift = br_row(f, hi, 0).p - br_row(f, lo, 0).p;
    S p_low = p - tt * shift;
    S p_high = p + (lift<S>(1.0) - tt) * shift;
    S bo_high, mu_high;
    branch_props_g(f, lo, p_low, bo_low, mu_low);
    branch_props_g(f, hi, p_high, bo_high, mu_high);
    S inv_bo = tt * (srecip(bo_high) - srecip(bo_low)) + srecip(bo_low);
    S inv_bo_mu = tt * (srecip(bo_high * mu_high) - srecip(bo_low * mu_low)) + srecip(bo_low * mu_low);
    bo = srecip(inv_bo);
    mu = inv_bo / inv_bo_mu;
    return;
  }
  bo = sat.bo;
  mu = sat.mu_o;
}
template <class S>
RF_HD void pvt_oil_g(const Fluid& f, const S& p, const S& rs, S& bo, S& mu) {
  pvt_oil_sat_g(f, pvt_saturated_g(f, p), p, rs, bo, mu);
}

// ---------------------------------------------------------------------------------------------
// Three-phase relative permeability (Corey + Stone II) and gas-oil capillary pressure
// ---------------------------------------------------------------------------------------------
// interpolate_piecewise (relperm.rs:124-147) on column y of n rows of three doubles (x first)
RF_HD double table3(const double* t, int n, int y, double x) {
  if (x <= t[0]) return t[y];
  for (int r = 0; r + 1 < n; ++r) {
    const double x0 = t[3 * r], x1 = t[3 * r + 3];
    if (x <= x1) {
      if (fabs(x1 - x0) <= 2.220446049250313e-16) return t[3 * r + 3 + y];
      const double fr = clamp01((x - x0) / (x1 - x0), 0.0, 1.0);
      return t[3 * r + y] + fr * (t[3 * r + 3 + y] - t[3 * r + y]);
    }
  }
  return t[3 * (n - 1) + y];
}
// interpolate_piecewise_generic (relperm.rs:9-40): segment from the value, derivative of the
// active segment
template <class S>
RF_HD S table3_g(const double* t, int n, int y, const S& x) {
  const double xv = value(x);
  if (xv <= t[0]) return lift<S>(t[y]);
  for (int r = 0; r + 1 < n; ++r) {
    const double x0 = t[3 * r], x1 = t[3 * r + 3];
    if (xv <= x1) {
      if (fabs(x1 - x0) <= 2.220446049250313e-16) return lift<S>(t[3 * r + 3 + y]);
      S fr = ceil_at(floor_at((x - x0) / (x1 - x0), 0.0), 1.0);
      const double y0 = t[3 * r + y], y1 = t[3 * r + 3 + y];
      return fr * (y1 - y0) + y0;
    }
  }
  return lift<S>(t[3 * (n - 1) + y]);
}

RF_HD double k_rw3(const Fluid& s, double sw) {
  if (s.n_swof) return table3(s.pvt + s.swof_off, s.n_swof, 1, sw);
  const double e = clamp01((sw - s.s3_wc) / (1.0 - s.s3_wc - s.s3_or), 0.0, 1.0);
  return s.s3_krw * pow(e, s.s3_nw);
}
RF_HD double k_rg3(const Fluid& s, double sg) {
  if (s.n_sgof) return table3(s.pvt + s.sgof_off, s.n_sgof, 1, sg);
  const double denom = 1.0 - s.s3_wc - s.s3_gc - s.s3_gr;
  if (denom <= 0.0) return 0.0;
  const double e = clamp01((sg - s.s3_gc) / denom, 0.0, 1.0);
  return s.s3_krg * pow(e, s.s3_ng);
}
RF_HD double k_ro_water3(const Fluid& s, double sw) {
  if (s.n_swof) return table3(s.pvt + s.swof_off, s.n_swof, 2, sw);
  const double e = clamp01((1.0 - sw - s.s3_or) / (1.0 - s.s3_wc - s.s3_or), 0.0, 1.0);
  return s.s3_kro * pow(e, s.s3_no);
}
RF_HD double k_ro_gas3(const Fluid& s, double sg) {
  if (s.n_sgof) return table3(s.pvt + s.sgof_off, s.n_sgof, 2, sg);
  const double denom = 1.0 - s.s3_wc - s.s3_org;
  if (denom <= 0.0) return 0.0;
  const double e = clamp01((1.0 - s.s3_wc - sg - s.s3_org) / denom, 0.0, 1.0);
  return s.s3_kro * pow(e, s.s3_no);
}
RF_HD double k_ro_stone2(const Fluid& s, double sw, double sg) {
  const double kro_max = s.s3_kro;
  const double kro_w = k_ro_water3(s, sw), kro_g = k_ro_gas3(s, sg);
  const double krw = k_rw3(s, sw), krg = k_rg3(s, sg);
  const double v = kro_max * ((kro_w / kro_max + krw) * (kro_g / kro_max + krg) - krw - krg);
  return clamp01(v, 0.0, kro_max);
}

template <class S>
RF_HD S k_rw3_g(const Fluid& s, const S& sw) {
  if (s.n_swof) return table3_g(s.pvt + s.swof_off, s.n_swof, 1, sw);
  const double denom = 1.0 - s.s3_wc - s.s3_or;
  S e = ceil_at(floor_at((sw - s.s3_wc) / denom, 0.0), 1.0);
  return spow(e, s.s3_nw) * s.s3_krw;
}
template <class S>
RF_HD S k_rg3_g(const Fluid& s, const S& sg) {
  if (s.n_sgof) return table3_g(s.pvt + s.sgof_off, s.n_sgof, 1, sg);
  const double denom = 1.0 - s.s3_wc - s.s3_gc - s.s3_gr;
  S e = ceil_at(floor_at((sg - s.s3_gc) / denom, 0.0), 1.0);
  return spow(e, s.s3_ng) * s.s3_krg;
}
template <class S>
RF_HD S k_ro_water3_g(const Fluid& s, const S& sw) {
  if (s.n_swof) return table3_g(s.pvt + s.swof_off, s.n_swof, 2, sw);
  const double denom = 1.0 - s.s3_wc - s.s3_or;
  S e = ceil_at(floor_at((lift<S>(1.0 - s.s3_or) - sw) / denom, 0.0), 1.0);
  return spow(e, s.s3_no) * s.s3_kro;
}
template <class S>
RF_HD S k_ro_gas3_g(const Fluid& s, const S& sg) {
  if (s.n_sgof) return table3_g(s.pvt + s.sgof_off, s.n_sgof, 2, sg);
  const double denom = 1.0 - s.s3_wc - s.s3_org;
  S e = ceil_at(floor_at((lift<S>(1.0 - s.s3_wc - s.s3_org) - sg) / denom, 0.0), 1.0);
  return spow(e, s.s3_no) * s.s3_kro;
}
// k_ro_stone2_generic (relperm.rs:431-457): zero derivative at and beyond either clamp bound
template <class S>
RF_HD S k_ro_stone2_g(const Fluid& s, const S& sw, const S& sg) {
  const double kro_max = s.s3_kro;
  S kro_w = k_ro_water3_g(s, sw), kro_g = k_ro_gas3_g(s, sg);
  S krw = k_rw3_g(s, sw), krg = k_rg3_g(s, sg);
  S v = ((kro_w / kro_max + krw) * (kro_g / kro_max + krg) - krw - krg) * kro_max;
  if (value(v) <= 0.0 || value(v) >= kro_max) return lift<S>(clamp01(value(v), 0.0, kro_max));
  return v;
}
// analytic two-phase Corey (relperm.rs:491-520), the three-phase mode's curves without SCAL3
template <class S>
RF_HD void corey_analytic(const Fluid& f, const S& sw, S& krw, S& kro) {
  const double denom = 1.0 - f.s_wc - f.s_or;
  S ew = ceil_at(floor_at((sw - f.s_wc) / denom, 0.0), 1.0);
  krw = spow(ew, f.n_w) * f.krw_max;
  S eo = ceil_at(floor_at((lift<S>(1.0 - f.s_or) - sw) / denom, 0.0), 1.0);
  kro = spow(eo, f.n_o) * f.kro_max;
}

// capillary_pressure_og_generic (capillary.rs:130-153), used by the flux when both the gas-oil
// parameters and the three-phase SCAL are set (flux.rs:137-142)
template <class S>
RF_HD S pc_og(const Fluid& f, const S& sg) {
  if (!(f.has_pc_og && f.has_scal3)) return lift<S>(0.0);
  const double denom = 1.0 - f.s3_wc - f.s3_org;
  if (denom <= 0.0) return lift<S>(f.pcog_entry * 20.0);
  S so = lift<S>(1.0 - f.s3_wc) - sg;
  S e = ceil_at(floor_at((so - f.s3_org) / denom, 0.0), 1.0);
  const double pc_max = f.pcog_entry * 20.0;
  if (value(e) <= 0.0) return lift<S>(pc_max);
  S pc = spow(e, -1.0 / f.pcog_lambda) * f.pcog_entry;
  return ceil_at(floor_at(pc, 0.0), pc_max);
}

// ---------------------------------------------------------------------------------------------
// Simulator-level accessors, densities and mobilities (three-phase mode always has a table)
// ---------------------------------------------------------------------------------------------
// get_b_o_for_rs / get_mu_o_for_rs (pvt.rs:649-659, 792-803), get_b_g / get_mu_g (:665-671, 835-841)
RF_HD double bo_for_rs(const Fluid& f, double p, double rs) {
  double bo, mu;
  pvt_interpolate_oil(f, p, rs, bo, mu);
  return bo;
}
RF_HD double mu_o_for_rs(const Fluid& f, double p, double rs) {
  double bo, mu;
  pvt_interpolate_oil(f, p, rs, bo, mu);
  return mu;
}
RF_HD double get_b_g(const Fluid& f, double p) { return pvt_interpolate(f, p).bg; }
RF_HD double get_mu_g(const Fluid& f, double p) { return pvt_interpolate(f, p).mu_g; }

// oil_density_generic / gas_density_generic (pvt.rs:988-1009)
template <class S>
RF_HD S oil_density3(const Fluid& f, const S& p, const S& rs) {
  S bo, mu;
  pvt_oil_g(f, p, rs, bo, mu);
  return (lift<S>(f.rho_o) + rs * f.rho_g) / floor_at(bo, 1e-9);
}
template <class S>
RF_HD S gas_density3(const Fluid& f, const S& p) {
  return lift<S>(f.rho_g) / floor_at(pvt_saturated_g(f, p).bg, 1e-9);
}

template <class S>
struct Mob3 {
  S w, o, g;
};
// phase_mobilities_for_state_generic, three-phase branch (mobility.rs:196-249)
template <class S>
RF_HD_CALL Mob3<S> mobilities3(const Fluid& f, const S& sw, const S& sg, const S& p, const S& rs) {
  const S mu_w = lift<S>(f.mu_w);
  Mob3<S> m;
  S bo, mu_o;
  pvt_oil_g(f, p, rs, bo, mu_o);
  if (!f.has_scal3) {
    S krw, kro;
    corey_analytic(f, sw, krw, kro);
    m.w = krw / mu_w;
    m.o = kro / mu_o;
    m.g = lift<S>(0.0);
    return m;
  }
  m.w = k_rw3_g(f, sw) / mu_w;
  m.o = k_ro_stone2_g(f, sw, sg) / mu_o;
  m.g = k_rg3_g(f, sg) / pvt_saturated_g(f, p).mu_g;
  return m;
}
// phase_mobilities (mobility.rs:114-149), plain f64, three-phase branch
inline Mob3<double> mobilities3_f64(const Fluid& f, double sw, double sg, double p, double rs) {
  if (!f.has_scal3) return Mob3<double>{corey_krw(f, sw) / f.mu_w, corey_kro(f, sw) / mu_o_for_rs(f, p, rs), 0.0};
  return Mob3<double>{k_rw3(f, sw) / f.mu_w, k_ro_stone2(f, sw, sg) / mu_o_for_rs(f, p, rs),
                      k_rg3(f, sg) / get_mu_g(f, p)};
}

// ---------------------------------------------------------------------------------------------
// The gas flash
// ---------------------------------------------------------------------------------------------
// solve_rs_for_dissolved_gas (step.rs:65-104): 64 bisection steps on So PV rs / Bo(p, rs)
RF_HD_CALL double solve_rs_plain(const Fluid& f, double p, double sw, double sg, double pv, double dissolved,
                            double rs_upper) {
  const double target = fmax(dissolved, 0.0);
  if (target <= 0.0 || rs_upper <= 0.0) return 0.0;
  const double so = fmax(1.0 - sw - sg, 0.0);
  if (so <= 1e-12 || pv <= 0.0) return 0.0;
  double lo = 0.0, hi = fmax(rs_upper, 0.0);
  for (int i = 0; i < 64; ++i) {
    const double mid = 0.5 * (lo + hi);
    double bo, mu;
    pvt_interpolate_oil(f, p, mid, bo, mu);
    const double d = (so * pv / fmax(bo, 1e-9)) * mid;
    if (d < target)
      lo = mid;
    else
      hi = mid;
  }
  return 0.5 * (lo + hi);
}

// split_gas_inventory_after_transport (step.rs:106-200), plain; base: the DRSDT0 Rs cap (read
// only when f.drsdt0)
RF_HD_CALL void split_gas_plain(const Fluid& f, double p, double pv, double sw, double free_sc, double dissolved_sc,
                                double base, double& sg, double& so, double& rs) {
  const double total_hc = fmax(1.0 - sw, 0.0);
  const double bg = fmax(get_b_g(f, p), 1e-9);
  const double free_t = fmax(free_sc, 0.0);
  const double sg_t = clamp01((free_t * bg) / fmax(pv, 1e-9), 0.0, total_hc);
  const double so_t = fmax(total_hc - sg_t, 0.0);
  const double dissolved = fmax(dissolved_sc, 0.0);
  const double rs_max = fmax(pvt_interpolate(f, p).rs, 0.0);
  const bool redis = !f.drsdt0;
  const double cap = redis ? rs_max : fmin(fmax(base, 0.0), rs_max);
  double bo_cap, mu;
  pvt_interpolate_oil(f, p, cap, bo_cap, mu);
  bo_cap = fmax(bo_cap, 1e-9);
  if (!redis) {
    const double max_t = (so_t * pv / bo_cap) * cap;
    if (dissolved <= max_t + 1e-9) {
      rs = solve_rs_plain(f, p, sw, sg_t, pv, dissolved, cap);
      sg = sg_t;
      so = so_t;
      return;
    }
  }
  const double total_gas = free_t + dissolved;
  double rs_sat, bo_sat;
  if (redis) {
    double bo_sat_raw;
    pvt_interpolate_oil(f, p, rs_max, bo_sat_raw, mu);
    rs_sat = rs_max;
    bo_sat = fmax(bo_sat_raw, 1e-9);
  } else {
    rs_sat = cap;
    bo_sat = bo_cap;
  }
  const double max_all = (total_hc * pv / bo_sat) * rs_sat;
  if (redis && total_gas <= max_all + 1e-9) {
    rs = solve_rs_plain(f, p, sw, 0.0, pv, total_gas, rs_sat);
    sg = 0.0;
    so = total_hc;
    return;
  }
  const double denom = (1.0 / bg) - (rs_sat / bo_sat);
  const double sg_sat = fabs(denom) > 1e-12 ? ((total_gas / pv) - (total_hc * rs_sat / bo_sat)) / denom : sg_t;
  sg = clamp01(sg_sat, redis ? 0.0 : sg_t, total_hc);
  so = fmax(total_hc - sg, 0.0);
  rs = rs_sat;
}

// dissolved_gas_value_generic (flash_ad.rs:29-43)
template <class S>
RF_HD S dissolved_gas_g(const Fluid& f, const S& p, const S& rs, const S& so, const S& pv) {
  S bo, mu;
  pvt_oil_g(f, p, rs, bo, mu);
  return (so * pv / floor_at(bo, 1e-9)) * rs;
}
// solve_rs_for_dissolved_gas_generic (flash_ad.rs:46-100): the plain root, with its derivative
// from one implicit-function Newton step
template <class S>
RF_HD S solve_rs_g(const Fluid& f, const S& p, const S& sw, const S& sg, const S& pv, const S& dissolved,
                   double rs_upper) {
  const double rs_star = solve_rs_plain(f, value(p), value(sw), value(sg), value(pv), value(dissolved), rs_upper);
  S so = floor_at(lift<S>(1.0) - sw - sg, 0.0);
  S target = floor_at(dissolved, 0.0);
  const double dgdrs = dissolved_gas_g<Dual<1>>(f, dconst<1>(value(p)), dvar<1>(rs_star, 0), dconst<1>(value(so)),
                                                dconst<1>(value(pv)))
                           .d[0];
  if (fabs(dgdrs) < 1e-14) return lift<S>(rs_star);
  S g = dissolved_gas_g<S>(f, p, lift<S>(rs_star), so, pv) - target;
  return lift<S>(rs_star) - g / dgdrs;
}
// split_gas_inventory_after_transport_generic (flash_ad.rs:104-207)
template <class S>
RF_HD_CALL void split_gas_g(const Fluid& f, const S& p, const S& pv, const S& sw, const S& free_sc,
                            const S& dissolved_sc, double base, S& sg, S& so, S& rs) {
  S total_hc = floor_at(lift<S>(1.0) - sw, 0.0);
  const SatProps<S> sat = pvt_saturated_g(f, p);
  S bg = floor_at(sat.bg, 1e-9);
  S free_t = floor_at(free_sc, 0.0);
  S sg_t = smin(floor_at((free_t * bg) / floor_at(pv, 1e-9), 0.0), total_hc);
  S so_t = floor_at(total_hc - sg_t, 0.0);
  S dissolved = floor_at(dissolved_sc, 0.0);
  S rs_max = floor_at(sat.rs, 0.0);
  const bool redis = !f.drsdt0;
  S cap = redis ? rs_max : smin(lift<S>(fmax(base, 0.0)), rs_max);
  S bo_cap, mu;
  pvt_oil_sat_g(f, sat, p, cap, bo_cap, mu);
  bo_cap = floor_at(bo_cap, 1e-9);
  if (!redis) {
    S max_t = (so_t * pv / bo_cap) * cap;
    if (value(dissolved) <= value(max_t) + 1e-9) {
      rs = solve_rs_g(f, p, sw, sg_t, pv, dissolved, value(cap));
      sg = sg_t;
      so = so_t;
      return;
    }
  }
  S total_gas = free_t + dissolved;
  S rs_sat, bo_sat;
  if (redis) {
    S bo_sat_raw;
    pvt_oil_sat_g(f, sat, p, rs_max, bo_sat_raw, mu);
    rs_sat = rs_max;
    bo_sat = floor_at(bo_sat_raw, 1e-9);
  } else {
    rs_sat = cap;
    bo_sat = bo_cap;
  }
  S max_all = (total_hc * pv / bo_sat) * rs_sat;
  if (redis && value(total_gas) <= value(max_all) + 1e-9) {
    rs = solve_rs_g(f, p, sw, lift<S>(0.0), pv, total_gas, value(rs_sat));
    sg = lift<S>(0.0);
    so = total_hc;
    return;
  }
  S denom = srecip(bg) - (rs_sat / bo_sat);
  S sg_sat = fabs(value(denom)) > 1e-12 ? ((total_gas / pv) - (total_hc * rs_sat / bo_sat)) / denom : sg_t;
  sg = smin(smax(sg_sat, redis ? lift<S>(0.0) : sg_t), total_hc);
  so = floor_at(total_hc - sg, 0.0);
  rs = rs_sat;
}

// classify_cell_regime (flash.rs:13-40): 0 saturated, 1 undersaturated
RF_HD int classify_regime(const Fluid& f, double p, double sg, double rs, double base) {
  if (sg > 1e-9) return 0;
  double rs_sat = pvt_interpolate(f, p).rs;
  if (f.drsdt0) rs_sat = fmin(rs_sat, base);
  return rs < rs_sat - 1e-6 ? 1 : 0;
}

// resolve_cell_flash (flash.rs:43-160) and derive_cell (state.rs:823-854), plain
struct Derived3 {
  int regime;
  double so, sg, rs, bo, bg;
};
RF_HD Derived3 derive_cell3(const Fluid& f, double p, double sw, double hc, int regime, double base) {
  Derived3 d;
  const double raw_total = 1.0 - sw;
  d.regime = regime;
  if (regime == 0) {
    d.sg = hc;
    d.rs = pvt_interpolate(f, p).rs;
    if (f.drsdt0) d.rs = fmin(d.rs, base);
    d.so = raw_total - d.sg;
  } else {
    double rs_cap = fmax(pvt_interpolate(f, p).rs, 0.0);
    if (f.drsdt0) rs_cap = fmin(rs_cap, fmax(base, 0.0));
    const double rs_trial = hc;
    if (rs_trial <= rs_cap + 1e-6) {
      d.so = raw_total;
      d.sg = 0.0;
      d.rs = rs_trial;
    } else {
      const double bo_trial = fmax(bo_for_rs(f, p, rs_trial), 1e-9);
      const double dissolved = raw_total * rs_trial / bo_trial;
      split_gas_plain(f, p, 1.0, sw, 0.0, dissolved, base, d.sg, d.so, d.rs);
      d.regime = d.sg > 1e-12 ? 0 : 1;
    }
  }
  double mu;
  pvt_interpolate_oil(f, p, d.rs, d.bo, mu);
  d.bg = pvt_interpolate(f, p).bg;
  return d;
}

// ---------------------------------------------------------------------------------------------
// Cell properties, inventory and face flux
// ---------------------------------------------------------------------------------------------
template <class S>
struct Props3 {
  S so, sg, rs, bo, bg;
};
// cell_props_generic, black-oil branch (properties.rs:37-133)
template <class S>
RF_HD_CALL Props3<S> cell_props3(const Fluid& f, int regime, const S& p, const S& sw, const S& hc, double base) {
  const S raw_total = lift<S>(1.0) - sw;
  const SatProps<S> sat = pvt_saturated_g(f, p);
  Props3<S> pr;
  S mu;
  if (regime == 0) {
    pr.sg = hc;
    pr.rs = sat.rs;
    if (f.drsdt0) pr.rs = ceil_at(pr.rs, base);
    pr.so = raw_total - pr.sg;
    pvt_oil_sat_g(f, sat, p, pr.rs, pr.bo, mu);
    pr.bg = sat.bg;
    return pr;
  }
  S rs_cap = floor_at(sat.rs, 0.0);
  if (f.drsdt0) rs_cap = smin(rs_cap, lift<S>(fmax(base, 0.0)));
  const S& rs_trial = hc;
  if (value(rs_trial) <= value(rs_cap) + 1e-6) {
    pr.sg = lift<S>(0.0);
    pr.so = raw_total;
    pr.rs = rs_trial;
  } else {
    S bo_t;
    pvt_oil_sat_g(f, sat, p, rs_trial, bo_t, mu);
    bo_t = floor_at(bo_t, 1e-9);
    S dissolved = raw_total * rs_trial / bo_t;
    split_gas_g(f, p, lift<S>(1.0), sw, lift<S>(0.0), dissolved, base, pr.sg, pr.so, pr.rs);
  }
  pvt_oil_sat_g(f, sat, p, pr.rs, pr.bo, mu);
  pr.bg = sat.bg;
  return pr;
}

// component inventory [water, oil, gas] (properties.rs:157-169)
template <class S>
RF_HD void inventory3(const Fluid& f, double pv_ref, int regime, const S& p, const S& sw, const S& hc, double base,
                      S out[3]) {
  Props3<S> pr = cell_props3(f, regime, p, sw, hc, base);
  S pv = lift<S>(pv_ref) * sexp((p - f.p_rref) * f.c_r);
  out[0] = pv * sw * inv_bw(f, p);
  out[1] = pv * pr.so / floor_at(pr.bo, 1e-9);
  out[2] = pv * pr.sg / floor_at(pr.bg, 1e-9) + out[1] * pr.rs;
}

// face_flux_terms_generic, three-phase (flux.rs:42-191); slots 0-2 cell i, 3-5 cell j for Dual<6>
template <class S>
RF_HD void face_flux3(const Fluid& f, double trans, double depth_i, double depth_j, int reg_i, const S& pi,
                      const S& swi, const S& hci, int reg_j, const S& pj, const S& swj, const S& hcj, S out[3],
                      double base_i = 0.0, double base_j = 0.0) {
  Props3<S> ci = cell_props3(f, reg_i, pi, swi, hci, base_i);
  Props3<S> cj = cell_props3(f, reg_j, pj, swj, hcj, base_j);
  S pcwi = pcow(f, swi), pcwj = pcow(f, swj);
  S pcgi = pc_og(f, ci.sg), pcgj = pc_og(f, cj.sg);
  S gw = lift<S>(0.0), go = lift<S>(0.0), gg = lift<S>(0.0);
  if (f.gravity) {
    const double dz = kGravity * (depth_i - depth_j) * 1e-5;
    S rwi = inv_bw(f, pi) * f.rho_w, rwj = inv_bw(f, pj) * f.rho_w;
    S roi = oil_density3(f, pi, ci.rs), roj = oil_density3(f, pj, cj.rs);
    S rgi = gas_density3(f, pi), rgj = gas_density3(f, pj);
    gw = (rwi + rwj) * 0.5 * dz;
    go = (roi + roj) * 0.5 * dz;
    gg = (rgi + rgj) * 0.5 * dz;
  }
  S dphi_w = (pi - pj) - (pcwi - pcwj) - gw;
  S dphi_o = (pi - pj) - go;
  S dphi_g = (pi - pj) + (pcgi - pcgj) - gg;
  const bool up_w = value(dphi_w) >= 0.0, up_o = value(dphi_o) >= 0.0, up_g = value(dphi_g) >= 0.0;
  // each phase's mobility is evaluated at its upwind cell only (the other cell's is not used)
  const Mob3<S> m_up = up_w ? mobilities3(f, swi, ci.sg, pi, ci.rs) : mobilities3(f, swj, cj.sg, pj, cj.rs);
  Mob3<S> m_other = m_up;
  if (up_o != up_w || up_g != up_w)
    m_other = up_w ? mobilities3(f, swj, cj.sg, pj, cj.rs) : mobilities3(f, swi, ci.sg, pi, ci.rs);
  const S& mob_w = m_up.w;
  const S& mob_o = up_o == up_w ? m_up.o : m_other.o;
  const S& mob_g = up_g == up_w ? m_up.g : m_other.g;
  S p_w = up_w ? pi : pj;
  S bo_o = up_o ? ci.bo : cj.bo;
  S rs_o = up_o ? ci.rs : cj.rs;
  S bg_g = up_g ? ci.bg : cj.bg;
  out[0] = mob_w * dphi_w * trans * inv_bw(f, p_w);
  S qo_res = mob_o * dphi_o * trans;
  S qo = qo_res / floor_at(bo_o, 1e-9);
  S qg_free = mob_g * dphi_g * trans / floor_at(bg_g, 1e-9);
  S qg_dis = qo * rs_o;
  out[1] = qo;
  out[2] = qg_free + qg_dis;
}

// ---------------------------------------------------------------------------------------------
// Wells (fim/wells_ad.rs:44-229)
// ---------------------------------------------------------------------------------------------
template <class S>
struct Frac3 {
  S w, o, g;
};
template <class S>
RF_HD Frac3<S> producer_fractions3(const Fluid& f, const Props3<S>& pr, const S& p, const S& sw) {
  Mob3<S> m = mobilities3(f, sw, pr.sg, p, pr.rs);
  S lw = lift<S>(0.0) + floor_at(m.w, 0.0);
  S lo = lift<S>(0.0) + floor_at(m.o, 0.0);
  S lg = lift<S>(0.0) + floor_at(m.g, 0.0);
  S lt = floor_at(lw + lo + lg, kF64Eps);
  Frac3<S> r;
  r.w = ceil_at(floor_at(lw / lt, 0.0), 1.0);
  r.o = ceil_at(floor_at(lo / lt, 0.0), 1.0);
  r.g = ceil_at(floor_at(lg / lt, 0.0), 1.0);
  return r;
}
template <class S>
RF_HD S connection_rate3(const Fluid& f, double wi, double head, bool injector, int regime, const S& p, const S& sw,
                         const S& hc, const S& bhp, double base = 0.0) {
  Props3<S> pr = cell_props3(f, regime, p, sw, hc, base);
  Mob3<S> m = mobilities3(f, sw, pr.sg, p, pr.rs);
  S cm = floor_at(m.w + m.o + m.g, 0.0);
  S raw = (cm * (p - bhp - lift<S>(head))) * wi;
  if (injector) return value(raw) < 0.0 ? raw : lift<S>(0.0);
  return value(raw) > 0.0 ? raw : lift<S>(0.0);
}
template <class S>
RF_HD void component_coefficients3(const Fluid& f, bool injector, int regime, const S& p, const S& sw, const S& hc,
                                   S out[3], double base = 0.0) {
  Props3<S> pr = cell_props3(f, regime, p, sw, hc, base);
  if (injector) {
    if (f.inject_gas) {
      out[0] = lift<S>(0.0);
      out[1] = lift<S>(0.0);
      out[2] = srecip(floor_at(pr.bg, 1e-9));
      return;
    }
    out[0] = inv_bw(f, p);
    out[1] = lift<S>(0.0);
    out[2] = lift<S>(0.0);
    return;
  }
  Frac3<S> fr = producer_fractions3(f, pr, p, sw);
  S bo = floor_at(pr.bo, 1e-9), bg = floor_at(pr.bg, 1e-9);
  S oc = fr.o / bo;
  out[0] = fr.w * inv_bw(f, p);
  out[1] = oc;
  out[2] = fr.g / bg + oc * pr.rs;
}
template <class S>
RF_HD S surface_rate3(const Fluid& f, bool injector, int regime, const S& p, const S& sw, const S& hc, const S& q,
                      double base = 0.0) {
  Props3<S> pr = cell_props3(f, regime, p, sw, hc, base);
  if (injector) {
    S clamped = floor_at(-q, 0.0);
    if (f.inject_gas) return clamped / floor_at(pr.bg, 1e-9);
    return clamped * inv_bw(f, p);
  }
  Frac3<S> fr = producer_fractions3(f, pr, p, sw);
  return floor_at(q, 0.0) * fr.o / floor_at(pr.bo, 1e-9);
}

}  // namespace rf
