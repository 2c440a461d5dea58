// rf_physics.cuh — two-phase oil-water physics of the fully implicit step, written once as
// __host__ __device__ templates over `double` and the dual number `Dual<N>`.  The host uses the
// double instantiation for the per-well control logic (BHP solve, well relaxation); kernels use
// Dual<3>/Dual<4>/Dual<6> for exact Jacobian blocks.
//
// Reference semantics kept (src/lib/ressim/src/…):
//   fim/ad.rs:21-417           dual arithmetic, value-selected max/min branches
//   fim/properties.rs:37-212   two-phase cell properties and accumulation
//   fim/flux.rs:42-118         face flux with upwinding on the potential's value (dphi >= 0)
//   pvt.rs:603-626,988-1009    PVTW water FVF, base oil FVF and densities
//   relperm.rs:602-629         Corey sampled at equally spaced knots, linear in between
//   capillary.rs:73-97         Brooks-Corey Pc capped at 20x entry pressure
//   fim/wells_ad.rs:44-378     connection rate, producer fractions, component coefficients, FB
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define RF_HD __host__ __device__ __forceinline__
// large bodies that several call sites share (kept out of line on the device to bound code size)
#define RF_HD_CALL __host__ __device__ __noinline__ inline
#else
#define RF_HD inline
#define RF_HD_CALL inline
#endif

namespace rf {

constexpr double kF64Eps = 2.220446049250313080847263336181640625e-16;
constexpr double kDarcy = 8.5269888e-3;  // mD*m^2/(m*cP) -> m^3/day/bar
constexpr double kGravity = 9.80665;
constexpr double kFbEpsilon = 1e-6;
constexpr int kMaxKnots = 64;

// ---------------------------------------------------------------------------------------------
// Dual numbers
// ---------------------------------------------------------------------------------------------
template <int N>
struct Dual {
  double v;
  double d[N];
};

template <int N>
RF_HD Dual<N> dconst(double v) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = 0.0;
  return r;
}
template <int N>
RF_HD Dual<N> dvar(double v, int slot) {
  Dual<N> r = dconst<N>(v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (i == slot) ? 1.0 : 0.0;
  return r;
}
template <int N>
RF_HD Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
RF_HD Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
RF_HD Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
RF_HD Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  const double inv = 1.0 / b.v;
  const double inv2 = inv * inv;
  Dual<N> r;
  r.v = a.v * inv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) * inv2;
  return r;
}
template <int N>
RF_HD Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
RF_HD Dual<N> operator+(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v + b;
  return r;
}
template <int N>
RF_HD Dual<N> operator-(const Dual<N>& a, double b) {
  Dual<N> r = a;
  r.v = a.v - b;
  return r;
}
template <int N>
RF_HD Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
RF_HD Dual<N> operator/(const Dual<N>& a, double b) {
  const double inv = 1.0 / b;
  Dual<N> r;
  r.v = a.v * inv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * inv;
  return r;
}

// scalar helpers over double and Dual<N>
template <class S>
struct Lift;
template <>
struct Lift<double> {
  RF_HD static double c(double v) { return v; }
};
template <int N>
struct Lift<Dual<N>> {
  RF_HD static Dual<N> c(double v) { return dconst<N>(v); }
};
template <class S>
RF_HD S lift(double v) {
  return Lift<S>::c(v);
}
RF_HD double value(double x) { return x; }
template <int N>
RF_HD double value(const Dual<N>& x) {
  return x.v;
}
RF_HD double sexp(double x) { return exp(x); }
RF_HD double spow(double x, double p) { return pow(x, p); }
RF_HD double ssqrt(double x) { return sqrt(x); }
RF_HD double floor_at(double x, double f) { return fmax(x, f); }
RF_HD double ceil_at(double x, double c) { return fmin(x, c); }
RF_HD double smin(double a, double b) { return fmin(a, b); }
template <int N>
RF_HD Dual<N> sexp(const Dual<N>& a) {
  Dual<N> r;
  r.v = exp(a.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * r.v;
  return r;
}
template <int N>
RF_HD Dual<N> spow(const Dual<N>& a, double p) {
  Dual<N> r;
  r.v = pow(a.v, p);
  const double coef = p * pow(a.v, p - 1.0);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * coef;
  return r;
}
template <int N>
RF_HD Dual<N> ssqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = sqrt(a.v);
  const double coef = 0.5 / r.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * coef;
  return r;
}
template <int N>
RF_HD Dual<N> floor_at(const Dual<N>& a, double f) {
  return a.v >= f ? a : dconst<N>(f);
}
template <int N>
RF_HD Dual<N> ceil_at(const Dual<N>& a, double c) {
  return a.v <= c ? a : dconst<N>(c);
}
template <int N>
RF_HD Dual<N> smin(const Dual<N>& a, const Dual<N>& b) {
  return a.v <= b.v ? a : b;
}

// Stencil slot order of a block row: z-, y-, x-, diagonal, x+, y+, z+.  This is also the
// ascending column order, and the order in which the reference's assembly loop adds face terms
// into a cell's rows (faces owned by lower-index neighbours first).
enum { kZm = 0, kYm = 1, kXm = 2, kDiag = 3, kXp = 4, kYp = 5, kZp = 6 };

// Control of one physical well as the assembly kernels read it (fim/wells.rs:691-798).
struct WellControlH {
  int enabled, rate_controlled, uses_surface_target, has_target, injector;
  double target_rate, bhp_limit, bhp_target;
};

// ---------------------------------------------------------------------------------------------
// Fluid / rock / SCAL parameters (plain data, passed by value to kernels)
// ---------------------------------------------------------------------------------------------
struct Fluid {
  double mu_o, mu_w, c_o, c_w, rho_o, rho_w, rho_g;
  double b_o, b_w, p_wref, c_r, p_rref;
  int gravity;
  double s_wc, s_or, n_w, n_o, krw_max, kro_max;
  int table_points;  // > 0: tabulated Corey with this many knots; 0: analytic Corey
  double pc_entry, pc_lambda;
  double knot_lo, knot_hi, knot_step;
  double knot_x[kMaxKnots], knot_krw[kMaxKnots], knot_kro[kMaxKnots];
  // three-phase black-oil mode (rf_blackoil.cuh); zero in two-phase mode
  int three_phase, has_scal3, has_pc_og, inject_gas;
  int drsdt0;  // gas redissolution off: Rs capped at the cell's Rs at the substep start
  double mu_g;
  double s3_wc, s3_or, s3_nw, s3_no, s3_krw, s3_kro, s3_gc, s3_gr, s3_org, s3_ng, s3_krg;
  double pcog_entry, pcog_lambda;
  // PVT table, flat: n_sat saturated rows of (p, rs, bo, mu_o, bg, mu_g); at pvt_hdr one
  // (rs, first row, row count) triple per undersaturated-oil branch; at pvt_rows the branch rows.
  // Device memory in the kernels' copy of this struct, host memory in the host's copy.
  const double* pvt;
  int pvt_n_sat, pvt_n_br, pvt_hdr, pvt_rows;
  double pvt_c_o;
  // SWOF rows (sw, krw, krow) at pvt + swof_off and SGOF rows (sg, krg, krog) at pvt + sgof_off
  // in the same flat array; n_swof = 0: the three-phase Corey curves
  int swof_off, n_swof, sgof_off, n_sgof;
};

// analytic Corey values (relperm.rs:491-520), used to sample the table knots on the host
inline double corey_krw(const Fluid& f, double sw) {
  double e = (sw - f.s_wc) / (1.0 - f.s_wc - f.s_or);
  e = e < 0.0 ? 0.0 : (e > 1.0 ? 1.0 : e);
  return f.krw_max * std::pow(e, f.n_w);
}
inline double corey_kro(const Fluid& f, double sw) {
  double e = (1.0 - sw - f.s_or) / (1.0 - f.s_wc - f.s_or);
  e = e < 0.0 ? 0.0 : (e > 1.0 ? 1.0 : e);
  return f.kro_max * std::pow(e, f.n_o);
}
// Samples the knots once on the host: knot i sits at min(lo + i*step, hi).
inline void fill_knots(Fluid& f) {
  const int pts = f.table_points < 2 ? 2 : f.table_points;
  f.knot_lo = f.s_wc;
  f.knot_hi = 1.0 - f.s_or;
  const double span = (f.knot_hi - f.knot_lo) > 1e-12 ? (f.knot_hi - f.knot_lo) : 1e-12;
  f.knot_step = span / double(pts - 1);
  for (int i = 0; i < pts && i < kMaxKnots; ++i) {
    const double x = std::fmin(f.knot_lo + double(i) * f.knot_step, f.knot_hi);
    f.knot_x[i] = x;
    f.knot_krw[i] = corey_krw(f, x);
    f.knot_kro[i] = corey_kro(f, x);
  }
}

// ---- PVT ----
template <class S>
RF_HD S inv_bw(const Fluid& f, const S& p) {
  S x = (p - f.p_wref) * f.c_w;
  return (lift<S>(1.0) + x * (lift<S>(1.0) + x * 0.5)) / fmax(f.b_w, 1e-9);
}
RF_HD double water_fvf(const Fluid& f, double p) { return 1.0 / fmax(inv_bw(f, p), 1e-9); }
template <class S>
RF_HD S oil_fvf(const Fluid& f, const S& p) {
  return floor_at(lift<S>(f.b_o) * sexp(p * (-f.c_o)), 1e-9);
}
RF_HD double oil_fvf_plain(const Fluid& f, double p) { return fmax(f.b_o * exp(-f.c_o * p), 1e-9); }

// ---- relative permeability ----
template <class S>
RF_HD void relperm(const Fluid& f, const S& sw, S& krw, S& kro) {
  if (f.table_points > 0) {
    const int pts = f.table_points < 2 ? 2 : f.table_points;
    const double v = value(sw);
    if (v <= f.knot_lo) {
      krw = lift<S>(f.knot_krw[0]);
      kro = lift<S>(f.knot_kro[0]);
      return;
    }
    if (v >= f.knot_hi) {
      krw = lift<S>(f.knot_krw[pts - 1]);
      kro = lift<S>(f.knot_kro[pts - 1]);
      return;
    }
    int seg = int(floor((v - f.knot_lo) / f.knot_step));
    if (seg > pts - 2) seg = pts - 2;
    const double x0 = f.knot_x[seg], x1 = f.knot_x[seg + 1];
    S t = ceil_at(floor_at((sw - x0) / (x1 - x0), 0.0), 1.0);
    krw = t * (f.knot_krw[seg + 1] - f.knot_krw[seg]) + f.knot_krw[seg];
    kro = t * (f.knot_kro[seg + 1] - f.knot_kro[seg]) + f.knot_kro[seg];
    return;
  }
  const double denom = 1.0 - f.s_wc - f.s_or;
  S ew = ceil_at(floor_at((sw - f.s_wc) / denom, 0.0), 1.0);
  krw = spow(ew, f.n_w) * f.krw_max;
  S eo = ceil_at(floor_at((lift<S>(1.0 - f.s_or) - sw) / denom, 0.0), 1.0);
  kro = spow(eo, f.n_o) * f.kro_max;
}

template <class S>
struct Mob {
  S w, o;
};
template <class S>
RF_HD Mob<S> mobilities(const Fluid& f, const S& sw) {
  S krw, kro;
  relperm(f, sw, krw, kro);
  Mob<S> m;
  m.w = krw / lift<S>(f.mu_w);
  m.o = kro / lift<S>(f.mu_o);
  return m;
}

// ---- capillary pressure ----
template <class S>
RF_HD S pcow(const Fluid& f, const S& sw) {
  const double denom = 1.0 - f.s_wc - f.s_or;
  S e = ceil_at(floor_at((sw - f.s_wc) / denom, 0.0), 1.0);
  if (value(e) >= 1.0) return lift<S>(0.0);
  const double pc_max = f.pc_entry * 20.0;
  if (value(e) <= 0.0) return lift<S>(pc_max);
  S pc = spow(e, -1.0 / f.pc_lambda) * f.pc_entry;
  return ceil_at(floor_at(pc, 0.0), pc_max);
}

// ---- cell properties and inventory (two-phase: sg from the regularised third unknown) ----
template <class S>
struct Props {
  S so, sg, bo;
};
template <class S>
RF_HD Props<S> cell_props(const Fluid& f, const S& p, const S& sw, const S& hc) {
  const S one = lift<S>(1.0);
  const S total = floor_at(one - sw, 0.0);
  Props<S> r;
  r.sg = smin(floor_at(hc, 0.0), total);
  r.so = floor_at(one - sw - r.sg, 0.0);
  r.bo = oil_fvf(f, p);
  return r;
}

// component inventory [water, oil, gas] (properties.rs:157-169) with rs = 0 and bg = 1
template <class S>
RF_HD void inventory(const Fluid& f, double pv_ref, const S& p, const S& sw, const S& hc, S out[3]) {
  Props<S> pr = cell_props(f, p, sw, hc);
  S pv = lift<S>(pv_ref) * sexp((p - f.p_rref) * f.c_r);
  out[0] = pv * sw * inv_bw(f, p);
  out[1] = pv * pr.so / floor_at(pr.bo, 1e-9);
  out[2] = pv * pr.sg / floor_at(lift<S>(1.0), 1e-9) + out[1] * lift<S>(0.0);
}

// ---- face flux in surface units per day; slots 0-2 cell i, 3-5 cell j when S = Dual<6> ----
template <class S>
RF_HD void face_flux(const Fluid& f, double trans, double depth_i, double depth_j, const S& pi, const S& swi,
                     const S& pj, const S& swj, S out[3]) {
  S pcwi = pcow(f, swi), pcwj = pcow(f, swj);
  S gw = lift<S>(0.0), go = lift<S>(0.0);
  if (f.gravity) {
    S rwi = inv_bw(f, pi) * f.rho_w, rwj = inv_bw(f, pj) * f.rho_w;
    S roi = lift<S>(f.rho_o) / oil_fvf(f, pi), roj = lift<S>(f.rho_o) / oil_fvf(f, pj);
    const double dz = kGravity * (depth_i - depth_j) * 1e-5;
    gw = (rwi + rwj) * 0.5 * dz;
    go = (roi + roj) * 0.5 * dz;
  }
  S dphi_w = (pi - pj) - (pcwi - pcwj) - gw;
  S dphi_o = (pi - pj) - go;
  Mob<S> mi = mobilities(f, swi), mj = mobilities(f, swj);
  const bool up_w = value(dphi_w) >= 0.0, up_o = value(dphi_o) >= 0.0;
  S mob_w = up_w ? mi.w : mj.w;
  S p_w = up_w ? pi : pj;
  S mob_o = up_o ? mi.o : mj.o;
  S bo_o = up_o ? oil_fvf(f, pi) : oil_fvf(f, pj);
  out[0] = mob_w * dphi_w * trans * inv_bw(f, p_w);
  S qo = mob_o * dphi_o * trans;
  out[1] = qo / floor_at(bo_o, 1e-9);
  out[2] = lift<S>(0.0);
}

// ---- wells ----
template <class S>
RF_HD S connection_rate(const Fluid& f, double wi, double head, bool injector, const S& p, const S& sw,
                        const S& bhp) {
  Mob<S> m = mobilities(f, sw);
  S cm = floor_at(m.w + m.o + lift<S>(0.0), 0.0);
  S raw = (cm * (p - bhp - lift<S>(head))) * wi;
  if (injector) return value(raw) < 0.0 ? raw : lift<S>(0.0);
  return value(raw) > 0.0 ? raw : lift<S>(0.0);
}
template <class S>
struct Frac {
  S w, o, g;
};
template <class S>
RF_HD Frac<S> producer_fractions(const Fluid& f, const S& sw) {
  Mob<S> m = mobilities(f, sw);
  S lw = lift<S>(0.0) + floor_at(m.w, 0.0);
  S lo = lift<S>(0.0) + floor_at(m.o, 0.0);
  S lg = lift<S>(0.0) + floor_at(lift<S>(0.0), 0.0);
  S lt = floor_at(lw + lo + lg, kF64Eps);
  Frac<S> r;
  r.w = ceil_at(floor_at(lw / lt, 0.0), 1.0);
  r.o = ceil_at(floor_at(lo / lt, 0.0), 1.0);
  r.g = ceil_at(floor_at(lg / lt, 0.0), 1.0);
  return r;
}
template <class S>
RF_HD void component_coefficients(const Fluid& f, bool injector, const S& p, const S& sw, const S& hc,
                                  S out[3]) {
  if (injector) {
    out[0] = inv_bw(f, p);
    out[1] = lift<S>(0.0);
    out[2] = lift<S>(0.0);
    return;
  }
  Frac<S> fr = producer_fractions(f, sw);
  Props<S> pr = cell_props(f, p, sw, hc);
  S bo = floor_at(pr.bo, 1e-9), bg = floor_at(lift<S>(1.0), 1e-9);
  S oc = fr.o / bo;
  out[0] = fr.w * inv_bw(f, p);
  out[1] = oc;
  out[2] = fr.g / bg + oc * lift<S>(0.0);
}
template <class S>
RF_HD S surface_rate(const Fluid& f, bool injector, const S& p, const S& sw, const S& hc, const S& q) {
  if (injector) return floor_at(-q, 0.0) * inv_bw(f, p);
  Frac<S> fr = producer_fractions(f, sw);
  Props<S> pr = cell_props(f, p, sw, hc);
  return floor_at(q, 0.0) * fr.o / floor_at(pr.bo, 1e-9);
}
template <class S>
RF_HD S reservoir_rate(bool injector, const S& q) {
  return injector ? floor_at(-q, 0.0) : floor_at(q, 0.0);
}
RF_HD void fb_gradient(double a, double b, double& da, double& db) {
  const double n = sqrt(a * a + b * b + 2.0 * kFbEpsilon * kFbEpsilon);
  da = a / n - 1.0;
  db = b / n - 1.0;
}
RF_HD double fischer_burmeister(double a, double b) {
  const double e = 2.0 * kFbEpsilon * kFbEpsilon;
  return sqrt((a * a + b * b) + e) - a - b;
}

}  // namespace rf
