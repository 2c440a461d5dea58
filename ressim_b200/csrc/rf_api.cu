// rf_api.cu — host control of the device FIM path and the C ABI (include/ressim_fim.h).
//
// The control flow mirrors the reference's OPM-aligned production path:
//   outer controller  fim/timestep.rs:989-1848  (trial dt, 0.33 restart factor, 16 retries,
//                                                PID + iteration-count growth)
//   Newton attempt    fim/newton.rs:970-3360    (CNV/MB acceptance from the third residual
//                                                evaluation on, relaxed linear acceptance below
//                                                0.01 reduction, oscillation relaxation, per-cell
//                                                chop, raw saturations)
//   wells             fim/state.rs:109-177, 433-553 and fim/wells.rs:389-504, 737-798
//                     (initial BHP from the rate target, control bounds, relaxation toward local
//                     consistency), evaluated on the host from the perforated cells' state
// All per-cell work (assembly, norms, linear solve, update, reductions) runs on the device; the
// host only reads scalars and the perforated cells' state.
#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <atomic>
#include <mutex>
#include <thread>
#include <tuple>

#include "rf_blackoil.cuh"
#include "rf_fiber.hpp"
#include "rf_fluid.hpp"
#include "rf_ops.hpp"
#include "rf_state.hpp"

namespace rf {

// ---------------------------------------------------------------------------------------------
// wells on the host
// ---------------------------------------------------------------------------------------------
static WellControlH well_control(const Ctx& c, int w) {
  const RfWell& rep = c.wells[c.topo.well_rep[w]];
  const bool inj = c.topo.well_inj[w] != 0;
  const bool expl = rep.has_schedule && (rep.schedule_control != 0 || !std::isnan(rep.schedule_target_rate) ||
                                         !std::isnan(rep.schedule_target_surface_rate) ||
                                         !std::isnan(rep.schedule_bhp_limit) || !rep.schedule_enabled);
  WellControlH k{};
  k.injector = inj;
  k.enabled = expl ? rep.schedule_enabled != 0 : (inj ? c.inj_enabled : 1);
  const int fam_rate = inj ? (c.inj_rate_ctl && c.inj_enabled) : c.prod_rate_ctl;
  k.rate_controlled = !k.enabled ? 0 : (expl ? rep.schedule_control == 2 : fam_rate);
  k.uses_surface_target =
      expl ? !std::isnan(rep.schedule_target_surface_rate) : !std::isnan(inj ? c.tgt_inj_surf : c.tgt_prod_surf);
  k.has_target = 0;
  k.target_rate = 0.0;
  if (k.rate_controlled) {
    if (expl) {
      const double t = !std::isnan(rep.schedule_target_surface_rate)
                           ? rep.schedule_target_surface_rate
                           : (!std::isnan(rep.schedule_target_rate) ? rep.schedule_target_rate : 0.0);
      k.has_target = 1;
      k.target_rate = fmax(t, 0.0);
    } else if (fam_rate) {
      const double t = inj ? (!std::isnan(c.tgt_inj_surf) ? c.tgt_inj_surf : c.tgt_inj)
                           : (!std::isnan(c.tgt_prod_surf) ? c.tgt_prod_surf : c.tgt_prod);
      k.has_target = 1;
      k.target_rate = fmax(t, 0.0);
    }
  }
  const double fam_limit = inj ? c.bhp_max : c.bhp_min;
  k.bhp_limit = expl ? (!std::isnan(rep.schedule_bhp_limit) ? rep.schedule_bhp_limit : fam_limit) : fam_limit;
  k.bhp_target = rep.bhp;
  return k;
}

// perforated-cell state, 3 doubles per perforation (p, sw, hc), and the regimes (three-phase)
struct PerfCells {
  std::vector<double> v;
  std::vector<int> reg;
  std::vector<double> rs0;  // gas redissolution off: the cell's Rs at the substep start (the cap)
  double p(int k) const { return v[3 * k]; }
  double sw(int k) const { return v[3 * k + 1]; }
  double hc(int k) const { return v[3 * k + 2]; }
  int regime(int k) const { return reg.empty() ? 0 : reg[k]; }
  double base(int k) const { return rs0.empty() ? 0.0 : rs0[k]; }
};

static void gather_perf(Ctx& c, const double* p, const double* sw, const double* hc, PerfCells& pc) {
  if (!c.fluid.three_phase) {
    gather_perf_cells(c, p, sw, hc, pc.v);
    pc.reg.clear();
    return;
  }
  std::vector<double> t;
  gather_perf_cells3(c, p, sw, hc, c.d_reg.p, t);
  const int P = c.topo.n_perfs;
  pc.v.resize(3 * size_t(P));
  pc.reg.resize(P);
  for (int k = 0; k < P; ++k) {
    for (int e = 0; e < 3; ++e) pc.v[3 * k + e] = t[4 * k + e];
    pc.reg[k] = int(t[4 * k + 3]);
  }
  pc.rs0.clear();
  if (c.fluid.drsdt0) {
    gather_perf_cells3(c, c.d_rs.p, c.d_rs.p, c.d_rs.p, nullptr, t);
    pc.rs0.resize(P);
    for (int k = 0; k < P; ++k) pc.rs0[k] = t[4 * k];
  }
}

// producer_control_state (fim/wells.rs:834-859), three-phase
struct ProducerState3 {
  double wf, of, gf, bo, bg, rs;
};
static ProducerState3 producer_state3(const Fluid& f, double p, double sw, const Derived3& d) {
  const Mob3<double> m = mobilities3_f64(f, sw, d.sg, p, d.rs);
  const double lw = fmax(m.w, 0.0), lo = fmax(m.o, 0.0), lg = fmax(m.g, 0.0);
  const double lt = fmax(lw + lo + lg, kF64Eps);
  ProducerState3 s;
  s.wf = clamp01(lw / lt, 0.0, 1.0);
  s.of = clamp01(lo / lt, 0.0, 1.0);
  s.gf = clamp01(lg / lt, 0.0, 1.0);
  s.bo = fmax(d.bo, 1e-9);
  s.bg = fmax(d.bg, 1e-9);
  s.rs = fmax(d.rs, 0.0);
  return s;
}

static bool connection_rate_for_bhp(const Ctx& c, const PerfCells& pc, int k, double bhp, double& q) {
  if (c.fluid.three_phase) {
    // fim/wells.rs:1098-1129 with the cell's flashed Sg and Rs
    const Fluid& f = c.hfluid;
    const Derived3 d = derive_cell3(f, pc.p(k), pc.sw(k), pc.hc(k), pc.regime(k), pc.base(k));
    const Mob3<double> m = mobilities3_f64(f, pc.sw(k), d.sg, pc.p(k), d.rs);
    if (!c.topo.perf_has_wi[k]) return false;
    const double mob = fmax(m.w + m.o + m.g, 0.0);
    const double raw = c.topo.perf_wi[k] * mob * (pc.p(k) - (bhp + c.head_offset[c.topo.perf_entry[k]]));
    if (!std::isfinite(raw)) return false;
    q = c.topo.perf_inj[k] ? fmin(raw, 0.0) : fmax(raw, 0.0);
    return true;
  }
  Mob<double> m = mobilities<double>(c.fluid, pc.sw(k));
  if (!c.topo.perf_has_wi[k]) return false;
  const double mob = fmax(m.w + m.o + 0.0, 0.0);
  const double raw = c.topo.perf_wi[k] * mob * (pc.p(k) - (bhp + c.head_offset[c.topo.perf_entry[k]]));
  if (!std::isfinite(raw)) return false;
  q = c.topo.perf_inj[k] ? fmin(raw, 0.0) : fmax(raw, 0.0);
  return true;
}

static double surface_rate_sc(const Ctx& c, const PerfCells& pc, int k, double q) {
  if (c.fluid.three_phase) {
    // perforation_surface_rate_sc_day (fim/wells.rs:1147-1170)
    const Fluid& f = c.hfluid;
    const Derived3 d = derive_cell3(f, pc.p(k), pc.sw(k), pc.hc(k), pc.regime(k), pc.base(k));
    if (c.topo.perf_inj[k]) {
      if (f.inject_gas) return fmax(-q, 0.0) / fmax(d.bg, 1e-9);
      return fmax(-q, 0.0) * inv_bw(f, pc.p(k));
    }
    const ProducerState3 ps = producer_state3(f, pc.p(k), pc.sw(k), d);
    return fmax(q, 0.0) * ps.of / fmax(ps.bo, 1e-9);
  }
  if (c.topo.perf_inj[k]) return fmax(-q, 0.0) * inv_bw(c.fluid, pc.p(k));
  Mob<double> m = mobilities<double>(c.fluid, pc.sw(k));
  const double lw = fmax(m.w, 0.0), lo = fmax(m.o, 0.0), lg = 0.0;
  const double lt = fmax(lw + lo + lg, kF64Eps);
  const double of = fmin(fmax(lo / lt, 0.0), 1.0);
  const double bo = fmax(oil_fvf_plain(c.fluid, pc.p(k)), 1e-9);
  return fmax(q, 0.0) * of / fmax(bo, 1e-9);
}

static double total_rate_for_bhp(const Ctx& c, const PerfCells& pc, int w, const WellControlH& k, double bhp) {
  double total = 0.0;
  for (int a = c.topo.well_ptr[w]; a < c.topo.well_ptr[w + 1]; ++a) {
    const int perf = c.topo.well_perfs[a];
    double q;
    if (!connection_rate_for_bhp(c, pc, perf, bhp, q)) continue;
    if (k.uses_surface_target)
      total += surface_rate_sc(c, pc, perf, q);
    else
      total += k.injector ? fmax(-q, 0.0) : fmax(q, 0.0);
  }
  return total;
}

static bool solve_bhp_from_target(const Ctx& c, const PerfCells& pc, int w, double& out) {
  const WellControlH k = well_control(c, w);
  if (!k.enabled || !k.rate_controlled) return false;
  const int a0 = c.topo.well_ptr[w], a1 = c.topo.well_ptr[w + 1];
  if (a0 == a1 || !k.has_target) return false;
  double minp = INFINITY, maxp = -INFINITY;
  for (int a = a0; a < a1; ++a) {
    const int perf = c.topo.well_perfs[a];
    const double z = pc.p(perf) - c.head_offset[c.topo.perf_entry[perf]];
    minp = fmin(minp, z);
    maxp = fmax(maxp, z);
  }
  if (!std::isfinite(minp) || !std::isfinite(maxp)) return false;
  const double target = k.target_rate, limit = k.bhp_limit;
  if (target >= total_rate_for_bhp(c, pc, w, k, limit) - 1e-9) {
    out = limit;
    return true;
  }
  if (k.injector) {
    double lo = fmin(minp, limit), hi = limit;
    for (int it = 0; it < 64; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (total_rate_for_bhp(c, pc, w, k, mid) < target)
        lo = mid;
      else
        hi = mid;
    }
    out = 0.5 * (lo + hi);
  } else {
    double lo = limit, hi = fmax(maxp, limit);
    for (int it = 0; it < 64; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (total_rate_for_bhp(c, pc, w, k, mid) > target)
        lo = mid;
      else
        hi = mid;
    }
    out = 0.5 * (lo + hi);
  }
  return true;
}

static void enforce_control_bounds(const Ctx& c, double pmax, std::vector<double>& bhp) {
  const double pu = fmax(fmax(c.bhp_max, 1.0), pmax) + 500.0;
  for (int w = 0; w < c.topo.n_wells; ++w) {
    const WellControlH k = well_control(c, w);
    double lo, hi;
    if (k.injector) {
      lo = 1e-6;
      hi = fmax(pu, fmax(k.bhp_limit, c.bhp_max));
    } else {
      lo = fmax(fmin(k.bhp_limit, c.bhp_min), 1e-6);
      hi = pu;
    }
    double b = bhp[w];
    if (b < lo) b = lo;
    if (b > hi) b = hi;
    bhp[w] = b;
  }
}

static void relax_wells(const Ctx& c, const PerfCells& pc, std::vector<double>& bhp, std::vector<double>& q) {
  for (int w = 0; w < c.topo.n_wells; ++w) {
    const WellControlH k = well_control(c, w);
    double cons = k.bhp_target;
    bool have = true;
    if (k.enabled && k.rate_controlled) have = solve_bhp_from_target(c, pc, w, cons);
    if (!have) continue;
    const double prop = bhp[w];
    const double bl = prop + 0.9 * (cons - prop);
    double d = bl - cons;
    d = d < -25.0 ? -25.0 : (d > 25.0 ? 25.0 : d);
    bhp[w] = fmax(cons + d, 1e-6);
    for (int a = c.topo.well_ptr[w]; a < c.topo.well_ptr[w + 1]; ++a) {
      const int perf = c.topo.well_perfs[a];
      double cq = 0.0;
      if (k.enabled && !connection_rate_for_bhp(c, pc, perf, bhp[w], cq)) cq = 0.0;
      const double pq = q[perf];
      const double bq = pq + 0.75 * (cq - pq);
      const double tr = fmax(0.1 * fabs(cq), 250.0);
      double dq = bq - cq;
      dq = dq < -tr ? -tr : (dq > tr ? tr : dq);
      const double qn = cq + dq;
      q[perf] = !k.enabled ? 0.0 : (k.injector ? fmin(qn, 0.0) : fmax(qn, 0.0));
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Newton attempt
// ---------------------------------------------------------------------------------------------
struct WellState {
  std::vector<double> bhp, q;
};
struct NewtonReport {
  bool converged = false;
  int newton_iterations = 0, linear_solves = 0, linear_iterations = 0;
};

struct FamNorms {
  double w = INFINITY, o = INFINITY, g = INFINITY, well = INFINITY, perf = INFINITY;
};
static bool family_osc(double f0, double f1, double f2) {
  if (!(std::isfinite(f0) && std::isfinite(f1) && std::isfinite(f2)) || f0 <= 0.0) return false;
  const double d1 = fabs(f0 - f2) / f0, d2 = fabs(f0 - f1) / f0;
  return d1 < 0.2 && 0.2 < d2;
}

struct CnvMb {
  bool accept;
};
static bool cnv_mb_accept(const double* st, int n, bool final_it, double cnv_tol = 0.0, double mb_tol = 0.0) {
  // st: [0..2] family maxima, [3..5] FVF sums, [6..8] max |r|/pv, [9..11] residual sums,
  // [12] pore-volume sum, [13] violating pore volume
  const double nn = double(n > 0 ? n : 1);
  const double bavg[3] = {st[3] / nn, st[4] / nn, st[5] / nn};
  double cnv[3], mb[3];
  for (int k = 0; k < 3; ++k) {
    cnv[k] = bavg[k] * st[6 + k];
    mb[k] = fabs(bavg[k] * st[9 + k]) / fmax(st[12], 1e-9);
  }
  bool pv_relax = st[13] < 0.03 * st[12];
  double mbt = final_it ? 1e-6 : 1e-7, cnvt = final_it ? 1.0 : 1e-2;
  if (cnv_tol > 0.0) {  // controller option: fixed tolerances, no relaxed tiers
    cnvt = cnv_tol;
    mbt = mb_tol > 0.0 ? mb_tol : mbt;
    pv_relax = false;
  }
  bool ok = true;
  for (int k = 0; k < 3; ++k) ok = ok && (cnv[k] <= cnvt || (pv_relax && cnv[k] <= 1.0)) && mb[k] <= mbt;
  return ok;
}

static void upload_wells(Ctx& c, const WellState& ws) {
  if (c.topo.n_wells)
    RF_CUDA(cudaMemcpyAsync(c.d_bhp.p, ws.bhp.data(), sizeof(double) * c.topo.n_wells, cudaMemcpyHostToDevice, c.stream));
  if (c.topo.n_perfs)
    RF_CUDA(cudaMemcpyAsync(c.d_q.p, ws.q.data(), sizeof(double) * c.topo.n_perfs, cudaMemcpyHostToDevice, c.stream));
}

static void tail_norms(Ctx& c, const WellState& ws, FamNorms& fam) {
  const int W = c.topo.n_wells, P = c.topo.n_perfs;
  if (W + P == 0) return;
  std::vector<double> rt(W + P);
  d2h(c, rt.data(), c.d_res_tail.p, sizeof(double) * rt.size());
  d2h_wait(c);
  double fw = 0.0, fp = 0.0;
  for (int w = 0; w < W; ++w) {
    const WellControlH k = well_control(c, w);
    const double scale = (k.enabled && k.rate_controlled && k.has_target) ? 1.0 : fmax(fabs(ws.bhp[w]), 1.0);
    fw = fmax(fw, fabs(rt[w]) / scale);
  }
  for (int p = 0; p < P; ++p) fp = fmax(fp, fabs(rt[W + p]) / fmax(fabs(ws.q[p]), 1.0));
  fam.well = W ? fw : INFINITY;
  fam.perf = P ? fp : INFINITY;
}

static void upload_controls(Ctx& c) {
  const int W = c.topo.n_wells;
  if (!W) return;
  std::vector<WellControlH> k(W);
  for (int w = 0; w < W; ++w) k[w] = well_control(c, w);
  RF_CUDA(cudaMemcpyAsync(c.d_ctrl.p, k.data(), sizeof(WellControlH) * W, cudaMemcpyHostToDevice, c.stream));
  stream_wait(c);
}

static void swap_state(Ctx& c) {
  std::swap(c.d_p, c.d_cp);
  std::swap(c.d_sw, c.d_csw);
  std::swap(c.d_hc, c.d_chc);
}

// run_fim_timestep: the iterate starts from the substep start state held in (d_pp, d_psw, d_phc)
static NewtonReport run_newton(Ctx& c, WellState& ws, double dt) {
  NewtonReport rep;
  const size_t nb = sizeof(double) * c.n;
  RF_CUDA(cudaMemcpyAsync(c.d_p.p, c.d_pp.p, nb, cudaMemcpyDeviceToDevice, c.stream));
  RF_CUDA(cudaMemcpyAsync(c.d_sw.p, c.d_psw.p, nb, cudaMemcpyDeviceToDevice, c.stream));
  RF_CUDA(cudaMemcpyAsync(c.d_hc.p, c.d_phc.p, nb, cudaMemcpyDeviceToDevice, c.stream));
  upload_controls(c);
  FamNorms n1, n2;
  double relax = 1.0;
  const int max_it = 20;
  double st[kNormQuantities + 1];
  std::vector<double> dx_tail;
  PerfCells pc;
  for (int it = 0; it < max_it; ++it) {
    {
      PhaseScope ps(c, kPhAssembly);
      upload_wells(c, ws);
      launch_assembly(c, dt);
      launch_norms(c, dt, st);
    }
    FamNorms fam;
    fam.w = st[0];
    fam.o = st[1];
    fam.g = st[2];
    tail_norms(c, ws, fam);
    const int osc = int(family_osc(fam.w, n1.w, n2.w)) + int(family_osc(fam.o, n1.o, n2.o)) +
                    int(family_osc(fam.g, n1.g, n2.g)) + int(family_osc(fam.well, n1.well, n2.well)) +
                    int(family_osc(fam.perf, n1.perf, n2.perf));
    if (osc >= 1) relax = fmax(relax - 0.1, 0.5);
    n2 = n1;
    n1 = fam;
    const bool final_it = it + 1 == max_it;
    if (it >= 2 && cnv_mb_accept(st, c.n, final_it, c.ctl_cnv, c.ctl_mb)) {
      rep.converged = true;
      rep.newton_iterations = it + 1;
      return rep;
    }
    LinResult lin = linear_solve_full(c, dx_tail);
    rep.linear_solves++;
    rep.linear_iterations += lin.iterations;
    if (!lin.converged || !lin.finite) {
      const double red = lin.final_residual_norm / fmax(lin.rhs_norm, 1e-30);
      const bool relaxed = lin.finite && std::isfinite(red) && red < 0.01;
      if (!relaxed) {
        rep.converged = false;
        rep.newton_iterations = it + 1;
        return rep;
      }
    }
    // wells: relaxed + chopped update of BHP (dbhp-max-rel 1.0, floor 1 bar) and rates
    PhaseScope ps_update(c, kPhUpdate);
    const int W = c.topo.n_wells, P = c.topo.n_perfs;
    WellState cand = ws;
    for (int w = 0; w < W; ++w) {
      const double b = ws.bhp[w];
      const double d = dx_tail[w] * relax;
      const double cap = 1.0 * fabs(b);
      const double lim = fabs(d) > cap ? copysign(1.0, d) * cap : d;
      const double ch = (b + lim < 1.0) ? 1.0 - b : lim;
      cand.bhp[w] = b + 1.0 * ch;
    }
    for (int p = 0; p < P; ++p) cand.q[p] = ws.q[p] + 1.0 * (dx_tail[W + p] * relax);
    double pmax;
    bool finite;
    if (c.fluid.three_phase)
      apply_cell_update3(c, relax, pmax, finite);
    else
      apply_cell_update(c, relax, pmax, finite);
    enforce_control_bounds(c, pmax, cand.bhp);
    gather_perf(c, c.d_cp.p, c.d_csw.p, c.d_chc.p, pc);
    relax_wells(c, pc, cand.bhp, cand.q);
    enforce_control_bounds(c, pmax, cand.bhp);
    for (double v : cand.bhp) finite = finite && std::isfinite(v);
    for (double v : cand.q) finite = finite && std::isfinite(v);
    if (!finite) {
      rep.converged = false;
      rep.newton_iterations = it + 1;
      return rep;
    }
    swap_state(c);
    ws = cand;
  }
  upload_wells(c, ws);
  launch_assembly(c, dt);
  launch_norms(c, dt, st);
  rep.newton_iterations = max_it;
  rep.converged = cnv_mb_accept(st, c.n, true, c.ctl_cnv, c.ctl_mb);
  return rep;
}

// ---------------------------------------------------------------------------------------------
// outer controller
// ---------------------------------------------------------------------------------------------
static double pid_dt(double dt, const double e[3]) {
  const double tol = 0.1;
  if (e[2] > tol) return dt * tol / e[2];
  if (e[0] == 0.0 || e[1] == 0.0 || e[2] == 0.0) return std::numeric_limits<double>::max();
  return dt * pow(e[1] / e[2], 0.075) * pow(tol / e[2], 0.175) * pow(e[1] * e[1] / (e[0] * e[2]), 0.01);
}
static double iteration_dt(double dt, int its) {
  const double x = double(its), t = 8.0;
  if (x > t) return dt / (1.0 + (x - t) / t * 1.0);
  return dt * (1.0 + (t - x) / t * 3.2);
}
static double growth_factor(double dt, int its, const double e[3], int retries) {
  double f = 3.0;
  const double fp = pid_dt(dt, e) / dt, fi = iteration_dt(dt, its) / dt;
  if (fp < f) f = fp;
  if (fi < f) f = fi;
  if (retries > 0 && 2.0 < f) f = 2.0;
  return f;
}

static WellState initial_well_state(Ctx& c) {
  WellState ws;
  const int W = c.topo.n_wells, P = c.topo.n_perfs;
  ws.bhp.resize(W);
  ws.q.assign(P, 0.0);
  for (int w = 0; w < W; ++w) ws.bhp[w] = well_control(c, w).bhp_target;
  PerfCells pc;
  gather_perf(c, c.d_pp.p, c.d_psw.p, c.d_phc.p, pc);
  for (int w = 0; w < W; ++w) {
    double b;
    if (solve_bhp_from_target(c, pc, w, b)) ws.bhp[w] = b;
  }
  for (int p = 0; p < P; ++p) {
    const int w = c.topo.perf_well[p];
    double q = 0.0;
    if (well_control(c, w).enabled) {
      if (!connection_rate_for_bhp(c, pc, p, ws.bhp[w], q)) q = 0.0;
    }
    ws.q[p] = q;
  }
  return ws;
}

static void record_step(Ctx& c, const WellState& ws, double dt, double water_change, double oil_removed,
                        const double sums[7]) {
  PerfCells pc;
  gather_perf_cells(c, c.d_p.p, c.d_sw.p, c.d_hc.p, pc.v);
  double prod_oil = 0, prod_liq = 0, prod_liq_res = 0, inj = 0, inj_res = 0, winj_res = 0, pwat_res = 0, winj_sc = 0,
         pwat_sc = 0;
  int prc = 0, irc = 0, pbl = 0, ibl = 0;
  for (int w = 0; w < c.topo.n_wells; ++w) {
    const WellControlH k = well_control(c, w);
    if (k.enabled && k.rate_controlled) {
      const double b = ws.bhp[w];
      const bool lim = k.injector ? b >= k.bhp_limit - 1e-6 : b <= k.bhp_limit + 1e-6;
      if (k.injector) {
        irc++;
        ibl += lim;
      } else {
        prc++;
        pbl += lim;
      }
    }
  }
  for (int p = 0; p < c.topo.n_perfs; ++p) {
    const double q = ws.q[p];
    if (c.topo.perf_inj[p]) {
      const double c0 = q * inv_bw(c.fluid, pc.p(p));
      inj_res += fmax(-q, 0.0);
      inj += fmax(-c0, 0.0);
      winj_res += fmax(-q, 0.0);
      winj_sc += fmax(-c0, 0.0);
      continue;
    }
    Mob<double> m = mobilities<double>(c.fluid, pc.sw(p));
    const double lw = fmax(m.w, 0.0), lo = fmax(m.o, 0.0);
    const double lt = fmax(lw + lo + 0.0, kF64Eps);
    const double wf = fmin(fmax(lw / lt, 0.0), 1.0), of = fmin(fmax(lo / lt, 0.0), 1.0);
    const double bo = fmax(oil_fvf_plain(c.fluid, pc.p(p)), 1e-9);
    const double c0 = q * wf * inv_bw(c.fluid, pc.p(p));
    const double c1 = q * of / fmax(bo, 1e-9);
    prod_liq_res += fmax(q, 0.0);
    pwat_res += fmax(q, 0.0) * wf;
    pwat_sc += fmax(c0, 0.0);
    prod_oil += fmax(c1, 0.0);
    prod_liq += fmax(c0, 0.0) + fmax(c1, 0.0);
  }
  c.cum_inj += winj_res * dt;
  c.cum_prod += pwat_res * dt;
  c.cum_mb += (winj_sc - pwat_sc) * dt - water_change;
  c.cum_mb_oil += prod_oil * dt - oil_removed;
  RfTimePointRates r{};
  r.time = c.time_days + dt;
  r.total_production_oil = prod_oil;
  r.total_production_liquid = prod_liq;
  r.total_production_liquid_reservoir = prod_liq_res;
  r.total_injection = inj;
  r.total_injection_reservoir = inj_res;
  r.material_balance_error_m3 = fabs(c.cum_mb);
  r.material_balance_error_oil_m3 = fabs(c.cum_mb_oil);
  r.avg_reservoir_pressure = sums[5] > 0.0 ? sums[4] / sums[5] : 0.0;
  r.avg_water_saturation = c.n > 0 ? sums[6] / c.n : 0.0;
  r.producer_bhp_limited_fraction = prc > 0 ? double(pbl) / prc : 0.0;
  r.injector_bhp_limited_fraction = irc > 0 ? double(ibl) / irc : 0.0;
  c.rate_history.push_back(r);
}

// record_fim_step_report, three-phase (reporting.rs:553-734, fim/wells.rs:1634-1667): injector
// surface rates of water or gas, producer component rates from the flashed cell state, the gas
// ledger and the producing GOR.  sums: state_sums3 over the written-back state.
static void record_step3(Ctx& c, const WellState& ws, double dt, double water_change, double oil_removed,
                         double gas_change, const double sums[kStateQ3]) {
  const Fluid& f = c.hfluid;
  PerfCells pc;
  gather_perf(c, c.d_p.p, c.d_sw.p, c.d_hc.p, pc);
  double prod_oil = 0, prod_liq = 0, prod_liq_res = 0, inj = 0, inj_res = 0, winj_res = 0, pwat_res = 0, winj_sc = 0,
         pwat_sc = 0, prod_gas = 0, ginj_sc = 0;
  int prc = 0, irc = 0, pbl = 0, ibl = 0;
  for (int w = 0; w < c.topo.n_wells; ++w) {
    const WellControlH k = well_control(c, w);
    if (k.enabled && k.rate_controlled) {
      const double b = ws.bhp[w];
      const bool lim = k.injector ? b >= k.bhp_limit - 1e-6 : b <= k.bhp_limit + 1e-6;
      if (k.injector) {
        irc++;
        ibl += lim;
      } else {
        prc++;
        pbl += lim;
      }
    }
  }
  for (int p = 0; p < c.topo.n_perfs; ++p) {
    const double q = ws.q[p];
    const Derived3 d = derive_cell3(f, pc.p(p), pc.sw(p), pc.hc(p), pc.regime(p), pc.base(p));
    if (c.topo.perf_inj[p]) {
      inj_res += fmax(-q, 0.0);
      if (f.inject_gas) {
        const double c2 = q / fmax(d.bg, 1e-9);
        inj += fmax(-c2, 0.0);
        ginj_sc += fmax(-c2, 0.0);
        continue;
      }
      const double c0 = q * inv_bw(f, pc.p(p));
      inj += fmax(-c0, 0.0);
      winj_res += fmax(-q, 0.0);
      winj_sc += fmax(-c0, 0.0);
      continue;
    }
    const ProducerState3 ps = producer_state3(f, pc.p(p), pc.sw(p), d);
    const double c0 = q * ps.wf * inv_bw(f, pc.p(p));
    const double c1 = q * ps.of / fmax(ps.bo, 1e-9);
    const double c2 = q * ps.gf / fmax(ps.bg, 1e-9) + c1 * ps.rs;
    prod_gas += fmax(c2, 0.0);
    prod_liq_res += fmax(q, 0.0);
    pwat_res += fmax(q, 0.0) * ps.wf;
    pwat_sc += fmax(c0, 0.0);
    prod_oil += fmax(c1, 0.0);
    prod_liq += fmax(c0, 0.0) + fmax(c1, 0.0);
  }
  c.cum_inj += winj_res * dt;
  c.cum_prod += pwat_res * dt;
  c.cum_mb += (winj_sc - pwat_sc) * dt - water_change;
  c.cum_mb_oil += prod_oil * dt - oil_removed;
  c.cum_mb_gas += (ginj_sc - prod_gas) * dt - gas_change;
  RfTimePointRates r{};
  r.time = c.time_days + dt;
  r.total_production_oil = prod_oil;
  r.total_production_liquid = prod_liq;
  r.total_production_liquid_reservoir = prod_liq_res;
  r.total_injection = inj;
  r.total_injection_reservoir = inj_res;
  r.material_balance_error_m3 = fabs(c.cum_mb);
  r.material_balance_error_oil_m3 = fabs(c.cum_mb_oil);
  r.avg_reservoir_pressure = sums[6] > 0.0 ? sums[5] / sums[6] : 0.0;
  r.avg_water_saturation = c.n > 0 ? sums[7] / c.n : 0.0;
  r.producer_bhp_limited_fraction = prc > 0 ? double(pbl) / prc : 0.0;
  r.injector_bhp_limited_fraction = irc > 0 ? double(ibl) / irc : 0.0;
  r.total_production_gas = prod_gas;
  r.avg_gas_saturation = c.n > 0 ? sums[8] / c.n : 0.0;
  r.material_balance_error_gas_m3 = fabs(c.cum_mb_gas);
  r.producing_gor = prod_oil > 1e-9 ? prod_gas / prod_oil : 0.0;
  c.rate_history.push_back(r);
}

// refresh_well_head_offsets (well_control.rs:192-276), on the state entering a report step: each
// completion's head carries its physical well's datum BHP along the wellbore, density * g *
// (depth(k) - datum) * 1e-5 bar.  Datum: the group's first explicit datum_depth_m, else its
// shallowest completion.  Density: the first explicit wellbore_density_kg_m3, else the mean over
// the group of the water density (injector) or the mobility-weighted mixture density (producer,
// analytic Corey at the completion cell's state), each at the cell's pressure.  The per-completion
// heads are copied to the device for the connection rows.
static void refresh_head_offsets(Ctx& c) {
  const Topology& t = c.topo;
  c.head_offset.assign(c.wells.size(), 0.0);
  if (c.fluid.gravity && t.n_perfs > 0) {
    PerfCells pc;
    std::vector<double> sg_rs;  // three-phase: the simulator's (Sg, Rs, -, -) per perforation
    if (c.fluid.three_phase) {
      std::vector<double> a;
      gather_perf_cells3(c, c.d_p.p, c.d_sw.p, c.d_sg.p, nullptr, a);
      gather_perf_cells3(c, c.d_rs.p, c.d_rs.p, c.d_rs.p, nullptr, sg_rs);
      pc.v.resize(3 * size_t(t.n_perfs));
      for (int k = 0; k < t.n_perfs; ++k) {
        pc.v[3 * k] = a[4 * k];
        pc.v[3 * k + 1] = a[4 * k + 1];
        pc.v[3 * k + 2] = 0.0;
        sg_rs[4 * k + 1] = sg_rs[4 * k];  // Rs
        sg_rs[4 * k] = a[4 * k + 2];      // Sg
      }
    } else {
      gather_perf_cells(c, c.d_p.p, c.d_sw.p, c.d_hc.p, pc.v);
    }
    const Fluid& f = c.fluid.three_phase ? c.hfluid : c.fluid;
    for (int w = 0; w < t.n_wells; ++w) {
      double datum = NAN, density = NAN;
      for (int q = t.well_ptr[w]; q < t.well_ptr[w + 1]; ++q) {
        const double d = c.wells[t.perf_entry[t.well_perfs[q]]].datum_depth_m;
        if (std::isfinite(d)) {
          datum = d;
          break;
        }
      }
      if (!std::isfinite(datum)) {
        datum = INFINITY;
        for (int q = t.well_ptr[w]; q < t.well_ptr[w + 1]; ++q)
          datum = fmin(datum, c.depth_layer[c.wells[t.perf_entry[t.well_perfs[q]]].k]);
      }
      for (int q = t.well_ptr[w]; q < t.well_ptr[w + 1]; ++q) {
        const double d = c.wells[t.perf_entry[t.well_perfs[q]]].wellbore_density_kg_m3;
        if (std::isfinite(d) && d >= 0.0) {
          density = d;
          break;
        }
      }
      if (!std::isfinite(density)) {
        double total = 0.0, count = 0.0;
        for (int q = t.well_ptr[w]; q < t.well_ptr[w + 1]; ++q) {
          const int k = t.well_perfs[q];
          const double p = pc.p(k), sw = pc.sw(k);
          const double rho_w = inv_bw(f, p) * f.rho_w;
          double rho;
          if (f.three_phase) {
            // producer_control_phase_fractions_for_pressures (well_control.rs:373-398)
            const double sg = sg_rs[4 * k], rs = sg_rs[4 * k + 1];
            if (t.perf_inj[k]) {
              rho = f.inject_gas ? gas_density3<double>(f, p) : rho_w;
            } else {
              double lw, lo, lg = 0.0;
              if (f.has_scal3) {
                lw = fmax(k_rw3(f, sw) / f.mu_w, 0.0);
                lo = fmax(k_ro_stone2(f, sw, sg) / mu_o_for_rs(f, p, rs), 0.0);
                lg = fmax(k_rg3(f, sg) / get_mu_g(f, p), 0.0);
              } else {
                lw = fmax(corey_krw(f, sw) / f.mu_w, 0.0);
                lo = fmax(corey_kro(f, sw) / mu_o_for_rs(f, p, rs), 0.0);
              }
              const double lt = fmax(lw + lo + lg, kF64Eps);
              const double fw = std::clamp(lw / lt, 0.0, 1.0), fo = std::clamp(lo / lt, 0.0, 1.0),
                           fg = std::clamp(lg / lt, 0.0, 1.0);
              rho = fw * rho_w + fo * oil_density3<double>(f, p, fmax(rs, 0.0)) + fg * gas_density3<double>(f, p);
            }
          } else if (t.perf_inj[k]) {
            rho = rho_w;
          } else {
            const double lw = fmax(corey_krw(f, sw) / f.mu_w, 0.0), lo = fmax(corey_kro(f, sw) / f.mu_o, 0.0);
            const double lt = fmax(lw + lo, kF64Eps);
            const double fw = std::clamp(lw / lt, 0.0, 1.0), fo = std::clamp(lo / lt, 0.0, 1.0);
            rho = fw * rho_w + fo * (f.rho_o / oil_fvf_plain(f, p));  // no gas phase
          }
          if (std::isfinite(rho) && rho > 0.0) {
            total += rho;
            count += 1.0;
          }
        }
        density = count > 0.0 ? total / count : 0.0;
      }
      for (int q = t.well_ptr[w]; q < t.well_ptr[w + 1]; ++q) {
        const int e = t.perf_entry[t.well_perfs[q]];
        const double h = density * 9.80665 * (c.depth_layer[c.wells[e].k] - datum) * 1e-5;
        c.head_offset[e] = std::isfinite(h) ? h : 0.0;
      }
    }
  }
  if (t.n_perfs > 0) {
    std::vector<double> head(t.n_perfs);
    for (int k = 0; k < t.n_perfs; ++k) head[k] = c.head_offset[t.perf_entry[k]];
    RF_CUDA(cudaMemcpyAsync(c.d_perf_head.p, head.data(), sizeof(double) * head.size(), cudaMemcpyHostToDevice,
                            c.stream));
    stream_wait(c);
  }
}

static int step(Ctx& c, double target, RfStepReport* out) {
  RfStepReport rep{};
  RF_CUDA(cudaEventRecord(c.ev0, c.stream));
  adjoint_on_step_begin(c);
  refresh_head_offsets(c);
  double stepped = 0.0;
  int substeps = 0, warning = 0;
  const int max_sub = 100000;
  double last_dt = target, growth = 3.0;
  double errs[3] = {0.1, 0.1, 0.1};
  c.last_warning.clear();
  const size_t nb = sizeof(double) * c.n;
  while (stepped < target && substeps < max_sub) {
    const double remaining = target - stepped;
    double proposed;
    if (substeps == 0)
      proposed = c.time_days <= 1e-12 ? fmin(remaining, remaining <= 1.0 + 1e-12 ? 0.25 : 1.0) : remaining;
    else
      proposed = fmin(remaining, last_dt * growth);
    double trial = c.ctl_one_substep ? remaining : fmin(proposed, remaining);
    int retry = 0;
    // previous_state = FimState::from_simulator: the accepted state with the written-back
    // (two-phase: zero) gas primary
    RF_CUDA(cudaMemcpyAsync(c.d_pp.p, c.d_p.p, nb, cudaMemcpyDeviceToDevice, c.stream));
    RF_CUDA(cudaMemcpyAsync(c.d_psw.p, c.d_sw.p, nb, cudaMemcpyDeviceToDevice, c.stream));
    if (c.fluid.three_phase)
      from_simulator3(c);  // regimes and hc = Sg (saturated) or Rs (undersaturated)
    else
      RF_CUDA(cudaMemsetAsync(c.d_phc.p, 0, nb, c.stream));
    const WellState ws0 = initial_well_state(c);
    for (;;) {
      WellState ws = ws0;
      NewtonReport nr = run_newton(c, ws, trial);
      rep.newton_iterations += nr.newton_iterations;
      rep.linear_iterations += nr.linear_iterations;
      rep.linear_solves += nr.linear_solves;
      if (nr.converged && c.fluid.three_phase) {
        // relative change, and the inventories of the simulator state before the write-back
        double sb[kStateQ3], sa[kStateQ3];
        state_sums3(c, c.d_pp.p, c.d_psw.p, c.d_phc.p, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_pp.p, c.d_psw.p, sb);
        const double rc = sb[1] > 0.0 ? sb[0] / sb[1] : 0.0;
        errs[0] = errs[1];
        errs[1] = errs[2];
        errs[2] = rc;
        growth = growth_factor(trial, nr.newton_iterations, errs, retry);
        derive3(c);  // write back So, Sg, Rs
        for (int p = 0; p < c.topo.n_perfs; ++p) c.wells[c.topo.perf_entry[p]].bhp = ws.bhp[c.topo.perf_well[p]];
        state_sums3(c, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_p.p, c.d_sw.p, sa);
        record_step3(c, ws, trial, sa[2] - sb[2], sb[3] - sa[3], sa[4] - sb[4], sa);
        adjoint_on_substep_accepted(c, trial);
        c.time_days += trial;
        stepped += trial;
        last_dt = trial;
        substeps++;
        rep.substeps++;
        rep.last_dt_days = trial;
        break;
      }
      if (nr.converged) {
        double sums_prev[7], sums_new[7];
        state_sums(c, c.d_pp.p, c.d_psw.p, c.d_phc.p, c.d_p.p, c.d_sw.p, c.d_hc.p, sums_new);
        state_sums(c, c.d_pp.p, c.d_psw.p, c.d_phc.p, c.d_pp.p, c.d_psw.p, c.d_phc.p, sums_prev);
        const double rc = sums_new[1] > 0.0 ? sums_new[0] / sums_new[1] : 0.0;
        errs[0] = errs[1];
        errs[1] = errs[2];
        errs[2] = rc;
        growth = growth_factor(trial, nr.newton_iterations, errs, retry);
        // write back: the two-phase gas primary is zero in the simulator state
        RF_CUDA(cudaMemsetAsync(c.d_hc.p, 0, nb, c.stream));
        for (int p = 0; p < c.topo.n_perfs; ++p) c.wells[c.topo.perf_entry[p]].bhp = ws.bhp[c.topo.perf_well[p]];
        double sums_after[7];
        state_sums(c, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_p.p, c.d_sw.p, c.d_hc.p, sums_after);
        record_step(c, ws, trial, sums_after[2] - sums_prev[2], sums_prev[3] - sums_after[3], sums_after);
        adjoint_on_substep_accepted(c, trial);
        c.time_days += trial;
        stepped += trial;
        last_dt = trial;
        substeps++;
        rep.substeps++;
        rep.last_dt_days = trial;
        break;
      }
      if (c.ctl_one_substep) {  // controller option: no retries
        warning = 2;
        c.last_warning = "FIM Newton step did not converge in the one substep of the report step";
        break;
      }
      const double next = trial * 0.33;
      retry++;
      rep.retries++;
      if (!std::isfinite(next) || next <= 1e-12) {
        warning = 1;
        c.last_warning = "FIM Newton step collapsed timestep";
        break;
      }
      if (retry >= 16) {
        warning = 2;
        c.last_warning = "FIM Newton step exceeded retry budget";
        break;
      }
      trial = next;
    }
    if (warning) {
      // restore the last accepted state
      RF_CUDA(cudaMemcpyAsync(c.d_p.p, c.d_pp.p, nb, cudaMemcpyDeviceToDevice, c.stream));
      RF_CUDA(cudaMemcpyAsync(c.d_sw.p, c.d_psw.p, nb, cudaMemcpyDeviceToDevice, c.stream));
      RF_CUDA(cudaMemcpyAsync(c.d_hc.p, c.d_phc.p, nb, cudaMemcpyDeviceToDevice, c.stream));
      break;
    }
  }
  if (!warning && substeps == max_sub && stepped < target) warning = 3;
  prof_resolve(c);
  RF_CUDA(cudaEventRecord(c.ev1, c.stream));
  if (fiber_active()) fiber_wait_event(c.ev1);
  RF_CUDA(cudaEventSynchronize(c.ev1));
  float ms = 0.f;
  RF_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
  rep.device_ms = ms;
  rep.warning = warning;
  rep.time_days = c.time_days;
  rep.advanced_days = stepped;
  if (out) *out = rep;
  return warning ? RF_STEP_WARNING : RF_OK;
}

// ---------------------------------------------------------------------------------------------
// setup
// ---------------------------------------------------------------------------------------------
static double harmonic(double a, double b) { return a + b == 0.0 ? 0.0 : 2.0 * a * b / (a + b); }

static bool peaceman_wi(const Ctx& c, const RfWell& w, int id, double& out) {
  const double kx = c.kx[id], ky = c.ky[id];
  if (!std::isfinite(kx) || !std::isfinite(ky) || kx <= 0.0 || ky <= 0.0) return false;
  const double r_eq = 0.28 * std::sqrt(std::sqrt(kx / ky) * c.dx * c.dx + std::sqrt(ky / kx) * c.dy * c.dy) /
                      (std::pow(kx / ky, 0.25) + std::pow(ky / kx, 0.25));
  if (!std::isfinite(r_eq) || r_eq <= w.well_radius) return false;
  const double k_avg = std::sqrt(kx * ky);
  const double denom = std::log(r_eq / w.well_radius) + w.skin;
  if (!std::isfinite(k_avg) || k_avg <= 0.0 || !std::isfinite(denom) || std::fabs(denom) <= kF64Eps) return false;
  out = kDarcy * 2.0 * M_PI * k_avg * c.dz[id / (c.nx * c.ny)] / denom;
  return true;
}

static int load(Ctx& c, const RfDeck* d) {
  if (!d || d->abi_version != RF_ABI_VERSION) {
    c.err = "deck is null or was built for another ABI version";
    return RF_ERR_INVALID;
  }
  if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0) {
    c.err = "grid dimensions must be positive";
    return RF_ERR_INVALID;
  }
  if (d->three_phase_mode) {
    if (d->n_pvt_rows < 1 || !d->pvt_rows) {
      c.err = "three-phase mode without a PVT table is not supported";
      return RF_ERR_UNSUPPORTED;
    }
  } else if (d->n_pvt_rows > 0 && d->pvt_rows) {
    c.err = "a PVT table in two-phase mode is not implemented by the device path";
    return RF_ERR_UNSUPPORTED;
  }
  c.nx = d->nx;
  c.ny = d->ny;
  c.nz = d->nz;
  c.n = c.nx * c.ny * c.nz;
  const int n = c.n;
  c.dx = d->dx;
  c.dy = d->dy;
  c.dz.assign(d->dz, d->dz + c.nz);
  c.porosity.assign(d->porosity, d->porosity + n);
  c.kx.assign(d->perm_x, d->perm_x + n);
  c.ky.assign(d->perm_y, d->perm_y + n);
  c.kz.assign(d->perm_z, d->perm_z + n);
  {
    const int rc = fluid_from_deck(d, c.fluid, c.h_pvt, c.err);
    if (rc != RF_OK) return rc;
  }
  c.hfluid = c.fluid;
  c.wells.assign(d->wells, d->wells + d->n_wells);
  c.inj_rate_ctl = d->injector_rate_controlled;
  c.prod_rate_ctl = d->producer_rate_controlled;
  c.inj_enabled = d->injector_enabled;
  c.tgt_inj = d->target_injector_rate_m3_day;
  c.tgt_prod = d->target_producer_rate_m3_day;
  c.tgt_inj_surf = d->target_injector_surface_rate_m3_day;
  c.tgt_prod_surf = d->target_producer_surface_rate_m3_day;
  c.bhp_min = d->well_bhp_min;
  c.bhp_max = d->well_bhp_max;
  c.head_offset.assign(c.wells.size(), 0.0);
  // depth of each layer centre and pore volumes
  c.depth_layer.resize(c.nz);
  for (int k = 0; k < c.nz; ++k) {
    double dep = d->depth_reference_m;
    for (int l = 0; l < k; ++l) dep += c.dz[l];
    c.depth_layer[k] = dep + c.dz[k] * 0.5;
  }
  c.pv.resize(n);
  for (int i = 0; i < n; ++i) c.pv[i] = c.dx * c.dy * c.dz[i / (c.nx * c.ny)] * c.porosity[i];
  // physical wells (fim/wells.rs:544-594)
  Topology& t = c.topo;
  std::map<std::tuple<int, int, int, int, uint64_t, uint64_t, uint64_t>, int> groups;
  std::vector<std::vector<int>> perfs_of;
  std::vector<int> cell_taken(n, 0);
  for (int e = 0; e < int(c.wells.size()); ++e) {
    const RfWell& w = c.wells[e];
    if (w.i < 0 || w.i >= c.nx || w.j < 0 || w.j >= c.ny || w.k < 0 || w.k >= c.nz) {
      c.err = "well completion outside the grid";
      return RF_ERR_INVALID;
    }
    std::tuple<int, int, int, int, uint64_t, uint64_t, uint64_t> key;
    if (w.physical_well_id >= 0) {
      key = std::make_tuple(0, w.physical_well_id, 0, 0, 0, 0, 0);
    } else {
      uint64_t b, r, s;
      std::memcpy(&b, &w.bhp, 8);
      std::memcpy(&r, &w.well_radius, 8);
      std::memcpy(&s, &w.skin, 8);
      key = std::make_tuple(1, w.injector, w.i, w.j, b, r, s);
    }
    int pw;
    auto it = groups.find(key);
    if (it == groups.end()) {
      pw = t.n_wells++;
      groups[key] = pw;
      t.well_rep.push_back(e);
      t.well_inj.push_back(w.injector != 0);
      perfs_of.emplace_back();
    } else {
      pw = it->second;
    }
    const int cell = w.k * c.nx * c.ny + w.j * c.nx + w.i;
    if (cell_taken[cell]++) {
      c.err = "multiple well completions in the same cell are not supported";
      return RF_ERR_INVALID;
    }
    const int k = t.n_perfs++;
    t.perf_cell.push_back(cell);
    t.perf_well.push_back(pw);
    t.perf_entry.push_back(e);
    t.perf_inj.push_back(w.injector != 0);
    double wi = 0.0;
    const bool has = peaceman_wi(c, w, cell, wi);
    t.perf_has_wi.push_back(has);
    t.perf_wi.push_back(wi);
    perfs_of[pw].push_back(k);
  }
  t.well_ptr.assign(1, 0);
  for (int w = 0; w < t.n_wells; ++w) {
    for (int k : perfs_of[w]) t.well_perfs.push_back(k);
    t.well_ptr.push_back(int(t.well_perfs.size()));
    t.max_perfs_per_well = std::max(t.max_perfs_per_well, int(perfs_of[w].size()));
  }
  if (t.max_perfs_per_well > 255 || t.n_perfs > 1000) {
    c.err = "more than 255 perforations per well or 1000 in total is not supported";
    return RF_ERR_UNSUPPORTED;
  }
  c.h_p.assign(n, 300.0);
  c.h_sw.assign(n, 0.3);
  return RF_OK;
}

static void build_pattern(Ctx& c) {
  const int n = c.n, nx = c.nx, ny = c.ny, nz = c.nz, nxy = nx * ny;
  std::vector<std::vector<int>> extra(n);
  const Topology& t = c.topo;
  for (int w = 0; w < t.n_wells; ++w)
    for (int a = t.well_ptr[w]; a < t.well_ptr[w + 1]; ++a)
      for (int b = t.well_ptr[w]; b < t.well_ptr[w + 1]; ++b)
        extra[t.perf_cell[t.well_perfs[a]]].push_back(t.perf_cell[t.well_perfs[b]]);
  c.h_row_ptr.assign(n + 1, 0);
  c.h_col.clear();
  c.h_diag.assign(n, -1);
  c.h_stencil.assign(size_t(n) * 7, -1);
  for (int i = 0; i < n; ++i) {
    const int ci = i % nx, cj = (i / nx) % ny, ck = i / nxy;
    std::vector<int> cols;
    if (ck > 0) cols.push_back(i - nxy);
    if (cj > 0) cols.push_back(i - nx);
    if (ci > 0) cols.push_back(i - 1);
    cols.push_back(i);
    if (ci + 1 < nx) cols.push_back(i + 1);
    if (cj + 1 < ny) cols.push_back(i + nx);
    if (ck + 1 < nz) cols.push_back(i + nxy);
    for (int e : extra[i]) cols.push_back(e);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    const int base = int(c.h_col.size());
    for (size_t k = 0; k < cols.size(); ++k) {
      const int j = cols[k], pos = base + int(k);
      c.h_col.push_back(j);
      int slot = -1;
      if (j == i) slot = kDiag;
      else if (j == i - nxy && ck > 0) slot = kZm;
      else if (j == i - nx && cj > 0) slot = kYm;
      else if (j == i - 1 && ci > 0) slot = kXm;
      else if (j == i + 1 && ci + 1 < nx) slot = kXp;
      else if (j == i + nx && cj + 1 < ny) slot = kYp;
      else if (j == i + nxy && ck + 1 < nz) slot = kZp;
      if (slot >= 0) c.h_stencil[size_t(i) * 7 + slot] = pos;
      if (j == i) c.h_diag[i] = pos;
    }
    c.h_row_ptr[i + 1] = int(c.h_col.size());
  }
  c.nnzb = int(c.h_col.size());
  auto find_pos = [&](int r, int col) {
    auto b = c.h_col.begin() + c.h_row_ptr[r], e = c.h_col.begin() + c.h_row_ptr[r + 1];
    return int(std::lower_bound(b, e, col) - c.h_col.begin());
  };
  c.h_fill_off.clear();
  c.h_fill_pos.clear();
  c.h_tinv_off.clear();
  c.h_perf_row_blocks_off.assign(t.n_perfs, 0);
  int tinv = 0, rowoff = 0;
  for (int w = 0; w < t.n_wells; ++w) {
    c.h_fill_off.push_back(int(c.h_fill_pos.size()));
    const int m = t.well_ptr[w + 1] - t.well_ptr[w];
    for (int a = 0; a < m; ++a)
      for (int b = 0; b < m; ++b)
        c.h_fill_pos.push_back(find_pos(t.perf_cell[t.well_perfs[t.well_ptr[w] + a]],
                                        t.perf_cell[t.well_perfs[t.well_ptr[w] + b]]));
    c.h_tinv_off.push_back(tinv);
    tinv += (1 + m) * (1 + m);
  }
  for (int p = 0; p < t.n_perfs; ++p) {
    c.h_perf_row_blocks_off[p] = rowoff;
    const int cell = t.perf_cell[p];
    rowoff += c.h_row_ptr[cell + 1] - c.h_row_ptr[cell];
  }
  c.d_tinv.alloc(tinv);
  c.d_jrr_perf.alloc(size_t(rowoff) * 9);
}

template <class T>
static void upload(DBuf<T>& b, const std::vector<T>& h) {
  b.alloc(h.size());
  if (!h.empty()) RF_CUDA(cudaMemcpy(b.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
}

static void setup_device(Ctx& c) {
  RF_CUDA(cudaGetDevice(&c.device));
  RF_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device));
  RF_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  c.h_pin_bytes = sizeof(double) * (16 * size_t(c.topo.n_wells + c.topo.n_perfs) + 4096);
  RF_CUDA(cudaMallocHost(&c.h_pin, c.h_pin_bytes));
  c.pin_pending.reserve(64);
  RF_CUDA(cudaEventCreate(&c.ev0));
  RF_CUDA(cudaEventCreate(&c.ev1));
  RF_CUDA(cudaEventCreateWithFlags(&c.ev_wait, cudaEventDisableTiming));
  const int n = c.n, nx = c.nx, ny = c.ny, nz = c.nz, nxy = nx * ny;
  std::vector<double> tx(n, 0.0), ty(n, 0.0), tz(n, 0.0);
  for (int i = 0; i < n; ++i) {
    const int ci = i % nx, cj = (i / nx) % ny, ck = i / nxy;
    if (ci + 1 < nx) tx[i] = kDarcy * (harmonic(c.kx[i], c.kx[i + 1]) * (c.dy * c.dz[ck]) / c.dx);
    if (cj + 1 < ny) ty[i] = kDarcy * (harmonic(c.ky[i], c.ky[i + nx]) * (c.dx * c.dz[ck]) / c.dy);
    if (ck + 1 < nz) {
      const double p1 = c.kz[i], p2 = c.kz[i + nxy];
      const double denom = p2 * c.dz[ck] + p1 * c.dz[ck + 1];
      tz[i] = denom <= 0.0 ? 0.0 : kDarcy * (2.0 * p1 * p2 * (c.dx * c.dy) / denom);
    }
  }
  upload(c.d_pv, c.pv);
  upload(c.d_tx, tx);
  upload(c.d_ty, ty);
  upload(c.d_tz, tz);
  upload(c.d_depth, c.depth_layer);
  for (auto* b : {&c.d_p, &c.d_sw, &c.d_hc, &c.d_pp, &c.d_psw, &c.d_phc, &c.d_cp, &c.d_csw, &c.d_chc}) b->alloc(n);
  RF_CUDA(cudaMemset(c.d_hc.p, 0, sizeof(double) * n));
  if (c.fluid.three_phase) {
    c.d_reg.alloc(n);
    for (auto* b : {&c.d_so, &c.d_sg, &c.d_rs}) b->alloc(n);
    RF_CUDA(cudaMemset(c.d_reg.p, 0, sizeof(int) * n));
    RF_CUDA(cudaMemset(c.d_sg.p, 0, sizeof(double) * n));
    RF_CUDA(cudaMemset(c.d_rs.p, 0, sizeof(double) * n));
    upload(c.d_pvt, c.h_pvt);
    c.fluid.pvt = c.d_pvt.p;
    c.hfluid.pvt = c.h_pvt.data();
  }
  build_pattern(c);
  upload(c.d_row_ptr, c.h_row_ptr);
  upload(c.d_col, c.h_col);
  upload(c.d_diag, c.h_diag);
  upload(c.d_stencil, c.h_stencil);
  upload(c.d_fill_off, c.h_fill_off);
  upload(c.d_fill_pos, c.h_fill_pos);
  upload(c.d_tinv_off, c.h_tinv_off);
  upload(c.d_perf_row_off, c.h_perf_row_blocks_off);
  c.d_res.alloc(3 * size_t(n));
  c.d_val.alloc(size_t(c.nnzb) * 9);
  const Topology& t = c.topo;
  upload(c.d_perf_cell, t.perf_cell);
  upload(c.d_perf_well, t.perf_well);
  upload(c.d_perf_inj, t.perf_inj);
  upload(c.d_perf_has_wi, t.perf_has_wi);
  upload(c.d_perf_wi, t.perf_wi);
  std::vector<double> head(t.n_perfs, 0.0);
  for (int p = 0; p < t.n_perfs; ++p) head[p] = c.head_offset[t.perf_entry[p]];
  upload(c.d_perf_head, head);
  upload(c.d_well_ptr, t.well_ptr);
  upload(c.d_well_perfs, t.well_perfs);
  c.d_ctrl.alloc(t.n_wells);
  c.d_bhp.alloc(t.n_wells);
  c.d_q.alloc(t.n_perfs);
  c.d_res_tail.alloc(t.n_wells + t.n_perfs);
  c.d_jrw.alloc(3 * size_t(t.n_perfs));
  c.d_jwr_perf.alloc(3 * size_t(t.n_perfs));
  c.d_jwr_ctrl.alloc(3 * size_t(t.n_perfs));
  c.d_jww_perf_bhp.alloc(t.n_perfs);
  c.d_jww_ctrl_q.alloc(t.n_perfs);
  c.d_jww_ctrl_bhp.alloc(t.n_wells);
  c.d_dx_tail.alloc(t.n_wells + t.n_perfs);
  c.d_rhs_red.alloc(3 * size_t(n));
  build_levels(c);
  setup_linear_workspace(c);
  // every upload above used the default stream; the context's stream is non-blocking
  RF_CUDA(cudaDeviceSynchronize());
}

static void free_ctx(Ctx& c) {
  adjoint_free(c);
  for (auto* b : {&c.d_pv, &c.d_tx, &c.d_ty, &c.d_tz, &c.d_depth, &c.d_p, &c.d_sw, &c.d_hc, &c.d_pp, &c.d_psw, &c.d_phc,
                  &c.d_cp, &c.d_csw, &c.d_chc, &c.d_res, &c.d_val, &c.d_perf_wi, &c.d_perf_head, &c.d_bhp, &c.d_q,
                  &c.d_res_tail, &c.d_jrw, &c.d_jwr_perf, &c.d_jwr_ctrl, &c.d_jww_perf_bhp, &c.d_jww_ctrl_q,
                  &c.d_jww_ctrl_bhp, &c.d_tinv, &c.d_rhs_red, &c.d_rhs_full, &c.d_dx_tail, &c.d_jrr_perf, &c.d_V,
                  &c.d_Z, &c.d_w, &c.d_x, &c.d_tmp, &c.d_tmp2, &c.d_cand, &c.d_cpr_w, &c.d_pval, &c.d_plu,
                  &c.d_pdiag, &c.d_lu, &c.d_dinv, &c.d_cres, &c.d_full, &c.d_dense, &c.d_pvec, &c.d_partials,
                  &c.d_scal, &c.d_so, &c.d_sg, &c.d_rs, &c.d_pvt})
    b->free();
  c.d_reg.free();
  for (auto* b : {&c.d_row_ptr, &c.d_col, &c.d_diag, &c.d_stencil, &c.d_fill_off, &c.d_fill_pos, &c.d_perf_cell,
                  &c.d_perf_well, &c.d_perf_inj, &c.d_perf_has_wi, &c.d_well_ptr, &c.d_well_perfs, &c.d_tinv_off,
                  &c.d_perf_row_off, &c.d_flag_dense, &c.d_dense_perm})
    b->free();
  for (auto* b : {&c.d_own_rows, &c.d_own_ptr, &c.d_fcnt, &c.d_bcnt, &c.d_fdep, &c.d_bdep, &c.d_pipe_status}) b->free();
  c.d_reqf.free();
  c.d_reqb.free();
  c.d_cons.free();
  for (auto* b : {&c.d_fval, &c.d_bval, &c.d_dval}) b->free();
  for (auto* b : {&c.d_fval32, &c.d_bval32, &c.d_dval32}) b->free();
  for (auto* b : {&c.d_lu32, &c.d_dinv32, &c.d_plu32, &c.d_pval32, &c.d_pdiag32, &c.d_pvec32, &c.d_sweep32})
    b->free();
  c.d_bmask.free();
  c.d_ctrl.free();
  for (auto* b : {&c.d_dir_a, &c.d_dir_lu, &c.d_dir_vec}) b->free();
  c.d_dir_perm.free();
  c.dir_rows = 0;
  free_level_plan(c);
  for (auto* b : {&c.d_tri_ptr, &c.d_tri_up, &c.d_tri_ip, &c.d_pt_ptr, &c.d_pt_lp, &c.d_pt_ue}) b->free();
  c.d_ref_b.free();
  c.d_fac_simple.free();
  c.d_ref_x.free();
  if (c.levels.d_rows) cudaFree(c.levels.d_rows);
  if (c.levels.d_ptr) cudaFree(c.levels.d_ptr);
  if (c.levels.d_long_rows) cudaFree(c.levels.d_long_rows);
  if (c.levels.d_long_ptr) cudaFree(c.levels.d_long_ptr);
  for (cudaEvent_t e : c.ev_pool) cudaEventDestroy(e);
  c.ev_pool.clear();
  if (c.d_bicg_iters) cudaFree(c.d_bicg_iters);
  c.d_bicg_iters = nullptr;
  if (c.ev0) cudaEventDestroy(c.ev0);
  if (c.ev1) cudaEventDestroy(c.ev1);
  if (c.ev_wait) cudaEventDestroy(c.ev_wait);
  if (c.h_pin) cudaFreeHost(c.h_pin);
  c.h_pin = nullptr;
  if (c.stream && c.stream_owned) cudaStreamDestroy(c.stream);
  c.stream = nullptr;
}

#include "rf_adjoint.inc"

}  // namespace rf

// =============================================================================================
// C ABI
// =============================================================================================
struct RfCtx {
  rf::Ctx c;
};

static std::mutex g_err_mu;
static std::string g_last_create_error;

template <class F>
static int32_t guarded(RfCtx* ctx, F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    if (ctx) ctx->c.err = e.what();
    return RF_ERR_CUDA;
  }
}

extern "C" {

int32_t rf_create(const RfDeck* deck, RfCtx** out) {
  if (!out) return RF_ERR_INVALID;
  *out = nullptr;
  auto* h = new RfCtx();
  int32_t rc = RF_OK;
  try {
    rc = rf::load(h->c, deck);
    if (rc == RF_OK) rf::setup_device(h->c);
  } catch (const std::exception& e) {
    h->c.err = e.what();
    rc = RF_ERR_CUDA;
  }
  if (rc != RF_OK) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_create_error = h->c.err;
    try {
      rf::free_ctx(h->c);
    } catch (...) {
    }
    delete h;
    return rc;
  }
  *out = h;
  return RF_OK;
}

int32_t rf_destroy(RfCtx* ctx) {
  if (!ctx) return RF_OK;
  rf::free_ctx(ctx->c);
  delete ctx;
  return RF_OK;
}

int32_t rf_last_error(const RfCtx* ctx, char* buf, size_t len) {
  if (!buf || len == 0) return RF_ERR_INVALID;
  std::string msg;
  if (ctx) {
    msg = ctx->c.err;
  } else {
    std::lock_guard<std::mutex> lk(g_err_mu);
    msg = g_last_create_error;
  }
  std::snprintf(buf, len, "%s", msg.c_str());
  return RF_OK;
}

int32_t rf_set_state(RfCtx* ctx, const double* p, const double* sw, const double* sg, const double* rs, double t) {
  if (!ctx || !p || !sw) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    rf::Ctx& c = ctx->c;
    if (c.fluid.three_phase) {
      // loadState (frontend.rs:931-1008): So = max(1 - Sw - Sg, 0)
      const size_t bytes = sizeof(double) * c.n;
      std::vector<double> hsg(c.n, 0.0), hrs(c.n, 0.0), hso(c.n);
      if (sg) hsg.assign(sg, sg + c.n);
      if (rs) hrs.assign(rs, rs + c.n);
      for (int i = 0; i < c.n; ++i) hso[i] = fmax(1.0 - sw[i] - hsg[i], 0.0);
      RF_CUDA(cudaMemcpyAsync(c.d_p.p, p, bytes, cudaMemcpyHostToDevice, c.stream));
      RF_CUDA(cudaMemcpyAsync(c.d_sw.p, sw, bytes, cudaMemcpyHostToDevice, c.stream));
      RF_CUDA(cudaMemcpyAsync(c.d_sg.p, hsg.data(), bytes, cudaMemcpyHostToDevice, c.stream));
      RF_CUDA(cudaMemcpyAsync(c.d_rs.p, hrs.data(), bytes, cudaMemcpyHostToDevice, c.stream));
      RF_CUDA(cudaMemcpyAsync(c.d_so.p, hso.data(), bytes, cudaMemcpyHostToDevice, c.stream));
      RF_CUDA(cudaMemsetAsync(c.d_hc.p, 0, bytes, c.stream));
      RF_CUDA(cudaStreamSynchronize(c.stream));
      c.time_days = t;
      return RF_OK;
    }
    for (int i = 0; i < c.n; ++i)
      if (sg && sg[i] != 0.0) {
        c.err = "a nonzero gas saturation needs the three-phase path";
        return RF_ERR_UNSUPPORTED;
      }
    (void)rs;
    c.h_p.assign(p, p + c.n);
    c.h_sw.assign(sw, sw + c.n);
    RF_CUDA(cudaMemcpyAsync(c.d_p.p, p, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream));
    RF_CUDA(cudaMemcpyAsync(c.d_sw.p, sw, sizeof(double) * c.n, cudaMemcpyHostToDevice, c.stream));
    RF_CUDA(cudaMemsetAsync(c.d_hc.p, 0, sizeof(double) * c.n, c.stream));
    RF_CUDA(cudaStreamSynchronize(c.stream));
    c.time_days = t;
    return RF_OK;
  });
}

int32_t rf_get_state(const RfCtx* cctx, double* p, double* sw, double* so, double* sg, double* rs, double* t) {
  if (!cctx) return RF_ERR_INVALID;
  RfCtx* ctx = const_cast<RfCtx*>(cctx);
  return guarded(ctx, [&]() -> int32_t {
    rf::Ctx& c = ctx->c;
    if (c.fluid.three_phase) {
      const size_t bytes = sizeof(double) * c.n;
      const double* src[5] = {c.d_p.p, c.d_sw.p, c.d_so.p, c.d_sg.p, c.d_rs.p};
      double* dst[5] = {p, sw, so, sg, rs};
      for (int a = 0; a < 5; ++a)
        if (dst[a]) RF_CUDA(cudaMemcpyAsync(dst[a], src[a], bytes, cudaMemcpyDeviceToHost, c.stream));
      RF_CUDA(cudaStreamSynchronize(c.stream));
      if (t) *t = c.time_days;
      return RF_OK;
    }
    std::vector<double> hp(c.n), hsw(c.n);
    RF_CUDA(cudaMemcpyAsync(hp.data(), c.d_p.p, sizeof(double) * c.n, cudaMemcpyDeviceToHost, c.stream));
    RF_CUDA(cudaMemcpyAsync(hsw.data(), c.d_sw.p, sizeof(double) * c.n, cudaMemcpyDeviceToHost, c.stream));
    RF_CUDA(cudaStreamSynchronize(c.stream));
    for (int i = 0; i < c.n; ++i) {
      if (p) p[i] = hp[i];
      if (sw) sw[i] = hsw[i];
      if (so) so[i] = fmax(1.0 - hsw[i], 0.0);
      if (sg) sg[i] = 0.0;
      if (rs) rs[i] = 0.0;
    }
    if (t) *t = c.time_days;
    return RF_OK;
  });
}

int32_t rf_get_well_bhp(const RfCtx* ctx, double* bhp, int32_t n) {
  if (!ctx || !bhp) return RF_ERR_INVALID;
  for (int i = 0; i < n && i < int(ctx->c.wells.size()); ++i) bhp[i] = ctx->c.wells[i].bhp;
  return RF_OK;
}

int32_t rf_step(RfCtx* ctx, double target_dt_days, RfStepReport* out) {
  if (!ctx || !(target_dt_days > 0.0) || !std::isfinite(target_dt_days)) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t { return rf::step(ctx->c, target_dt_days, out); });
}

int32_t rf_set_controller_options(RfCtx* ctx, int32_t one_substep_per_report_step, double cnv_tol, double mb_tol) {
  if (!ctx || !(cnv_tol >= 0.0) || !(mb_tol >= 0.0)) return RF_ERR_INVALID;
  ctx->c.ctl_one_substep = one_substep_per_report_step != 0;
  ctx->c.ctl_cnv = cnv_tol;
  ctx->c.ctl_mb = mb_tol;
  return RF_OK;
}

int32_t rf_set_linear_refinement(RfCtx* ctx, double rtol, int32_t max_passes) {
  if (!ctx || !(rtol >= 0.0) || !(rtol < 1.0) || max_passes < 0) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    rf::Ctx& c = ctx->c;
    if (rtol > 0.0 && !c.d_ref_b.p) {
      c.d_ref_b.alloc(size_t(3) * c.n);
      c.d_ref_x.alloc(size_t(3) * c.n);
    }
    c.lin_refine_rtol = rtol;
    c.lin_refine_passes = max_passes > 0 ? max_passes : 12;
    return RF_OK;
  });
}

int32_t rf_adjoint_record(RfCtx* ctx, int32_t enable) {
  if (!ctx) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t { return rf::adjoint_record(ctx->c, enable); });
}

int32_t rf_backward(RfCtx* ctx, const RfObjective* objective, double* value, double* dJ_dlnk, double* dJ_dcontrols,
                    int32_t n_controls) {
  if (!ctx || !objective) return RF_ERR_INVALID;
  if (objective->kind != RF_OBJECTIVE_CUMULATIVE_OIL) {
    ctx->c.err = "unknown objective kind";
    return RF_ERR_INVALID;
  }
  return guarded(ctx, [&]() -> int32_t { return rf::backward(ctx->c, value, dJ_dlnk, dJ_dcontrols, n_controls); });
}

int32_t rf_well_count(const RfCtx* ctx) { return ctx ? ctx->c.topo.n_wells : 0; }

int32_t rf_rate_history_len(const RfCtx* ctx) { return ctx ? int32_t(ctx->c.rate_history.size()) : 0; }

int32_t rf_rate_history_get(const RfCtx* ctx, int32_t index, RfTimePointRates* out) {
  if (!ctx || !out || index < 0 || index >= int32_t(ctx->c.rate_history.size())) return RF_ERR_INVALID;
  *out = ctx->c.rate_history[index];
  return RF_OK;
}

int32_t rf_linear_solve_bsr(RfCtx* ctx, int32_t n_block_rows, const int32_t* block_row_ptr, const int32_t* block_cols,
                            const double* block_vals, const double* rhs, double* x, RfLinearReport* out) {
  if (!ctx || !block_row_ptr || !block_cols || !block_vals || !rhs || !x) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    rf::Ctx& c = ctx->c;
    if (n_block_rows != c.n) {
      c.err = "the linear-solve seam takes systems on this context's grid (n_block_rows == cells)";
      return RF_ERR_INVALID;
    }
    // values are scattered into this context's block pattern; blocks outside it are rejected
    std::vector<double> vals(size_t(c.nnzb) * 9, 0.0);
    for (int i = 0; i < c.n; ++i)
      for (int k = block_row_ptr[i]; k < block_row_ptr[i + 1]; ++k) {
        const int j = block_cols[k];
        auto b = c.h_col.begin() + c.h_row_ptr[i], e = c.h_col.begin() + c.h_row_ptr[i + 1];
        auto it = std::lower_bound(b, e, j);
        if (it == e || *it != j) {
          c.err = "block outside the context's stencil-plus-well pattern";
          return RF_ERR_INVALID;
        }
        const size_t pos = size_t(it - c.h_col.begin());
        for (int q = 0; q < 9; ++q) vals[pos * 9 + q] += block_vals[size_t(k) * 9 + q];
      }
    RF_CUDA(cudaMemcpyAsync(c.d_val.p, vals.data(), sizeof(double) * vals.size(), cudaMemcpyHostToDevice, c.stream));
    RF_CUDA(cudaMemcpyAsync(c.d_rhs_red.p, rhs, sizeof(double) * 3 * c.n, cudaMemcpyHostToDevice, c.stream));
    RF_CUDA(cudaStreamSynchronize(c.stream));
    // systems of at most 512 rows: direct LU first, CPR-FGMRES when it does not converge
    // (fim/linear/mod.rs:279-300)
    rf::LinResult r;
    bool direct_ok = false, fell_back = false;
    if (rf::direct_rows(c, false) <= rf::kDirectSolveRows) {
      r = rf::linear_solve_direct(c, false, nullptr);
      direct_ok = r.converged;
      fell_back = !direct_ok;
    }
    if (!direct_ok) {
      r = rf::linear_solve_reduced(c);
      r.used_fallback = fell_back;
    }
    RF_CUDA(cudaMemcpyAsync(x, c.d_x.p, sizeof(double) * 3 * c.n, cudaMemcpyDeviceToHost, c.stream));
    RF_CUDA(cudaStreamSynchronize(c.stream));
    if (out) {
      out->converged = r.converged;
      out->iterations = r.iterations;
      out->rhs_norm = r.rhs_norm;
      out->final_residual_norm = r.final_residual_norm;
      out->used_fallback = r.used_fallback;
      out->backend = r.backend;
    }
    return RF_OK;
  });
}

int32_t rf_linear_solve_csr(RfCtx* ctx, int32_t n_rows, const int32_t* row_ptr, const int32_t* cols,
                            const double* vals, const double* rhs, double* x, RfLinearReport* out) {
  if (!ctx || !row_ptr || !cols || !vals || !rhs || !x) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    rf::Ctx& c = ctx->c;
    const rf::Topology& t = c.topo;
    const int n = c.n, n3 = 3 * n, W = t.n_wells, P = t.n_perfs, pts = n3 + W;
    if (n_rows != n3 + W + P) {
      c.err = "the full-system seam takes 3 x cells + wells + perforations rows (" + std::to_string(n3 + W + P) +
              " on this context), got " + std::to_string(n_rows);
      return RF_ERR_INVALID;
    }
    if (row_ptr[0] != 0) {
      c.err = "row_ptr[0] must be 0";
      return RF_ERR_INVALID;
    }
    for (int r = 0; r < n_rows; ++r)
      if (row_ptr[r + 1] < row_ptr[r]) {
        c.err = "row_ptr is not non-decreasing at row " + std::to_string(r);
        return RF_ERR_INVALID;
      }
    std::vector<int> cell_perf(n, -1);  // one completion per cell (checked at creation)
    for (int k = 0; k < P; ++k) cell_perf[t.perf_cell[k]] = k;
    std::vector<double> val(size_t(c.nnzb) * 9, 0.0), jrw(3 * size_t(P), 0.0), jwr_perf(3 * size_t(P), 0.0),
        jwr_ctrl(3 * size_t(P), 0.0), jww_perf_bhp(P, 0.0), jww_ctrl_q(P, 0.0), jww_ctrl_bhp(W, 0.0), diag(P, 0.0),
        res(n3), res_tail(size_t(W) + P);
    for (int r = 0; r < n_rows; ++r)
      for (int e = row_ptr[r]; e < row_ptr[r + 1]; ++e) {
        const int j = cols[e];
        const double v = vals[e];
        if (j < 0 || j >= n_rows) {
          c.err = "column " + std::to_string(j) + " of row " + std::to_string(r) + " is out of range";
          return RF_ERR_INVALID;
        }
        double* slot = nullptr;
        if (r < n3) {
          const int i = r / 3;
          if (j < n3) {
            auto b = c.h_col.begin() + c.h_row_ptr[i], end = c.h_col.begin() + c.h_row_ptr[i + 1];
            auto it = std::lower_bound(b, end, j / 3);
            if (it != end && *it == j / 3) slot = &val[size_t(it - c.h_col.begin()) * 9 + 3 * (r % 3) + j % 3];
          } else if (j >= pts && t.perf_cell[j - pts] == i) {
            slot = &jrw[3 * size_t(j - pts) + r % 3];
          }
        } else if (r < pts) {
          const int w = r - n3;
          if (j < n3) {
            const int k = cell_perf[j / 3];
            if (k >= 0 && t.perf_well[k] == w) slot = &jwr_ctrl[3 * size_t(k) + j % 3];
          } else if (j < pts) {
            if (j - n3 == w) slot = &jww_ctrl_bhp[w];
          } else if (t.perf_well[j - pts] == w) {
            slot = &jww_ctrl_q[j - pts];
          }
        } else {
          const int k = r - pts;
          if (j < n3) {
            if (j / 3 == t.perf_cell[k]) slot = &jwr_perf[3 * size_t(k) + j % 3];
          } else if (j < pts) {
            if (j - n3 == t.perf_well[k]) slot = &jww_perf_bhp[k];
          } else if (j - pts == k) {
            slot = &diag[k];
          }
        }
        if (slot) {
          *slot += v;
        } else if (v != 0.0) {
          c.err = "entry (" + std::to_string(r) + ", " + std::to_string(j) +
                  ") lies outside the device's cell pattern and well couplings";
          return RF_ERR_INVALID;
        }
      }
    for (int k = 0; k < P; ++k) {
      const double want = t.perf_has_wi[k] ? 1.0 : 0.0;
      if (diag[k] != want) {
        c.err = "perforation " + std::to_string(k) + " has diagonal " + std::to_string(diag[k]) +
                "; the device's perforation rows have " + std::to_string(want);
        return RF_ERR_INVALID;
      }
    }
    // the step path's storage holds residuals: rhs = -residual
    for (int r = 0; r < n3; ++r) res[r] = -rhs[r];
    for (int r = n3; r < n_rows; ++r) res_tail[r - n3] = -rhs[r];
    auto up = [&](double* dst, const std::vector<double>& src) {
      if (!src.empty())
        RF_CUDA(cudaMemcpyAsync(dst, src.data(), sizeof(double) * src.size(), cudaMemcpyHostToDevice, c.stream));
    };
    up(c.d_val.p, val);
    up(c.d_res.p, res);
    if (W > 0) {
      up(c.d_res_tail.p, res_tail);
      up(c.d_jrw.p, jrw);
      up(c.d_jwr_perf.p, jwr_perf);
      up(c.d_jwr_ctrl.p, jwr_ctrl);
      up(c.d_jww_perf_bhp.p, jww_perf_bhp);
      up(c.d_jww_ctrl_q.p, jww_ctrl_q);
      up(c.d_jww_ctrl_bhp.p, jww_ctrl_bhp);
    }
    RF_CUDA(cudaStreamSynchronize(c.stream));
    std::vector<double> dx_tail;
    const rf::LinResult r = rf::linear_solve_full(c, dx_tail);
    RF_CUDA(cudaMemcpyAsync(x, c.d_x.p, sizeof(double) * n3, cudaMemcpyDeviceToHost, c.stream));
    RF_CUDA(cudaStreamSynchronize(c.stream));
    for (size_t k = 0; k < dx_tail.size() && n3 + k < size_t(n_rows); ++k) x[n3 + k] = dx_tail[k];
    if (out) {
      out->converged = r.converged && r.finite;
      out->iterations = r.iterations;
      out->rhs_norm = r.rhs_norm;
      out->final_residual_norm = r.final_residual_norm;
      out->used_fallback = r.used_fallback;
      out->backend = r.backend;
    }
    return RF_OK;
  });
}

int64_t rf_kernel_launches(const RfCtx* ctx) { return ctx ? ctx->c.launches : 0; }

int32_t rf_set_cluster_size(RfCtx* ctx, int32_t ctas) {
  if (!ctx || ctas < 0 || ctas > 16) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    return rf::set_cluster_size(ctx->c, ctas == 0 ? rf::auto_cluster_size(ctx->c) : ctas);
  });
}

int32_t rf_set_pressure_solver(RfCtx* ctx, int32_t kind, int32_t threads) {
  if (!ctx || kind < RF_PRESSURE_SOLVER_AUTO || kind > RF_PRESSURE_SOLVER_LEVEL || threads < 0 || threads > 512)
    return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    rf::Ctx& c = ctx->c;
    if (kind == RF_PRESSURE_SOLVER_LEVEL && !c.lvl.built) {
      c.err = "the level-order solver does not support this pattern (level too wide or too many far rows)";
      return RF_ERR_UNSUPPORTED;
    }
    c.pressure_solver = kind;
    c.level_threads = threads;
    rf::level_plan_reshape(c);
    if (kind == RF_PRESSURE_SOLVER_LEVEL && !c.lvl.fits[c.precision == 1 ? 1 : 0]) {
      c.err = "the level-order pressure solver's window does not fit shared memory on this device";
      c.pressure_solver = RF_PRESSURE_SOLVER_AUTO;
      return RF_ERR_UNSUPPORTED;
    }
    return RF_OK;
  });
}

int32_t rf_set_linear_precision(RfCtx* ctx, int32_t mode) {
  if (!ctx || (mode != RF_PRECISION_FP64 && mode != RF_PRECISION_MIXED)) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    rf::set_linear_precision(ctx->c, mode);
    return RF_OK;
  });
}

int32_t rf_profile(RfCtx* ctx, int32_t enable, int32_t reset, double* out, int32_t n) {
  if (!ctx) return RF_ERR_INVALID;
  return guarded(ctx, [&]() -> int32_t {
    rf::Ctx& c = ctx->c;
    rf::prof_resolve(c);
    if (out) {
      long long it = 0;
      RF_CUDA(cudaMemcpyAsync(&it, c.d_bicg_iters, sizeof(long long), cudaMemcpyDeviceToHost, c.stream));
      RF_CUDA(cudaStreamSynchronize(c.stream));
      for (int k = 0; k < n && k < rf::kPhCount; ++k) out[k] = c.phase_ms[k];
      if (n > rf::kPhCount) out[rf::kPhCount] = double(it);
      if (n > rf::kPhCount + 1) out[rf::kPhCount + 1] = double(c.phase_count[rf::kPhBicgKernel]);
      if (n > rf::kPhCount + 2) out[rf::kPhCount + 2] = double(c.nnzb);
      if (n > rf::kPhCount + 3) out[rf::kPhCount + 3] = rf::level_solver_active(c) ? 1.0 : 0.0;
    }
    if (enable >= 0) c.profiling = enable > 0;
    if (reset) {
      for (int k = 0; k < rf::kPhCount; ++k) {
        c.phase_ms[k] = 0.0;
        c.phase_count[k] = 0;
      }
      RF_CUDA(cudaMemsetAsync(c.d_bicg_iters, 0, sizeof(long long), c.stream));
      RF_CUDA(cudaStreamSynchronize(c.stream));
    }
    return RF_OK;
  });
}

// ---------------------------------------------------------------------------------------------
// Ensemble batch: independent decks stepped together.  Every variant keeps its own context
// (device buffers, controller state).  Two ways of driving them:
//  - RF_BATCH_GROUPS (default): the variants are split into groups of about equal size mix, one
//    host thread and one CUDA stream per group; each variant's report step runs as a fiber on its
//    group's thread, and the group's pressure solves and block-ILU0 sweeps go out as one batched
//    launch per kind (rf_fiber.cu);
//  - RF_BATCH_THREADS: one stream per variant and a pool of host threads, each stepping one
//    variant at a time with its own launches.
// The variants never exchange data, and a variant's results are the same either way.
// ---------------------------------------------------------------------------------------------
struct RfBatch {
  std::vector<RfCtx*> ctx;
  std::vector<int> order;  // variant indices by descending cell count
  int threads = 1;
  int device = 0;
  int mode = RF_BATCH_GROUPS;
  std::vector<std::unique_ptr<rf::BatchGroup>> groups;
};

namespace {

// Hand the variants to groups of neighbours in size order (largest first), one stream each, or give
// every variant its own stream again.  A group advances from one batched launch to the next
// together, so a launch lasts as long as its largest solve: groups of similar sizes keep the
// small variants from waiting on large ones, and the groups of small variants finish early and
// leave the device to the large ones.
int32_t regroup(RfBatch* b, int mode) {
  for (auto& g : b->groups) cudaStreamSynchronize(g->stream);
  for (RfCtx* x : b->ctx) {
    rf::Ctx& c = x->c;
    if (!c.stream_owned) {
      c.stream = nullptr;
      if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) return RF_ERR_CUDA;
      c.stream_owned = 1;
    }
    c.batched = 0;
  }
  for (auto& g : b->groups)
    if (g->stream) cudaStreamDestroy(g->stream);
  b->groups.clear();
  b->mode = mode;
  if (mode != RF_BATCH_GROUPS) return RF_OK;
  const int n = int(b->ctx.size());
  const int G = std::max(1, std::min(b->threads, n));
  for (int k = 0; k < G; ++k) {
    auto g = std::make_unique<rf::BatchGroup>();
    if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) return RF_ERR_CUDA;
    b->groups.push_back(std::move(g));
  }
  for (int k = 0; k < n; ++k) {
    const int i = b->order[k];
    rf::BatchGroup& g = *b->groups[int((long long)k * G / n)];
    rf::Ctx& c = b->ctx[i]->c;
    cudaStreamSynchronize(c.stream);
    cudaStreamDestroy(c.stream);
    c.stream = g.stream;
    c.stream_owned = 0;
    c.batched = 1;
    g.members.push_back(i);
  }
  return RF_OK;
}

struct StepJob {
  RfCtx* ctx;
  double dt;
  RfStepReport* rep;
  int32_t rc;
};

void step_job(void* p) {
  StepJob* j = static_cast<StepJob*>(p);
  j->rc = rf_step(j->ctx, j->dt, j->rep);
}

// Fiber stack per variant: the controller's frames hold a few KB; vectors live on the heap.
constexpr size_t kFiberStack = 256 * 1024;

}  // namespace

int32_t rf_batch_create(const RfDeck* const* decks, int32_t n, int32_t host_threads, RfBatch** out) {
  if (!out || !decks || n <= 0) return RF_ERR_INVALID;
  *out = nullptr;
  auto* b = new RfBatch();
  cudaGetDevice(&b->device);
  for (int32_t i = 0; i < n; ++i) {
    RfCtx* c = nullptr;
    const int32_t rc = rf_create(decks[i], &c);
    if (rc != RF_OK) {
      {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_last_create_error = "variant " + std::to_string(i) + ": " + g_last_create_error;
      }
      for (RfCtx* x : b->ctx) rf_destroy(x);
      delete b;
      return rc;
    }
    b->ctx.push_back(c);
  }
  b->order.resize(n);
  for (int32_t i = 0; i < n; ++i) b->order[i] = i;
  std::stable_sort(b->order.begin(), b->order.end(),
                   [&](int x, int y) { return b->ctx[x]->c.n > b->ctx[y]->c.n; });
  // the host threads mostly wait on the device: up to 32 (the most hardware queues
  // CUDA_DEVICE_MAX_CONNECTIONS can give the streams) even on fewer cores
  const int hw = int(std::max(1u, std::thread::hardware_concurrency()));
  b->threads = host_threads > 0 ? host_threads : std::min<int>(n, std::max(hw, 32));
  const int32_t rc = regroup(b, RF_BATCH_GROUPS);
  if (rc != RF_OK) {
    rf_batch_destroy(b);
    return rc;
  }
  *out = b;
  return RF_OK;
}

int32_t rf_batch_destroy(RfBatch* b) {
  if (!b) return RF_OK;
  for (auto& g : b->groups) cudaStreamSynchronize(g->stream);
  for (RfCtx* c : b->ctx) rf_destroy(c);  // group streams are not the contexts' to destroy
  for (auto& g : b->groups)
    if (g->stream) cudaStreamDestroy(g->stream);
  b->groups.clear();
  delete b;
  return RF_OK;
}

int32_t rf_batch_set_mode(RfBatch* b, int32_t mode) {
  if (!b || (mode != RF_BATCH_GROUPS && mode != RF_BATCH_THREADS)) return RF_ERR_INVALID;
  if (mode == b->mode) return RF_OK;
  return regroup(b, mode);
}

int32_t rf_batch_size(const RfBatch* b) { return b ? int32_t(b->ctx.size()) : 0; }

RfCtx* rf_batch_context(RfBatch* b, int32_t i) {
  if (!b || i < 0 || i >= int32_t(b->ctx.size())) return nullptr;
  return b->ctx[i];
}

int32_t rf_batch_profile(RfBatch* b, int32_t enable, int32_t reset, double* out, int32_t n) {
  if (!b) return RF_ERR_INVALID;
  double v[1 + 3 * rf::kBatchKinds] = {double(b->groups.size())};
  for (auto& g : b->groups) {
    g->resolve_timing();
    for (int k = 0; k < rf::kBatchKinds; ++k) {
      v[1 + 3 * k] += double(g->launches[k]);
      v[2 + 3 * k] += double(g->items[k]);
      v[3 + 3 * k] += g->ms_by_kind[k];
    }
  }
  if (out)
    for (int32_t i = 0; i < n && i < int32_t(sizeof(v) / sizeof(v[0])); ++i) out[i] = v[i];
  for (auto& g : b->groups) {
    if (reset) g->reset_stats();
    if (enable >= 0) g->profiling = enable > 0;
  }
  return RF_OK;
}

int32_t rf_batch_step(RfBatch* b, double target_dt_days, RfStepReport* reports) {
  if (!b || !reports || !(target_dt_days > 0.0) || !std::isfinite(target_dt_days)) return RF_ERR_INVALID;
  const int n = int(b->ctx.size());
  std::vector<int32_t> rcs(n, RF_OK);
  if (b->mode == RF_BATCH_GROUPS) {
    std::vector<StepJob> jobs(n);
    for (int i = 0; i < n; ++i) jobs[i] = {b->ctx[i], target_dt_days, &reports[i], RF_OK};
    auto run_group = [&](rf::BatchGroup* g) {
      cudaSetDevice(b->device);
      std::vector<void*> args;
      for (int i : g->members) args.push_back(&jobs[i]);
      g->failed = false;
      rf::run_fibers(*g, step_job, args.data(), int(args.size()), kFiberStack);
      if (g->failed)
        for (int i : g->members) {
          jobs[i].rc = RF_ERR_CUDA;
          b->ctx[i]->c.err = "a batched launch of the variant's group failed";
        }
    };
    std::vector<std::thread> pool;
    for (size_t k = 1; k < b->groups.size(); ++k) pool.emplace_back(run_group, b->groups[k].get());
    if (!b->groups.empty()) run_group(b->groups[0].get());
    for (auto& t : pool) t.join();
    for (int i = 0; i < n; ++i) rcs[i] = jobs[i].rc;
  } else {
    std::atomic<int> next{0};
    auto work = [&]() {
      cudaSetDevice(b->device);
      for (int k = next.fetch_add(1); k < n; k = next.fetch_add(1)) {
        const int i = b->order[k];
        rcs[i] = rf_step(b->ctx[i], target_dt_days, &reports[i]);
      }
    };
    std::vector<std::thread> pool;
    const int extra = std::min(b->threads, n) - 1;
    for (int t = 0; t < extra; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
  }
  int32_t worst = RF_OK;
  for (int i = 0; i < n; ++i) {
    if (rcs[i] < 0) return rcs[i];
    if (rcs[i] > worst) worst = rcs[i];
  }
  return worst;
}

}  // extern "C"
