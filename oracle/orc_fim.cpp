// ORACLE — test infrastructure only (see orc_core.hpp).  Assembly, well Schur elimination,
// CPR-FGMRES with block-ILU0, the OPM-aligned Newton loop, the OPM timestep controller and the
// rate reporting of the reference FIM path, restated single-threaded on the CPU.
//
// Reference files followed (paths inside the reference project, src/lib/ressim/src/):
//   fim/assembly_ad.rs:239-983        residual/Jacobian assembly
//   fim/scaling.rs:139-223            equation/variable scaling
//   fim/newton.rs:970-3360            Newton driver (OpmAligned branches)
//   fim/newton/convergence.rs         norms, CNV/MB, per-cell chop
//   fim/newton/damping.rs:651-766     oscillation relaxation
//   fim/state.rs                      state init, update application, well relaxation
//   fim/linear/mod.rs:252-372         linear dispatch
//   fim/linear/well_schur.rs          well elimination and recovery
//   fim/linear/gmres_block_jacobi.rs  CPR build/apply, block-ILU0, pressure ILU0, BiCGStab, FGMRES
//   fim/timestep.rs:423-529,631-659,989-1848   outer controller
//   reporting.rs:553-734              per-substep rates and material balance
#include <cstdio>
#include <memory>
#include <set>
#include <string>

#include "orc_physics.hpp"

namespace orc {

// ============================================================================================
// Assembly
// ============================================================================================
struct EqScaling {
  std::vector<double> water, oil, gas, well, perf;
};
struct VarScaling {
  std::vector<double> p, sw, hc, bhp, q;
};
struct Assembly {
  std::vector<double> residual;
  Csr jac;
  EqScaling eq;
  VarScaling var;
};

static double well_constraint_scale(const Sim& s, const State& st, int w) {
  const Control c = physical_well_control(s, w);
  // control_slacks is Some exactly when the well is enabled, rate controlled and has a target.
  const bool slacks = c.enabled && c.rate_controlled && c.has_target;
  return slacks ? 1.0 : rmax(std::fabs(st.bhp[w]), 1.0);
}

static EqScaling build_equation_scaling(const Sim& s, const State& st, double dt) {
  EqScaling e;
  dt = rmax(dt, 1e-12);
  for (int i = 0; i < st.n_cells(); ++i) {
    const double pv_over_dt = rmax(std::fabs(s.pore_volume_m3(i) / dt), 1.0);
    const double p = st.cells[i].p;
    const double bo = rmax(get_b_o_cell(s, i, p), 1e-9);
    const double bg = rmax(get_b_g(s, p), 1e-9);
    const double bw = water_fvf(s, p);
    e.water.push_back(pv_over_dt / bw);
    e.oil.push_back(pv_over_dt / bo);
    e.gas.push_back(pv_over_dt / bg);
  }
  for (int w = 0; w < int(st.bhp.size()); ++w) e.well.push_back(well_constraint_scale(s, st, w));
  for (double q : st.q) e.perf.push_back(rmax(std::fabs(q), 1.0));
  return e;
}

static VarScaling build_variable_scaling(const State& st) {
  VarScaling v;
  for (const Cell& c : st.cells) {
    v.p.push_back(rmax(std::fabs(c.p), 1.0));
    v.sw.push_back(1.0);
    v.hc.push_back(c.regime == 0 ? 1.0 : rmax(std::fabs(c.hc), 1.0));
  }
  for (double b : st.bhp) v.bhp.push_back(rmax(std::fabs(b), 1.0));
  for (double q : st.q) v.q.push_back(rmax(std::fabs(q), 1.0));
  return v;
}

static inline void add_if_nonzero(std::vector<Trip>& t, int r, int c, double v) {
  if (std::fabs(v) > 1e-14) t.push_back({r, c, v});
}
static inline void scatter_block(std::vector<Trip>& t, int rc, int cc, const double b[3][3]) {
  for (int e = 0; e < 3; ++e)
    for (int v = 0; v < 3; ++v)
      if (std::fabs(b[e][v]) > 1e-14) t.push_back({3 * rc + e, 3 * cc + v, b[e][v]});
}

template <class S>
struct PerfInput {
  WellCell<S> cell;
  bool has_frac;
  Fractions<S> frac;
  S q;
};

template <class S>
static S well_actual_rate_g(const Sim& s, bool inj, bool surface, const std::vector<PerfInput<S>>& perfs) {
  S total = sc<S>(0.0);
  for (const auto& pi : perfs) {
    total = total + (surface ? perforation_surface_rate_g(s, inj, pi.cell, pi.has_frac ? &pi.frac : nullptr, pi.q)
                             : perforation_reservoir_rate_g(inj, pi.q));
  }
  return total;
}

static void add_well_residual_terms(const Sim& s, const State& st, double dt, std::vector<double>& r) {
  std::vector<std::vector<PerfInput<double>>> inputs(s.topo.wells.size());
  for (int perf = 0; perf < int(s.topo.perfs.size()); ++perf) {
    const Perf& pf = s.topo.perfs[perf];
    const Cell& c = st.cells[pf.cell];
    WellCell<double> wc{c.p, c.sw, c.hc, c.regime, c.base_rs};
    const double bhp = st.bhp[pf.well];
    const double q = st.q[perf];
    PerfInput<double> pi{wc, !pf.injector, {}, q};
    if (!pf.injector) pi.frac = producer_fractions_g<double>(s, wc);
    inputs[pf.well].push_back(pi);
    double coef[3];
    component_coefficients_g<double>(s, pf.injector, wc, pi.has_frac ? &pi.frac : nullptr, coef);
    for (int e = 0; e < 3; ++e) r[3 * pf.cell + e] += coef[e] * q * dt;
    if (pf.has_wi) {
      const double conn = connection_rate_g<double>(s, pf.wi, s.head_offset[pf.entry], pf.injector, wc, bhp);
      r[st.q_off(perf)] += q - conn;
    }
  }
  for (int w = 0; w < int(s.topo.wells.size()); ++w) {
    const bool inj = s.topo.wells[w].injector;
    const Control c = physical_well_control(s, w);
    const double bhp = st.bhp[w];
    if (!c.enabled || !c.rate_controlled) {
      r[st.bhp_off(w)] += bhp - c.bhp_target;
      continue;
    }
    if (!c.has_target) continue;
    const double actual = well_actual_rate_g<double>(s, inj, c.uses_surface_target, inputs[w]);
    const double bhp_slack = inj ? c.bhp_limit - bhp : bhp - c.bhp_limit;
    const double rate_slack = c.target_rate - actual;
    const double bs = rmax(std::fabs(c.bhp_limit), 1.0), rsc = rmax(std::fabs(c.target_rate), 1.0);
    r[st.bhp_off(w)] += fischer_burmeister_g<double>(bhp_slack / bs, rate_slack / rsc);
  }
}

static void add_well_jacobian_terms(const Sim& s, const State& st, double dt, std::vector<Trip>& t) {
  std::vector<std::vector<PerfInput<double>>> inputs(s.topo.wells.size());
  for (int perf = 0; perf < int(s.topo.perfs.size()); ++perf) {
    const Perf& pf = s.topo.perfs[perf];
    const Cell& c = st.cells[pf.cell];
    WellCell<double> wc{c.p, c.sw, c.hc, c.regime, c.base_rs};
    const double bhp = st.bhp[pf.well];
    const double q = st.q[perf];
    PerfInput<double> pi{wc, !pf.injector, {}, q};
    if (!pf.injector) pi.frac = producer_fractions_g<double>(s, wc);
    inputs[pf.well].push_back(pi);
    const int prow = st.q_off(perf), qcol = st.q_off(perf), bcol = st.bhp_off(pf.well);
    WellCell<Ad<4>> ca{ad_var<4>(c.p, 0), ad_var<4>(c.sw, 1), ad_var<4>(c.hc, 2), c.regime, c.base_rs};
    if (pf.has_wi) {
      Ad<4> conn = connection_rate_g<Ad<4>>(s, pf.wi, s.head_offset[pf.entry], pf.injector, ca,
                                            ad_var<4>(bhp, 3));
      t.push_back({prow, qcol, 1.0});
      add_if_nonzero(t, prow, 3 * pf.cell + 0, -conn.d[0]);
      add_if_nonzero(t, prow, 3 * pf.cell + 1, -conn.d[1]);
      add_if_nonzero(t, prow, 3 * pf.cell + 2, -conn.d[2]);
      add_if_nonzero(t, prow, bcol, -conn.d[3]);
    }
    Ad<4> qa = ad_var<4>(q, 3);
    Fractions<Ad<4>> fa;
    if (!pf.injector) fa = producer_fractions_g<Ad<4>>(s, ca);
    Ad<4> coef[3];
    component_coefficients_g<Ad<4>>(s, pf.injector, ca, pf.injector ? nullptr : &fa, coef);
    for (int e = 0; e < 3; ++e) {
      Ad<4> row = coef[e] * qa;
      const int er = 3 * pf.cell + e;
      for (int v = 0; v < 3; ++v) add_if_nonzero(t, er, 3 * pf.cell + v, row.d[v] * dt);
      add_if_nonzero(t, er, qcol, row.d[3] * dt);
    }
  }
  for (int w = 0; w < int(s.topo.wells.size()); ++w) {
    const bool inj = s.topo.wells[w].injector;
    const Control c = physical_well_control(s, w);
    const double bhp = st.bhp[w];
    const int row = st.bhp_off(w), bcol = st.bhp_off(w);
    if (!c.enabled || !c.rate_controlled) {
      t.push_back({row, bcol, 1.0});
      continue;
    }
    if (!c.has_target) continue;
    const double actual = well_actual_rate_g<double>(s, inj, c.uses_surface_target, inputs[w]);
    const double bhp_slack = inj ? c.bhp_limit - bhp : bhp - c.bhp_limit;
    const double rate_slack = c.target_rate - actual;
    const double bs = rmax(std::fabs(c.bhp_limit), 1.0), rsc = rmax(std::fabs(c.target_rate), 1.0);
    double da, db;
    fischer_burmeister_gradient(bhp_slack / bs, rate_slack / rsc, da, db);
    const double dslack = inj ? -1.0 : 1.0;
    add_if_nonzero(t, row, bcol, da * dslack / bs);
    const double factor = -db / rsc;
    for (int perf : s.topo.wells[w].perfs) {
      const Perf& pf = s.topo.perfs[perf];
      const Cell& cc = st.cells[pf.cell];
      WellCell<Ad<4>> ca{ad_var<4>(cc.p, 0), ad_var<4>(cc.sw, 1), ad_var<4>(cc.hc, 2), cc.regime, cc.base_rs};
      Ad<4> qa = ad_var<4>(st.q[perf], 3);
      Ad<4> rate;
      if (c.uses_surface_target) {
        Fractions<Ad<4>> fa;
        if (!inj) fa = producer_fractions_g<Ad<4>>(s, ca);
        rate = perforation_surface_rate_g<Ad<4>>(s, inj, ca, inj ? nullptr : &fa, qa);
      } else {
        rate = perforation_reservoir_rate_g<Ad<4>>(inj, qa);
      }
      for (int v = 0; v < 3; ++v) add_if_nonzero(t, row, 3 * pf.cell + v, factor * rate.d[v]);
      add_if_nonzero(t, row, st.q_off(perf), factor * rate.d[3]);
    }
  }
}

static Assembly assemble(const Sim& s, const State& prev, const State& st, double dt, bool residual_only) {
  Assembly a;
  const int n = st.n_cells();
  a.eq = build_equation_scaling(s, st, dt);
  a.var = build_variable_scaling(st);
  a.residual.assign(st.n_unknowns(), 0.0);
  auto& r = a.residual;
  for (int c = 0; c < n; ++c) {
    const Cell& x = st.cells[c];
    const Cell& px = prev.cells[c];
    double acc[3];
    cell_accumulation_g<double>(s, c, x.regime, x.p, x.sw, x.hc, px.p, px.sw, px.hc, px.regime, acc, x.base_rs);
    for (int e = 0; e < 3; ++e) r[3 * c + e] += acc[e];
  }
  auto face_res = [&](int i, int j, char dim, int ki, int kj) {
    const double gt = DARCY_METRIC_FACTOR * geometric_transmissibility(s, i, j, dim);
    if (gt <= 0.0) return;
    FaceIn<double> fi{st.cells[i].p, st.cells[i].sw, st.cells[i].hc, s.depth_at_k(ki), st.cells[i].regime,
                      st.cells[i].base_rs};
    FaceIn<double> fj{st.cells[j].p, st.cells[j].sw, st.cells[j].hc, s.depth_at_k(kj), st.cells[j].regime,
                      st.cells[j].base_rs};
    double f[3];
    face_flux_g<double>(s, gt, fi, fj, f);
    for (int e = 0; e < 3; ++e) {
      r[3 * i + e] += f[e] * dt;
      r[3 * j + e] += -f[e] * dt;
    }
  };
  for (int k = 0; k < s.nz; ++k)
    for (int j = 0; j < s.ny; ++j)
      for (int i = 0; i < s.nx; ++i) {
        const int id = s.idx(i, j, k);
        if (i + 1 < s.nx) face_res(id, s.idx(i + 1, j, k), 'x', k, k);
        if (j + 1 < s.ny) face_res(id, s.idx(i, j + 1, k), 'y', k, k);
        if (k + 1 < s.nz) face_res(id, s.idx(i, j, k + 1), 'z', k, k + 1);
      }
  add_well_residual_terms(s, st, dt, r);
  if (residual_only) return a;

  std::vector<Trip> t;
  t.reserve(size_t(n) * 9 * 7 + 64);
  for (int c = 0; c < n; ++c) {
    const Cell& x = st.cells[c];
    const Cell& px = prev.cells[c];
    Ad<3> acc[3];
    cell_accumulation_g<Ad<3>>(s, c, x.regime, ad_var<3>(x.p, 0), ad_var<3>(x.sw, 1), ad_var<3>(x.hc, 2), px.p,
                               px.sw, px.hc, px.regime, acc, x.base_rs);
    double b[3][3];
    for (int e = 0; e < 3; ++e)
      for (int v = 0; v < 3; ++v) b[e][v] = acc[e].d[v];
    scatter_block(t, c, c, b);
  }
  auto face_jac = [&](int i, int j, char dim, int ki, int kj) {
    const double gt = DARCY_METRIC_FACTOR * geometric_transmissibility(s, i, j, dim);
    if (gt <= 0.0) return;
    FaceIn<Ad<6>> fi{ad_var<6>(st.cells[i].p, 0), ad_var<6>(st.cells[i].sw, 1), ad_var<6>(st.cells[i].hc, 2),
                     s.depth_at_k(ki), st.cells[i].regime, st.cells[i].base_rs};
    FaceIn<Ad<6>> fj{ad_var<6>(st.cells[j].p, 3), ad_var<6>(st.cells[j].sw, 4), ad_var<6>(st.cells[j].hc, 5),
                     s.depth_at_k(kj), st.cells[j].regime, st.cells[j].base_rs};
    Ad<6> f[3];
    face_flux_g<Ad<6>>(s, gt, fi, fj, f);
    double bii[3][3], bij[3][3], bji[3][3], bjj[3][3];
    for (int e = 0; e < 3; ++e)
      for (int v = 0; v < 3; ++v) {
        bii[e][v] = f[e].d[v] * dt;
        bij[e][v] = f[e].d[3 + v] * dt;
        bji[e][v] = -f[e].d[v] * dt;
        bjj[e][v] = -f[e].d[3 + v] * dt;
      }
    scatter_block(t, i, i, bii);
    scatter_block(t, i, j, bij);
    scatter_block(t, j, i, bji);
    scatter_block(t, j, j, bjj);
  };
  for (int k = 0; k < s.nz; ++k)
    for (int j = 0; j < s.ny; ++j)
      for (int i = 0; i < s.nx; ++i) {
        const int id = s.idx(i, j, k);
        if (i + 1 < s.nx) face_jac(id, s.idx(i + 1, j, k), 'x', k, k);
        if (j + 1 < s.ny) face_jac(id, s.idx(i, j + 1, k), 'y', k, k);
        if (k + 1 < s.nz) face_jac(id, s.idx(i, j, k + 1), 'z', k, k + 1);
      }
  add_well_jacobian_terms(s, st, dt, t);
  a.jac = to_csr(st.n_unknowns(), t);
  return a;
}

// ============================================================================================
// Linear solve: CPR-FGMRES with block-ILU0 (tail-free systems) + well Schur elimination
// ============================================================================================
struct LinReport {
  std::vector<double> x;
  bool converged = false;
  int iterations = 0;
  double rhs_norm = 0, final_residual_norm = 0;
  bool used_fallback = false;  // direct route did not converge; CPR-FGMRES result
  int backend = 0;             // 0: CPR-FGMRES, 1: direct LU
  double reduction() const { return final_residual_norm / rmax(rhs_norm, 1e-30); }
};

struct Blk {
  double a[9];
};
static inline void blk_mul(const Blk& x, const Blk& y, Blk& z) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) z.a[3 * r + c] = x.a[3 * r] * y.a[c] + x.a[3 * r + 1] * y.a[3 + c] + x.a[3 * r + 2] * y.a[6 + c];
}
static inline Blk blk_inverse_or_diag(const Blk& b) {
  Dense d(3);
  for (int i = 0; i < 9; ++i) d.a[i] = b.a[i];
  Dense inv = invert_or_diag(d);
  Blk o;
  for (int i = 0; i < 9; ++i) o.a[i] = inv.a[i];
  return o;
}

// factorize_block_ilu0 / FimBlockIlu0Factors::apply (gmres_block_jacobi.rs:178-353)
struct BlockIlu {
  int nb = 0;
  std::vector<std::vector<std::pair<int, Blk>>> l, u;
  std::vector<Blk> dinv;
  void factor(const Csr& m) {
    nb = m.n / 3;
    std::vector<std::map<int, Blk>> rows(nb);
    for (int rb = 0; rb < nb; ++rb) {
      std::set<int> cols;
      cols.insert(rb);
      for (int loc = 0; loc < 3; ++loc) {
        const int r = 3 * rb + loc;
        for (int k = m.ptr[r]; k < m.ptr[r + 1]; ++k) {
          if (m.col[k] >= 3 * nb || std::fabs(m.val[k]) <= F64_EPS) continue;
          cols.insert(m.col[k] / 3);
        }
      }
      for (int cb : cols) {
        Blk b;
        for (int rr = 0; rr < 3; ++rr)
          for (int cc = 0; cc < 3; ++cc) b.a[3 * rr + cc] = m.at(3 * rb + rr, 3 * cb + cc);
        rows[rb][cb] = b;
      }
    }
    l.assign(nb, {});
    u.assign(nb, {});
    dinv.assign(nb, Blk{});
    for (int i = 0; i < nb; ++i) {
      std::vector<int> ks;
      for (auto& kv : rows[i])
        if (kv.first < i) ks.push_back(kv.first);
      for (int k : ks) {
        Blk lik;
        blk_mul(rows[i][k], dinv[k], lik);
        for (auto& ukj : u[k]) {
          auto it = rows[i].find(ukj.first);
          if (it != rows[i].end()) {
            Blk prod;
            blk_mul(lik, ukj.second, prod);
            for (int e = 0; e < 9; ++e) it->second.a[e] -= prod.a[e];
          }
        }
        l[i].push_back({k, lik});
        rows[i].erase(k);
      }
      Blk diag{};
      auto it = rows[i].find(i);
      if (it != rows[i].end()) diag = it->second;
      dinv[i] = blk_inverse_or_diag(diag);
      for (auto& kv : rows[i])
        if (kv.first > i) u[i].push_back(kv);
    }
  }
  void apply(const std::vector<double>& rhs, std::vector<double>& out) const {
    std::vector<double> y(3 * nb);
    for (int i = 0; i < nb; ++i) {
      double b[3] = {rhs[3 * i], rhs[3 * i + 1], rhs[3 * i + 2]};
      for (auto& kb : l[i]) {
        const double* yk = &y[3 * kb.first];
        for (int r = 0; r < 3; ++r) b[r] -= kb.second.a[3 * r] * yk[0] + kb.second.a[3 * r + 1] * yk[1] + kb.second.a[3 * r + 2] * yk[2];
      }
      for (int r = 0; r < 3; ++r) y[3 * i + r] = b[r];
    }
    out.assign(3 * nb, 0.0);
    for (int i = nb - 1; i >= 0; --i) {
      double b[3] = {y[3 * i], y[3 * i + 1], y[3 * i + 2]};
      for (auto& jb : u[i]) {
        const double* xj = &out[3 * jb.first];
        for (int r = 0; r < 3; ++r) b[r] -= jb.second.a[3 * r] * xj[0] + jb.second.a[3 * r + 1] * xj[1] + jb.second.a[3 * r + 2] * xj[2];
      }
      const Blk& d = dinv[i];
      for (int r = 0; r < 3; ++r) out[3 * i + r] = d.a[3 * r] * b[0] + d.a[3 * r + 1] * b[1] + d.a[3 * r + 2] * b[2];
    }
  }
};

// CPR preconditioner for a tail-free 3x3 block system (build_block_jacobi_preconditioner with
// BlockIlu0 smoother and QuasiImpes restriction, gmres_block_jacobi.rs:919-1363).
struct Cpr {
  int nb = 0;
  std::vector<std::array<double, 3>> restriction;  // prolongation is [1,0,0]
  std::vector<std::vector<std::pair<int, double>>> prow;  // coarse rows
  bool has_dense = false;
  Dense dense_inv;
  std::vector<std::vector<std::pair<int, double>>> pl, pu;
  std::vector<double> pdiag;
  BlockIlu ilu;

  void build(const Csr& m) {
    nb = m.n / 3;
    restriction.assign(nb, {0, 0, 0});
    for (int b = 0; b < nb; ++b) {
      Dense blk(3);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) blk(r, c) = m.at(3 * b + r, 3 * b + c);
      Dense inv = invert_or_diag(blk);
      double w[3] = {inv(0, 0), inv(0, 1), inv(0, 2)};
      double mx = 0.0;
      for (double x : w) mx = rmax(mx, std::fabs(x));
      if (mx > F64_EPS)
        for (double& x : w) x /= mx;
      restriction[b] = {w[0], w[1], w[2]};
    }
    prow.assign(nb, {});
    for (int b = 0; b < nb; ++b) {
      std::map<int, double> coef;
      for (int loc = 0; loc < 3; ++loc) {
        const double wt = restriction[b][loc];
        if (std::fabs(wt) <= F64_EPS) continue;
        const int r = 3 * b + loc;
        for (int k = m.ptr[r]; k < m.ptr[r + 1]; ++k) {
          const int col = m.col[k];
          if (col % 3 != 0) continue;  // prolongation weight zero for sw/hc columns
          coef[col / 3] += wt * m.val[k] * 1.0;
        }
      }
      for (auto& kv : coef)
        if (std::fabs(kv.second) > 1e-14) prow[b].push_back(kv);
    }
    has_dense = false;
    if (nb > 0 && nb <= 299) {
      Dense pm(nb);
      for (int r = 0; r < nb; ++r)
        for (auto& kv : prow[r]) pm(r, kv.first) = kv.second;
      has_dense = try_inverse(pm, dense_inv);
    }
    // factorize_pressure_ilu0 (gmres_block_jacobi.rs:746-808)
    pl.assign(nb, {});
    pu.assign(nb, {});
    pdiag.assign(nb, 1.0);
    auto row_entry = [](const std::vector<std::pair<int, double>>& e, int c) {
      auto it = std::lower_bound(e.begin(), e.end(), c, [](const std::pair<int, double>& a, int b) { return a.first < b; });
      return (it != e.end() && it->first == c) ? it->second : 0.0;
    };
    for (int r = 0; r < nb; ++r) {
      double diag_entry = 0.0;
      std::vector<std::pair<int, double>> lower, upper;
      for (auto& kv : prow[r]) {
        if (kv.first < r)
          lower.push_back(kv);
        else if (kv.first == r)
          diag_entry = kv.second;
        else
          upper.push_back(kv);
      }
      for (auto& kv : lower) {
        double s = kv.second;
        for (auto& lk : pl[r]) {
          if (lk.first >= kv.first) break;
          s -= lk.second * row_entry(pu[lk.first], kv.first);
        }
        const double d = pdiag[kv.first];
        pl[r].push_back({kv.first, std::fabs(d) > F64_EPS ? s / d : 0.0});
      }
      double ud = diag_entry;
      for (auto& lk : pl[r]) ud -= lk.second * row_entry(pu[lk.first], r);
      if (std::fabs(ud) <= F64_EPS) ud = std::fabs(diag_entry) > F64_EPS ? diag_entry : 1.0;
      pdiag[r] = ud;
      for (auto& kv : upper) {
        double s = kv.second;
        for (auto& lk : pl[r]) s -= lk.second * row_entry(pu[lk.first], kv.first);
        pu[r].push_back({kv.first, s});
      }
    }
    ilu.factor(m);
  }

  void pmatvec(const std::vector<double>& x, std::vector<double>& y) const {
    y.assign(nb, 0.0);
    for (int r = 0; r < nb; ++r) {
      double s = 0.0;
      for (auto& kv : prow[r]) s += kv.second * x[kv.first];
      y[r] = s;
    }
  }
  void pilu(const std::vector<double>& rhs, std::vector<double>& x) const {
    std::vector<double> y(nb);
    for (int r = 0; r < nb; ++r) {
      double s = rhs[r];
      for (auto& kv : pl[r]) s -= kv.second * y[kv.first];
      y[r] = s;
    }
    x.assign(nb, 0.0);
    for (int r = nb - 1; r >= 0; --r) {
      double s = y[r];
      for (auto& kv : pu[r]) s -= kv.second * x[kv.first];
      const double d = pdiag[r];
      x[r] = std::fabs(d) > F64_EPS ? s / d : s;
    }
  }
  // solve_pressure_with_bicgstab (gmres_block_jacobi.rs:660-729)
  std::vector<double> bicgstab(const std::vector<double>& rhs, int max_iters, double tol) const {
    const int n = nb;
    std::vector<double> x(n, 0.0), r = rhs, tmp;
    // r = rhs - A*0 = rhs
    pmatvec(x, tmp);
    for (int i = 0; i < n; ++i) r[i] = rhs[i] - tmp[i];
    if (vnorm(r) <= tol) return x;
    const std::vector<double> rh = r;
    double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
    std::vector<double> v(n, 0.0), p(n, 0.0), ph, s(n), sh, t;
    for (int it = 0; it < max_iters; ++it) {
      const double rho = vdot(rh, r);
      if (!std::isfinite(rho) || std::fabs(rho) < F64_EPS) break;
      if (it == 0) {
        p = r;
      } else {
        const double beta = (rho / rho_prev) * (alpha / omega);
        for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
      }
      pilu(p, ph);
      pmatvec(ph, v);
      const double vd = vdot(rh, v);
      if (!std::isfinite(vd) || std::fabs(vd) < F64_EPS) break;
      alpha = rho / vd;
      for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
      if (vnorm(s) <= tol) {
        for (int i = 0; i < n; ++i) x[i] += alpha * ph[i];
        break;
      }
      pilu(s, sh);
      pmatvec(sh, t);
      const double tt = vdot(t, t);
      if (!std::isfinite(tt) || tt <= F64_EPS) break;
      omega = vdot(t, s) / tt;
      if (!std::isfinite(omega) || std::fabs(omega) < F64_EPS) break;
      for (int i = 0; i < n; ++i) x[i] += alpha * ph[i] + omega * sh[i];
      for (int i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
      if (vnorm(r) <= tol) break;
      rho_prev = rho;
    }
    return x;
  }

  // BlockJacobiPreconditioner::apply with pressure correction (gmres_block_jacobi.rs:471-583)
  void apply(const Csr& m, const std::vector<double>& vec, std::vector<double>& out) const {
    out.assign(vec.size(), 0.0);
    std::vector<double> prhs(nb);
    for (int b = 0; b < nb; ++b) {
      double v = 0.0;
      for (int loc = 0; loc < 3; ++loc) v += restriction[b][loc] * vec[3 * b + loc];
      prhs[b] = v;
    }
    std::vector<double> corr;
    if (has_dense) {
      corr.assign(nb, 0.0);
      for (int r = 0; r < nb; ++r) {
        double s = 0.0;
        for (int c = 0; c < nb; ++c) s += dense_inv(r, c) * prhs[c];
        corr[r] = s;
      }
    } else {
      const double tol = rmax(vnorm(prhs), F64_EPS) * 1e-6;
      corr = bicgstab(prhs, 50, tol);
    }
    for (int b = 0; b < nb; ++b) out[3 * b] += 1.0 * corr[b];
    std::vector<double> ax;
    csr_matvec(m, out, ax);
    std::vector<double> cr(vec.size());
    for (size_t i = 0; i < vec.size(); ++i) cr[i] = vec[i] - ax[i];
    std::vector<double> sm;
    ilu.apply(cr, sm);
    for (size_t i = 0; i < vec.size(); ++i) out[i] += sm[i];
  }
};

// run_true_flexible_gmres (gmres_block_jacobi.rs:1470-1665)
static LinReport fgmres(const Csr& m, const std::vector<double>& rhs, const Cpr& pc) {
  LinReport rep;
  const int n = m.n;
  rep.rhs_norm = vnorm(rhs);
  const double tol = 1e-12 + 5e-3 * rmax(rep.rhs_norm, F64_EPS);
  const int restart = 30, max_it = std::max(20, restart);
  std::vector<double> sol(n, 0.0), ax;
  int iters = 0;
  while (iters < max_it) {
    csr_matvec(m, sol, ax);
    std::vector<double> res(n);
    for (int i = 0; i < n; ++i) res[i] = rhs[i] - ax[i];
    const double rn = vnorm(res);
    if (rn <= tol) {
      rep.x = sol;
      rep.converged = true;
      rep.iterations = iters;
      rep.final_residual_norm = rn;
      return rep;
    }
    const double beta = rn;
    const int cyc = std::min(restart, max_it - iters);
    std::vector<std::vector<double>> V, Z;
    V.push_back(res);
    for (double& x : V[0]) x /= beta;
    Dense H(cyc + 1);
    std::vector<double> cs(cyc, 0.0), sn(cyc, 0.0), g(cyc + 1, 0.0);
    g[0] = beta;
    const std::vector<double> origin = sol;
    std::vector<double> cand = origin;
    for (int j = 0; j < cyc; ++j) {
      std::vector<double> z, w;
      pc.apply(m, V[j], z);
      csr_matvec(m, z, w);
      Z.push_back(z);
      for (int p = 0; p <= j; ++p) {
        const double h = vdot(V[p], w);
        H(p, j) = h;
        for (int i = 0; i < n; ++i) w[i] -= V[p][i] * h;
      }
      const double nn = vnorm(w);
      H(j + 1, j) = nn;
      if (nn > F64_EPS) {
        for (double& x : w) x /= nn;
        V.push_back(w);
      }
      for (int p = 0; p < j; ++p) {
        const double a = H(p, j), b = H(p + 1, j);
        H(p, j) = cs[p] * a + sn[p] * b;
        H(p + 1, j) = -sn[p] * a + cs[p] * b;
      }
      const double a = H(j, j), b = H(j + 1, j);
      const double rad = std::hypot(a, b);
      double c, s;
      if (rad <= F64_EPS) {
        c = 1.0;
        s = 0.0;
      } else {
        c = a / rad;
        s = b / rad;
      }
      cs[j] = c;
      sn[j] = s;
      H(j, j) = c * a + s * b;
      H(j + 1, j) = -s * a + c * b;
      const double g0 = g[j], g1 = g[j + 1];
      g[j] = c * g0 + s * g1;
      g[j + 1] = -s * g0 + c * g1;
      ++iters;
      const int cols = j + 1;
      std::vector<double> y(cols, 0.0);
      for (int r = cols - 1; r >= 0; --r) {
        double sum = g[r];
        for (int cc = r + 1; cc < cols; ++cc) sum -= H(r, cc) * y[cc];
        const double d = H(r, r);
        y[r] = std::fabs(d) > F64_EPS ? sum / d : 0.0;
      }
      std::vector<double> upd(n, 0.0);
      for (int cc = 0; cc < cols; ++cc)
        for (int i = 0; i < n; ++i) upd[i] += Z[cc][i] * y[cc];
      for (int i = 0; i < n; ++i) cand[i] = origin[i] + upd[i];
      csr_matvec(m, cand, ax);
      std::vector<double> cres(n);
      for (int i = 0; i < n; ++i) cres[i] = rhs[i] - ax[i];
      const double trn = vnorm(cres);
      if (trn <= tol) {
        rep.x = cand;
        rep.converged = true;
        rep.iterations = iters;
        rep.final_residual_norm = trn;
        return rep;
      }
      if (nn <= F64_EPS || iters >= max_it) {
        rep.x = cand;
        rep.converged = false;
        rep.iterations = iters;
        rep.final_residual_norm = trn;
        return rep;
      }
    }
    sol = cand;
  }
  csr_matvec(m, sol, ax);
  std::vector<double> res(n);
  for (int i = 0; i < n; ++i) res[i] = rhs[i] - ax[i];
  rep.x = sol;
  rep.converged = false;
  rep.iterations = iters;
  rep.final_residual_norm = vnorm(res);
  return rep;
}

// Test-only refinement of every CPR-FGMRES solve, mirroring the device path's
// rf_set_linear_refinement (no counterpart in the reference): x += fgmres(b - A x) with the CPR of
// the first pass until |b - A x| <= g_lin_refine_rtol |b|, at most g_lin_refine_passes solves;
// 0 keeps the reference's single solve.
static double g_lin_refine_rtol = 0.0;
static int g_lin_refine_passes = 12;

static LinReport solve_tail_free(const Csr& m, const std::vector<double>& rhs) {
  Cpr pc;
  pc.build(m);
  if (g_lin_refine_rtol <= 0.0) return fgmres(m, rhs, pc);
  const int n = m.n;
  LinReport rep;
  rep.rhs_norm = vnorm(rhs);
  std::vector<double> x(n, 0.0), ax, r(n);
  for (int pass = 0;; ++pass) {
    csr_matvec(m, x, ax);
    for (int i = 0; i < n; ++i) r[i] = rhs[i] - ax[i];
    const double rn = vnorm(r);
    rep.final_residual_norm = rn;
    if (!std::isfinite(rn)) break;
    if (rn <= g_lin_refine_rtol * rep.rhs_norm || rep.rhs_norm == 0.0) {
      rep.converged = true;
      break;
    }
    if (pass == g_lin_refine_passes) break;
    const LinReport in = fgmres(m, r, pc);
    rep.iterations += in.iterations;
    for (int i = 0; i < n; ++i) x[i] += in.x[i];
  }
  rep.x = x;
  return rep;
}

// solve_with_well_elimination (well_schur.rs:70-238, 382-471)
static LinReport solve_with_wells(const Csr& J, const std::vector<double>& rhs, int n_cells) {
  const int ws = 3 * n_cells;
  const int tail = J.n - ws;
  if (tail == 0) return solve_tail_free(J, rhs);
  Dense tb(tail);
  for (int r = 0; r < tail; ++r)
    for (int k = J.ptr[ws + r]; k < J.ptr[ws + r + 1]; ++k)
      if (J.col[k] >= ws) tb(r, J.col[k] - ws) = J.val[k];
  Dense tinv = invert_or_diag(tb);
  std::vector<std::vector<std::pair<int, double>>> jwr(tail);
  for (int r = 0; r < tail; ++r)
    for (int k = J.ptr[ws + r]; k < J.ptr[ws + r + 1]; ++k)
      if (J.col[k] < ws && std::fabs(J.val[k]) > F64_EPS) jwr[r].push_back({J.col[k], J.val[k]});
  std::vector<std::pair<int, std::vector<std::pair<int, double>>>> jrw;
  for (int r = 0; r < ws; ++r) {
    std::vector<std::pair<int, double>> e;
    for (int k = J.ptr[r]; k < J.ptr[r + 1]; ++k)
      if (J.col[k] >= ws && std::fabs(J.val[k]) > F64_EPS) e.push_back({J.col[k] - ws, J.val[k]});
    if (!e.empty()) jrw.push_back({r, e});
  }
  std::vector<double> tir(tail, 0.0);
  for (int r = 0; r < tail; ++r) {
    double s = 0.0;
    for (int c = 0; c < tail; ++c) s += tinv(r, c) * rhs[ws + c];
    tir[r] = s;
  }
  std::vector<double> rrhs(rhs.begin(), rhs.begin() + ws);
  for (auto& re : jrw) {
    double corr = 0.0;
    for (auto& tv : re.second) corr += tv.second * tir[tv.first];
    rrhs[re.first] -= corr;
  }
  std::vector<Trip> t;
  for (int r = 0; r < ws; ++r)
    for (int k = J.ptr[r]; k < J.ptr[r + 1]; ++k)
      if (J.col[k] < ws) t.push_back({r, J.col[k], J.val[k]});
  for (auto& re : jrw) {
    std::vector<double> w(tail, 0.0);
    for (auto& tv : re.second)
      for (int t2 = 0; t2 < tail; ++t2) w[t2] += tv.second * tinv(tv.first, t2);
    for (int t2 = 0; t2 < tail; ++t2) {
      if (std::fabs(w[t2]) <= F64_EPS) continue;
      for (auto& cv : jwr[t2]) t.push_back({re.first, cv.first, -w[t2] * cv.second});
    }
  }
  Csr red = to_csr(ws, t);
  LinReport rr = solve_tail_free(red, rrhs);
  // recover_full_solution
  std::vector<double> rt(tail);
  for (int r = 0; r < tail; ++r) {
    double s = 0.0;
    for (auto& cv : jwr[r]) s += cv.second * rr.x[cv.first];
    rt[r] = rhs[ws + r] - s;
  }
  std::vector<double> x(J.n, 0.0);
  for (int i = 0; i < ws; ++i) x[i] = rr.x[i];
  for (int r = 0; r < tail; ++r) {
    double s = 0.0;
    for (int c = 0; c < tail; ++c) s += tinv(r, c) * rt[c];
    x[ws + r] = s;
  }
  std::vector<double> ax;
  csr_matvec(J, x, ax);
  std::vector<double> fr(J.n);
  for (int i = 0; i < J.n; ++i) fr[i] = rhs[i] - ax[i];
  const double frn = vnorm(fr), rn = vnorm(rhs);
  const double tol = 1e-12 + 5e-3 * rmax(rn, F64_EPS);
  LinReport rep;
  rep.x = x;
  rep.converged = rr.converged && frn <= tol;
  rep.iterations = rr.iterations;
  rep.rhs_norm = rn;
  rep.final_residual_norm = frn;
  return rep;
}

// Direct route for small systems (fim/linear/mod.rs:15, 56-67, 262-300).  With the default
// FgmresCpr kind on the native target, a full system (cells, well BHPs and perforation rates) of
// at most 512 rows goes to the sparse direct LU of sparse_lu_debug.rs:148-232 (faer `sp_lu`,
// then at most two refinement solves, each kept only when it cuts the residual below 95 % of the
// previous one); when that does not converge, CPR-FGMRES with well elimination runs instead.
// faer 0.24.4 (Cargo.lock; not part of the reference tree) factors with partial pivoting behind a
// fill-reducing ordering.  This restatement factors densely with row partial pivoting (the first
// largest |a_ik| of the column wins), which gives the same solution up to rounding; an exactly
// zero pivot counts as a failed factorisation.  Storage is column-major and every element is
// updated in the order of the device's direct solver, so both produce the same bits.
constexpr int kDirectSolveRows = 512;

struct DenseLu {
  int n = 0;
  std::vector<double> a;  // column-major: a[j * n + i]; unit-lower L below the diagonal, U on and above
  std::vector<int> perm;  // row i of P A is row perm[i] of A
  bool ok = false;
};

static DenseLu dense_lu(const Csr& J) {
  DenseLu f;
  const int n = J.n;
  f.n = n;
  f.a.assign(size_t(n) * n, 0.0);
  f.perm.resize(n);
  for (int i = 0; i < n; ++i) {
    f.perm[i] = i;
    for (int k = J.ptr[i]; k < J.ptr[i + 1]; ++k) f.a[size_t(J.col[k]) * n + i] += J.val[k];
  }
  double* a = f.a.data();
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::fabs(a[size_t(k) * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(a[size_t(k) * n + i]) > best) {
        best = std::fabs(a[size_t(k) * n + i]);
        p = i;
      }
    if (!(best > 0.0)) return f;  // zero (or NaN) pivot column
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(a[size_t(j) * n + k], a[size_t(j) * n + p]);
      std::swap(f.perm[k], f.perm[p]);
    }
    const double piv = a[size_t(k) * n + k];
    for (int i = k + 1; i < n; ++i) a[size_t(k) * n + i] = a[size_t(k) * n + i] / piv;
    for (int j = k + 1; j < n; ++j) {
      const double u = a[size_t(j) * n + k];
      if (u == 0.0) continue;
      for (int i = k + 1; i < n; ++i) {
        const double l = a[size_t(k) * n + i];
        if (l != 0.0) a[size_t(j) * n + i] = a[size_t(j) * n + i] - l * u;
      }
    }
  }
  f.ok = true;
  return f;
}

// x = U^-1 L^-1 P b, both triangular solves column by column
static std::vector<double> dense_lu_solve(const DenseLu& f, const std::vector<double>& b) {
  const int n = f.n;
  const double* a = f.a.data();
  std::vector<double> y(n);
  for (int i = 0; i < n; ++i) y[i] = b[f.perm[i]];
  for (int k = 0; k < n; ++k) {
    const double yk = y[k];
    if (yk == 0.0) continue;
    for (int i = k + 1; i < n; ++i) y[i] = y[i] - a[size_t(k) * n + i] * yk;
  }
  for (int k = n - 1; k >= 0; --k) {
    y[k] = y[k] / a[size_t(k) * n + k];
    const double xk = y[k];
    if (xk == 0.0) continue;
    for (int i = 0; i < k; ++i) y[i] = y[i] - a[size_t(k) * n + i] * xk;
  }
  return y;
}

static bool all_finite(const std::vector<double>& v) {
  for (double x : v)
    if (!std::isfinite(x)) return false;
  return true;
}

// sparse_lu_debug.rs:148-232 (solve)
static LinReport direct_solve(const Csr& J, const std::vector<double>& rhs) {
  LinReport rep;
  const int n = J.n;
  rep.backend = 1;
  rep.rhs_norm = vnorm(rhs);
  const DenseLu f = dense_lu(J);
  if (!f.ok) {
    rep.x.assign(n, 0.0);
    rep.final_residual_norm = rep.rhs_norm;
    return rep;
  }
  const double tol = 1e-12 + 5e-3 * rmax(rep.rhs_norm, F64_EPS);
  auto residual_of = [&](const std::vector<double>& x) {
    std::vector<double> ax, r(n);
    csr_matvec(J, x, ax);
    for (int i = 0; i < n; ++i) r[i] = rhs[i] - ax[i];
    return r;
  };
  std::vector<double> x = dense_lu_solve(f, rhs);
  std::vector<double> r = residual_of(x);
  double rn = vnorm(r);
  int solves = rn > 0.0 ? 1 : 0;
  for (int it = 0; it < 2; ++it) {
    if (!std::isfinite(rn) || rn <= tol) break;
    const std::vector<double> c = dense_lu_solve(f, r);
    if (!all_finite(c)) break;
    std::vector<double> cand(n);
    for (int i = 0; i < n; ++i) cand[i] = x[i] + c[i];
    std::vector<double> cr = residual_of(cand);
    const double crn = vnorm(cr);
    if (!std::isfinite(crn) || crn >= rn * 0.95) break;
    x = cand;
    r = cr;
    rn = crn;
    ++solves;
  }
  rep.x = x;
  rep.converged = rn <= tol;
  rep.iterations = solves;
  rep.final_residual_norm = rn;
  return rep;
}

// solve_linearized_system_with_routing (fim/linear/mod.rs:262-300), native target, FgmresCpr
static LinReport solve_linearized(const Csr& J, const std::vector<double>& rhs, int n_cells) {
  if (J.n <= kDirectSolveRows) {
    LinReport d = direct_solve(J, rhs);
    if (d.converged) return d;
    LinReport it = solve_with_wells(J, rhs, n_cells);
    it.used_fallback = true;
    return it;
  }
  return solve_with_wells(J, rhs, n_cells);
}

// ============================================================================================
// Newton
// ============================================================================================
struct FamilyNorms {
  double w = INFINITY, o = INFINITY, g = INFINITY, well = INFINITY, perf = INFINITY;
};

static double scaled_residual_inf_norm(const std::vector<double>& r, const EqScaling& e, FamilyNorms* fam) {
  const int n = int(e.water.size());
  double mx = 0.0, fw = 0, fo = 0, fg = 0, fwell = 0, fperf = 0;
  for (int i = 0; i < n; ++i) {
    const double a = std::fabs(r[3 * i]) / e.water[i];
    const double b = std::fabs(r[3 * i + 1]) / e.oil[i];
    const double c = std::fabs(r[3 * i + 2]) / e.gas[i];
    fw = rmax(fw, a);
    fo = rmax(fo, b);
    fg = rmax(fg, c);
  }
  int off = 3 * n;
  for (size_t i = 0; i < e.well.size(); ++i) fwell = rmax(fwell, std::fabs(r[off + i]) / e.well[i]);
  off += int(e.well.size());
  for (size_t i = 0; i < e.perf.size(); ++i) fperf = rmax(fperf, std::fabs(r[off + i]) / e.perf[i]);
  mx = rmax(rmax(rmax(fw, fo), rmax(fg, fwell)), fperf);
  if (fam) {
    fam->w = fw;
    fam->o = fo;
    fam->g = fg;
    fam->well = e.well.empty() ? INFINITY : fwell;
    fam->perf = e.perf.empty() ? INFINITY : fperf;
  }
  return mx;
}

static double scaled_update_inf_norm(const std::vector<double>& u, const VarScaling& v) {
  const int n = int(v.p.size());
  double mx = 0.0;
  for (int i = 0; i < n; ++i) {
    mx = rmax(mx, std::fabs(u[3 * i]) / v.p[i]);
    mx = rmax(mx, std::fabs(u[3 * i + 1]) / v.sw[i]);
    mx = rmax(mx, std::fabs(u[3 * i + 2]) / v.hc[i]);
  }
  int off = 3 * n;
  for (size_t i = 0; i < v.bhp.size(); ++i) mx = rmax(mx, std::fabs(u[off + i]) / v.bhp[i]);
  off += int(v.bhp.size());
  for (size_t i = 0; i < v.q.size(); ++i) mx = rmax(mx, std::fabs(u[off + i]) / v.q[i]);
  return mx;
}

// damping.rs:715-766
static bool family_is_oscillating(double f0, double f1, double f2) {
  if (!(std::isfinite(f0) && std::isfinite(f1) && std::isfinite(f2)) || f0 <= 0.0) return false;
  const double d1 = std::fabs(f0 - f2) / f0, d2 = std::fabs(f0 - f1) / f0;
  return d1 < 0.2 && 0.2 < d2;
}
static int detect_oscillation(const FamilyNorms& c, const FamilyNorms& p1, const FamilyNorms& p2) {
  return int(family_is_oscillating(c.w, p1.w, p2.w)) + int(family_is_oscillating(c.o, p1.o, p2.o)) +
         int(family_is_oscillating(c.g, p1.g, p2.g)) + int(family_is_oscillating(c.well, p1.well, p2.well)) +
         int(family_is_oscillating(c.perf, p1.perf, p2.perf));
}

}  // namespace orc

// Exported known-answer hooks and the full Newton/timestep driver live in orc_driver.cpp.
#include "orc_driver.inc"
