// rf_blackoil_rows.cuh — one cell's, one perforation's and one well's residual and Jacobian rows
// in the three-phase black-oil mode, as __host__ __device__ functions: the kernels k_cells3,
// k_perfs3 and k_wells3 run them per thread, and a host build runs the same code on the CPU
// against the oracle's assembly.  Contributions follow the reference's triplet order
// (fim/assembly_ad.rs:782-983): accumulation, then faces z-, y-, x-, x+, y+, z+, then wells;
// Jacobian entries with |v| <= 1e-14 are dropped before they are added.
#pragma once

#include "rf_blackoil.cuh"

namespace rf {

RF_HD double filt3(double v) { return fabs(v) > 1e-14 ? v : 0.0; }

template <int DIR_SIGN>
RF_HD_CALL void face_contrib3(const Fluid& f, double trans, double dt, double depth_lo,
                         double depth_hi, int reg_lo, double p_lo, double sw_lo, double hc_lo,
                         int reg_hi, double p_hi, double sw_hi, double hc_hi, double r[3],
                         double diag[9], double* off, double base_lo, double base_hi) {
  // lower-index cell = "i" (slots 0-2), higher = "j" (slots 3-5); DIR_SIGN +1: this cell is i
  double fv[3];
  face_flux3<double>(f, trans, depth_lo, depth_hi, reg_lo, p_lo, sw_lo, hc_lo, reg_hi, p_hi, sw_hi, hc_hi, fv,
                     base_lo, base_hi);
  Dual<6> fd[3];
  face_flux3<Dual<6>>(f, trans, depth_lo, depth_hi, reg_lo, dvar<6>(p_lo, 0), dvar<6>(sw_lo, 1), dvar<6>(hc_lo, 2),
                      reg_hi, dvar<6>(p_hi, 3), dvar<6>(sw_hi, 4), dvar<6>(hc_hi, 5), fd, base_lo, base_hi);
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    if (DIR_SIGN > 0) {
      r[e] += fv[e] * dt;
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        diag[3 * e + v] += filt3(fd[e].d[v] * dt);
        off[3 * e + v] = filt3(fd[e].d[3 + v] * dt);
      }
    } else {
      r[e] += -fv[e] * dt;
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        diag[3 * e + v] += filt3(-fd[e].d[3 + v] * dt);
        off[3 * e + v] = filt3(-fd[e].d[v] * dt);
      }
    }
  }
}

// Residual row and Jacobian block row of cell i (accumulation, then the six faces), written into
// res[3i..] and the row's blocks of val (stencil: 7 block positions per row, -1 absent).
RF_HD void cell_row3(const Fluid& f, int nx, int ny, int nz, int i, double dt,
                     const double* __restrict__ pv, const double* __restrict__ tx,
                     const double* __restrict__ ty, const double* __restrict__ tz,
                     const double* __restrict__ depth, const int* __restrict__ reg,
                     const double* __restrict__ p, const double* __restrict__ sw,
                     const double* __restrict__ hc, const double* __restrict__ pp,
                     const double* __restrict__ psw, const double* __restrict__ phc,
                     const int* __restrict__ row_ptr, const int* __restrict__ stencil,
                     double* __restrict__ res, double* __restrict__ val,
                     const double* __restrict__ base_rs) {
  const int nxy = nx * ny;
  const int ci = i % nx, cj = (i / nx) % ny, ck = i / nxy;
  for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
#pragma unroll
    for (int e = 0; e < 9; ++e) val[size_t(k) * 9 + e] = 0.0;

  // accumulation; the previous inventory uses the same (frozen) regime, as the substep's
  // previous state and first iterate are the same classified state
  const int ri = reg[i];
  // the DRSDT0 Rs cap of a cell: the simulator's Rs at the substep start
  auto base = [&](int c) { return f.drsdt0 ? base_rs[c] : 0.0; };
  const double bi = base(i);
  double cur[3], prev[3];
  inventory3<double>(f, pv[i], ri, p[i], sw[i], hc[i], bi, cur);
  inventory3<double>(f, pv[i], ri, pp[i], psw[i], phc[i], bi, prev);
  double r[3] = {0.0 + (cur[0] - prev[0]), 0.0 + (cur[1] - prev[1]), 0.0 + (cur[2] - prev[2])};
  double diag[9];
  {
    Dual<3> cd[3];
    inventory3<Dual<3>>(f, pv[i], ri, dvar<3>(p[i], 0), dvar<3>(sw[i], 1), dvar<3>(hc[i], 2), bi, cd);
#pragma unroll
    for (int e = 0; e < 3; ++e)
#pragma unroll
      for (int v = 0; v < 3; ++v) diag[3 * e + v] = filt3(cd[e].d[v]);
  }
  const int* st = stencil + size_t(i) * 7;
  double off[9];
  const double dk = depth[ck];
  const double pi = p[i], swi = sw[i], hci = hc[i];
  if (ck > 0) {
    const int nb = i - nxy;
    const double t = tz[nb];
    if (t > 0.0) {
      face_contrib3<-1>(f, t, dt, depth[ck - 1], dk, reg[nb], p[nb], sw[nb], hc[nb], ri, pi, swi, hci, r, diag, off,
                        base(nb), bi);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kZm]) * 9 + e] = off[e];
    }
  }
  if (cj > 0) {
    const int nb = i - nx;
    const double t = ty[nb];
    if (t > 0.0) {
      face_contrib3<-1>(f, t, dt, dk, dk, reg[nb], p[nb], sw[nb], hc[nb], ri, pi, swi, hci, r, diag, off,
                        base(nb), bi);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kYm]) * 9 + e] = off[e];
    }
  }
  if (ci > 0) {
    const int nb = i - 1;
    const double t = tx[nb];
    if (t > 0.0) {
      face_contrib3<-1>(f, t, dt, dk, dk, reg[nb], p[nb], sw[nb], hc[nb], ri, pi, swi, hci, r, diag, off,
                        base(nb), bi);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kXm]) * 9 + e] = off[e];
    }
  }
  if (ci + 1 < nx) {
    const int nb = i + 1;
    const double t = tx[i];
    if (t > 0.0) {
      face_contrib3<1>(f, t, dt, dk, dk, ri, pi, swi, hci, reg[nb], p[nb], sw[nb], hc[nb], r, diag, off,
                       bi, base(nb));
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kXp]) * 9 + e] = off[e];
    }
  }
  if (cj + 1 < ny) {
    const int nb = i + nx;
    const double t = ty[i];
    if (t > 0.0) {
      face_contrib3<1>(f, t, dt, dk, dk, ri, pi, swi, hci, reg[nb], p[nb], sw[nb], hc[nb], r, diag, off,
                       bi, base(nb));
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kYp]) * 9 + e] = off[e];
    }
  }
  if (ck + 1 < nz) {
    const int nb = i + nxy;
    const double t = tz[i];
    if (t > 0.0) {
      face_contrib3<1>(f, t, dt, dk, depth[ck + 1], ri, pi, swi, hci, reg[nb], p[nb], sw[nb], hc[nb], r, diag, off,
                       bi, base(nb));
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kZp]) * 9 + e] = off[e];
    }
  }
#pragma unroll
  for (int e = 0; e < 3; ++e) res[3 * i + e] = r[e];
#pragma unroll
  for (int e = 0; e < 9; ++e) val[size_t(st[kDiag]) * 9 + e] = diag[e];
}

// Perforation k: its source terms in the cell's rows and diagonal block, and its connection row.
RF_HD void perf_row3(const Fluid& f, int n_wells, int k, double dt, const int* __restrict__ perf_cell,
                     const int* __restrict__ perf_inj, const int* __restrict__ perf_well,
                     const int* __restrict__ perf_has_wi, const double* __restrict__ perf_wi,
                     const double* __restrict__ perf_head, const int* __restrict__ reg,
                     const double* __restrict__ p, const double* __restrict__ sw, const double* __restrict__ hc,
                     const double* __restrict__ bhp, const double* __restrict__ q, const int* __restrict__ diag_pos,
                     double* __restrict__ res, double* __restrict__ val, double* __restrict__ res_tail,
                     double* __restrict__ jrw, double* __restrict__ jwr_perf, double* __restrict__ jww_perf_bhp,
                     const double* __restrict__ base_rs) {
  const int c = perf_cell[k], w = perf_well[k], rg = reg[c];
  const double bc = f.drsdt0 ? base_rs[c] : 0.0;
  const bool inj = perf_inj[k] != 0;
  const double pc = p[c], swc = sw[c], hcc = hc[c], b = bhp[w], qk = q[k];
  double coef[3];
  component_coefficients3<double>(f, inj, rg, pc, swc, hcc, coef, bc);
#pragma unroll
  for (int e = 0; e < 3; ++e) res[3 * c + e] += coef[e] * qk * dt;
  double* dblk = val + size_t(diag_pos[c]) * 9;
  {
    Dual<4> P = dvar<4>(pc, 0), SW = dvar<4>(swc, 1), HC = dvar<4>(hcc, 2), Q = dvar<4>(qk, 3);
    Dual<4> ca[3];
    component_coefficients3<Dual<4>>(f, inj, rg, P, SW, HC, ca, bc);
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      Dual<4> row = ca[e] * Q;
#pragma unroll
      for (int v = 0; v < 3; ++v) dblk[3 * e + v] += filt3(row.d[v] * dt);
      jrw[3 * k + e] = filt3(row.d[3] * dt);
    }
  }
  if (perf_has_wi[k]) {
    const double conn = connection_rate3<double>(f, perf_wi[k], perf_head[k], inj, rg, pc, swc, hcc, b, bc);
    res_tail[n_wells + k] = 0.0 + (qk - conn);
    Dual<4> ca = connection_rate3<Dual<4>>(f, perf_wi[k], perf_head[k], inj, rg, dvar<4>(pc, 0), dvar<4>(swc, 1),
                                           dvar<4>(hcc, 2), dvar<4>(b, 3), bc);
#pragma unroll
    for (int v = 0; v < 3; ++v) jwr_perf[3 * k + v] = filt3(-ca.d[v]);
    jww_perf_bhp[k] = filt3(-ca.d[3]);
  } else {
    res_tail[n_wells + k] = 0.0;
#pragma unroll
    for (int v = 0; v < 3; ++v) jwr_perf[3 * k + v] = 0.0;
    jww_perf_bhp[k] = 0.0;
  }
}

// Control row of physical well w.
RF_HD void well_row3(const Fluid& f, int w, const WellControlH& c, const int* __restrict__ well_ptr,
                     const int* __restrict__ well_perfs, const int* __restrict__ perf_cell,
                     const int* __restrict__ reg, const double* __restrict__ p, const double* __restrict__ sw,
                     const double* __restrict__ hc, const double* __restrict__ bhp, const double* __restrict__ q,
                     double* __restrict__ res_tail, double* __restrict__ jwr_ctrl, double* __restrict__ jww_ctrl_q,
                     double* __restrict__ jww_ctrl_bhp, const double* __restrict__ base_rs) {
  const bool inj = c.injector != 0;
  auto base = [&](int cell) { return f.drsdt0 ? base_rs[cell] : 0.0; };
  const double b = bhp[w];
  for (int a = well_ptr[w]; a < well_ptr[w + 1]; ++a) {
    const int k = well_perfs[a];
#pragma unroll
    for (int v = 0; v < 3; ++v) jwr_ctrl[3 * k + v] = 0.0;
    jww_ctrl_q[k] = 0.0;
  }
  if (!c.enabled || !c.rate_controlled) {
    res_tail[w] = 0.0 + (b - c.bhp_target);
    jww_ctrl_bhp[w] = 1.0;
    return;
  }
  if (!c.has_target) {
    res_tail[w] = 0.0;
    jww_ctrl_bhp[w] = 0.0;
    return;
  }
  double actual = 0.0;
  for (int a = well_ptr[w]; a < well_ptr[w + 1]; ++a) {
    const int k = well_perfs[a], cell = perf_cell[k];
    actual = actual + (c.uses_surface_target
                           ? surface_rate3<double>(f, inj, reg[cell], p[cell], sw[cell], hc[cell], q[k], base(cell))
                           : reservoir_rate<double>(inj, q[k]));
  }
  const double bhp_slack = inj ? c.bhp_limit - b : b - c.bhp_limit;
  const double rate_slack = c.target_rate - actual;
  const double bs = fmax(fabs(c.bhp_limit), 1.0), rsc = fmax(fabs(c.target_rate), 1.0);
  res_tail[w] = 0.0 + fischer_burmeister(bhp_slack / bs, rate_slack / rsc);
  double da, db;
  fb_gradient(bhp_slack / bs, rate_slack / rsc, da, db);
  const double dslack = inj ? -1.0 : 1.0;
  jww_ctrl_bhp[w] = filt3(da * dslack / bs);
  const double factor = -db / rsc;
  for (int a = well_ptr[w]; a < well_ptr[w + 1]; ++a) {
    const int k = well_perfs[a], cell = perf_cell[k];
    Dual<4> P = dvar<4>(p[cell], 0), SW = dvar<4>(sw[cell], 1), HC = dvar<4>(hc[cell], 2), Q = dvar<4>(q[k], 3);
    Dual<4> rate = c.uses_surface_target ? surface_rate3<Dual<4>>(f, inj, reg[cell], P, SW, HC, Q, base(cell))
                                         : reservoir_rate<Dual<4>>(inj, Q);
#pragma unroll
    for (int v = 0; v < 3; ++v) jwr_ctrl[3 * k + v] = filt3(factor * rate.d[v]);
    jww_ctrl_q[k] = filt3(factor * rate.d[3]);
  }
}


}  // namespace rf
