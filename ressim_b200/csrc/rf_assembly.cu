// rf_assembly.cu — residual and Jacobian assembly of the fully implicit step on the device.
//
// k_cells     one thread per cell: accumulation (dual numbers over the cell's own [p, sw, hc])
//             and the six face fluxes (dual numbers over both neighbours), written straight into
//             the cell's block row.  Residual values use plain doubles, Jacobian blocks use dual
//             numbers, as the reference does (fim/assembly_ad.rs:782-983).  Contributions are
//             added in the reference's triplet order — accumulation, then faces z-, y-, x-, x+,
//             y+, z+ — so sums are deterministic; entries with |v| <= 1e-14 are dropped first.
// k_perfs     one thread per perforation: well source terms and the perforation rows
//             (fim/assembly_ad.rs:239-577).
// k_wells     one thread per physical well: the control row (BHP target or Fischer-Burmeister
//             rate/BHP complementarity, fim/wells_ad.rs:345-378).
// k_norms_*   deterministic reductions for scaled residual norms and OPM CNV/MB
//             (fim/newton/convergence.rs:3-26, 478-609).
#include "rf_ops.hpp"

namespace rf {

__device__ __forceinline__ double filt(double v) { return fabs(v) > 1e-14 ? v : 0.0; }

template <int DIR_SIGN>
__device__ __forceinline__ void face_contrib(const Fluid& f, double trans, double dt, double depth_lo,
                                             double depth_hi, double p_lo, double sw_lo, double p_hi,
                                             double sw_hi, double r[3], double diag[9], double* off) {
  // The face is always evaluated with the lower-index cell as "i" (slots 0-2) and the higher as
  // "j" (slots 3-5).  DIR_SIGN = -1: this cell is j (face from a lower neighbour); +1: this cell is i.
  double fv[3];
  face_flux<double>(f, trans, depth_lo, depth_hi, p_lo, sw_lo, p_hi, sw_hi, fv);
  Dual<6> fd[3];
  face_flux<Dual<6>>(f, trans, depth_lo, depth_hi, dvar<6>(p_lo, 0), dvar<6>(sw_lo, 1), dvar<6>(p_hi, 3),
                     dvar<6>(sw_hi, 4), fd);
  // hc (slots 2 and 5) never enters the two-phase flux, so its derivative columns are zero.
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    if (DIR_SIGN > 0) {
      r[e] += fv[e] * dt;
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        diag[3 * e + v] += filt(fd[e].d[v] * dt);
        off[3 * e + v] = filt(fd[e].d[3 + v] * dt);
      }
    } else {
      r[e] += -fv[e] * dt;
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        diag[3 * e + v] += filt(-fd[e].d[3 + v] * dt);
        off[3 * e + v] = filt(-fd[e].d[v] * dt);
      }
    }
  }
}

__global__ void __launch_bounds__(128) k_cells(Fluid f, int nx, int ny, int nz, double dt, const double* __restrict__ pv,
                                                const double* __restrict__ tx, const double* __restrict__ ty,
                                                const double* __restrict__ tz, const double* __restrict__ depth,
                                                const double* __restrict__ p, const double* __restrict__ sw,
                                                const double* __restrict__ hc, const double* __restrict__ pp,
                                                const double* __restrict__ psw, const double* __restrict__ phc,
                                                const int* __restrict__ row_ptr, const int* __restrict__ stencil,
                                                double* __restrict__ res, double* __restrict__ val) {
  const int n = nx * ny * nz;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int nxy = nx * ny;
  const int ci = i % nx, cj = (i / nx) % ny, ck = i / nxy;

  // zero every block of this row (stencil and well fill)
  for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
#pragma unroll
    for (int e = 0; e < 9; ++e) val[size_t(k) * 9 + e] = 0.0;

  // accumulation: residual with plain doubles, Jacobian block with Dual<3>
  double cur[3], prev[3];
  inventory<double>(f, pv[i], p[i], sw[i], hc[i], cur);
  inventory<double>(f, pv[i], pp[i], psw[i], phc[i], prev);
  double r[3] = {0.0 + (cur[0] - prev[0]), 0.0 + (cur[1] - prev[1]), 0.0 + (cur[2] - prev[2])};
  double diag[9];
  {
    Dual<3> cd[3];
    inventory<Dual<3>>(f, pv[i], dvar<3>(p[i], 0), dvar<3>(sw[i], 1), dvar<3>(hc[i], 2), cd);
#pragma unroll
    for (int e = 0; e < 3; ++e)
#pragma unroll
      for (int v = 0; v < 3; ++v) diag[3 * e + v] = filt(cd[e].d[v]);
  }
  const int* st = stencil + size_t(i) * 7;
  double off[9];
  const double dk = depth[ck];
  // z- face (neighbour below in index is the lower-index cell)
  if (ck > 0) {
    const int nb = i - nxy;
    const double t = tz[nb];
    if (t > 0.0) {
      face_contrib<-1>(f, t, dt, depth[ck - 1], dk, p[nb], sw[nb], p[i], sw[i], r, diag, off);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kZm]) * 9 + e] = off[e];
    }
  }
  if (cj > 0) {
    const int nb = i - nx;
    const double t = ty[nb];
    if (t > 0.0) {
      face_contrib<-1>(f, t, dt, dk, dk, p[nb], sw[nb], p[i], sw[i], r, diag, off);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kYm]) * 9 + e] = off[e];
    }
  }
  if (ci > 0) {
    const int nb = i - 1;
    const double t = tx[nb];
    if (t > 0.0) {
      face_contrib<-1>(f, t, dt, dk, dk, p[nb], sw[nb], p[i], sw[i], r, diag, off);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kXm]) * 9 + e] = off[e];
    }
  }
  if (ci + 1 < nx) {
    const int nb = i + 1;
    const double t = tx[i];
    if (t > 0.0) {
      face_contrib<1>(f, t, dt, dk, dk, p[i], sw[i], p[nb], sw[nb], r, diag, off);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kXp]) * 9 + e] = off[e];
    }
  }
  if (cj + 1 < ny) {
    const int nb = i + nx;
    const double t = ty[i];
    if (t > 0.0) {
      face_contrib<1>(f, t, dt, dk, dk, p[i], sw[i], p[nb], sw[nb], r, diag, off);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kYp]) * 9 + e] = off[e];
    }
  }
  if (ck + 1 < nz) {
    const int nb = i + nxy;
    const double t = tz[i];
    if (t > 0.0) {
      face_contrib<1>(f, t, dt, dk, depth[ck + 1], p[i], sw[i], p[nb], sw[nb], r, diag, off);
#pragma unroll
      for (int e = 0; e < 9; ++e) val[size_t(st[kZp]) * 9 + e] = off[e];
    }
  }
#pragma unroll
  for (int e = 0; e < 3; ++e) res[3 * i + e] = r[e];
#pragma unroll
  for (int e = 0; e < 9; ++e) val[size_t(st[kDiag]) * 9 + e] = diag[e];
}

// Perforation terms: source into the connected cell's rows and the perforation row.
__global__ void k_perfs(Fluid f, int n_wells, int n_perfs, double dt, const int* __restrict__ perf_cell,
                        const int* __restrict__ perf_well, const int* __restrict__ perf_inj,
                        const int* __restrict__ perf_has_wi, const double* __restrict__ perf_wi,
                        const double* __restrict__ perf_head, const double* __restrict__ p,
                        const double* __restrict__ sw, const double* __restrict__ hc, const double* __restrict__ bhp,
                        const double* __restrict__ q, const int* __restrict__ diag_pos, double* __restrict__ res,
                        double* __restrict__ val, double* __restrict__ res_tail, double* __restrict__ jrw,
                        double* __restrict__ jwr_perf, double* __restrict__ jww_perf_bhp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_perfs) return;
  const int c = perf_cell[k], w = perf_well[k];
  const bool inj = perf_inj[k] != 0;
  const double pc = p[c], swc = sw[c], hcc = hc[c], b = bhp[w], qk = q[k];
  double coef[3];
  component_coefficients<double>(f, inj, pc, swc, hcc, coef);
#pragma unroll
  for (int e = 0; e < 3; ++e) res[3 * c + e] += coef[e] * qk * dt;
  double* dblk = val + size_t(diag_pos[c]) * 9;
  {
    Dual<4> P = dvar<4>(pc, 0), SW = dvar<4>(swc, 1), HC = dvar<4>(hcc, 2), Q = dvar<4>(qk, 3);
    Dual<4> ca[3];
    component_coefficients<Dual<4>>(f, inj, P, SW, HC, ca);
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      Dual<4> row = ca[e] * Q;
#pragma unroll
      for (int v = 0; v < 3; ++v) dblk[3 * e + v] += filt(row.d[v] * dt);
      jrw[3 * k + e] = filt(row.d[3] * dt);
    }
  }
  if (perf_has_wi[k]) {
    const double conn = connection_rate<double>(f, perf_wi[k], perf_head[k], inj, pc, swc, b);
    res_tail[n_wells + k] = 0.0 + (qk - conn);
    Dual<4> ca = connection_rate<Dual<4>>(f, perf_wi[k], perf_head[k], inj, dvar<4>(pc, 0), dvar<4>(swc, 1),
                                          dvar<4>(b, 3));
#pragma unroll
    for (int v = 0; v < 3; ++v) jwr_perf[3 * k + v] = filt(-ca.d[v]);
    jww_perf_bhp[k] = filt(-ca.d[3]);
  } else {
    res_tail[n_wells + k] = 0.0;
#pragma unroll
    for (int v = 0; v < 3; ++v) jwr_perf[3 * k + v] = 0.0;
    jww_perf_bhp[k] = 0.0;
  }
}

// Control row of each physical well.
__global__ void k_wells(Fluid f, int n_wells, const WellControlH* __restrict__ ctrl, const int* __restrict__ well_ptr,
                        const int* __restrict__ well_perfs, const int* __restrict__ perf_cell,
                        const double* __restrict__ p, const double* __restrict__ sw, const double* __restrict__ hc,
                        const double* __restrict__ bhp, const double* __restrict__ q, double* __restrict__ res_tail,
                        double* __restrict__ jwr_ctrl, double* __restrict__ jww_ctrl_q,
                        double* __restrict__ jww_ctrl_bhp) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_wells) return;
  const WellControlH c = ctrl[w];
  const bool inj = c.injector != 0;
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
    actual = actual + (c.uses_surface_target ? surface_rate<double>(f, inj, p[cell], sw[cell], hc[cell], q[k])
                                             : reservoir_rate<double>(inj, q[k]));
  }
  const double bhp_slack = inj ? c.bhp_limit - b : b - c.bhp_limit;
  const double rate_slack = c.target_rate - actual;
  const double bs = fmax(fabs(c.bhp_limit), 1.0), rsc = fmax(fabs(c.target_rate), 1.0);
  res_tail[w] = 0.0 + fischer_burmeister(bhp_slack / bs, rate_slack / rsc);
  double da, db;
  fb_gradient(bhp_slack / bs, rate_slack / rsc, da, db);
  const double dslack = inj ? -1.0 : 1.0;
  jww_ctrl_bhp[w] = filt(da * dslack / bs);
  const double factor = -db / rsc;
  for (int a = well_ptr[w]; a < well_ptr[w + 1]; ++a) {
    const int k = well_perfs[a], cell = perf_cell[k];
    Dual<4> P = dvar<4>(p[cell], 0), SW = dvar<4>(sw[cell], 1), HC = dvar<4>(hc[cell], 2), Q = dvar<4>(q[k], 3);
    Dual<4> rate = c.uses_surface_target ? surface_rate<Dual<4>>(f, inj, P, SW, HC, Q) : reservoir_rate<Dual<4>>(inj, Q);
#pragma unroll
    for (int v = 0; v < 3; ++v) jwr_ctrl[3 * k + v] = filt(factor * rate.d[v]);
    jww_ctrl_q[k] = filt(factor * rate.d[3]);
  }
}

// ---- Newton norms: per-block partials of 13 quantities, then a fixed-order final pass ----
constexpr int kNormQ = 13;
__global__ void __launch_bounds__(kBlock) k_norms_cells(Fluid f, int n, double dt, const double* __restrict__ pv_ref,
                                                         const double* __restrict__ p, const double* __restrict__ res,
                                                         double* __restrict__ partials) {
  __shared__ double sh[32];
  double q[kNormQ];
#pragma unroll
  for (int k = 0; k < kNormQ; ++k) q[k] = 0.0;
  const double dtc = fmax(dt, 1e-12);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double pvr = pv_ref[i];
    const double pod = fmax(fabs(pvr / dtc), 1.0);
    const double pr = p[i];
    const double bw = water_fvf(f, pr);
    const double bo = fmax(oil_fvf_plain(f, pr), 1e-9);
    const double bg = fmax(1.0, 1e-9);
    const double rw = res[3 * i], ro = res[3 * i + 1], rg = res[3 * i + 2];
    q[0] = fmax(q[0], fabs(rw) / (pod / bw));
    q[1] = fmax(q[1], fabs(ro) / (pod / bo));
    q[2] = fmax(q[2], fabs(rg) / (pod / bg));
    q[3] += bw;
    q[4] += bo;
    q[5] += bg;
    const double pvc = fmax(pvr, 1e-9);
    q[6] = fmax(q[6], fabs(rw) / pvc);
    q[7] = fmax(q[7], fabs(ro) / pvc);
    q[8] = fmax(q[8], fabs(rg) / pvc);
    q[9] += rw;
    q[10] += ro;
    q[11] += rg;
    q[12] += pvc;
  }
#pragma unroll
  for (int k = 0; k < kNormQ; ++k) {
    const bool is_max = (k <= 2) || (k >= 6 && k <= 8);
    const double r = is_max ? block_max<kBlock>(q[k], sh) : block_sum<kBlock>(q[k], sh);
    if (threadIdx.x == 0) partials[size_t(blockIdx.x) * kNormQ + k] = r;
  }
}

__global__ void k_norms_final(int nblocks, const double* __restrict__ partials, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kNormQ) return;
  const bool is_max = (k <= 2) || (k >= 6 && k <= 8);
  double a = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    const double v = partials[size_t(b) * kNormQ + k];
    a = is_max ? fmax(a, v) : a + v;
  }
  out[k] = a;
}

// violating pore volume: cells whose max_c |r_c| * B_avg_c / pv exceeds the strict CNV tolerance
__global__ void __launch_bounds__(kBlock) k_cnv_violation(int n, const double* __restrict__ pv_ref,
                                                           const double* __restrict__ res,
                                                           const double* __restrict__ stats,
                                                           double* __restrict__ partials) {
  __shared__ double sh[32];
  const double inv_n = 1.0 / double(n > 0 ? n : 1);
  const double bw = stats[3] * inv_n, bo = stats[4] * inv_n, bg = stats[5] * inv_n;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double pvc = fmax(pv_ref[i], 1e-9);
    double cm = fabs(res[3 * i]) * bw / pvc;
    cm = fmax(cm, fabs(res[3 * i + 1]) * bo / pvc);
    cm = fmax(cm, fabs(res[3 * i + 2]) * bg / pvc);
    if (cm > 1e-2) acc += pvc;
  }
  const double r = block_sum<kBlock>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

__global__ void k_sum_final(int nblocks, const double* __restrict__ partials, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double a = 0.0;
  for (int b = 0; b < nblocks; ++b) a += partials[b];
  *out = a;
}

// ---- host launchers ----
void launch_assembly(Ctx& c, double dt) {
  if (c.fluid.three_phase) {
    launch_assembly3(c, dt);
    return;
  }
  const int n = c.n;
  k_cells<<<blocks_for(n, 128), 128, 0, c.stream>>>(c.fluid, c.nx, c.ny, c.nz, dt, c.d_pv.p, c.d_tx.p, c.d_ty.p,
                                                     c.d_tz.p, c.d_depth.p, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_pp.p,
                                                     c.d_psw.p, c.d_phc.p, c.d_row_ptr.p, c.d_stencil.p, c.d_res.p,
                                                     c.d_val.p);
  c.launches++;
  if (c.topo.n_perfs > 0) {
    k_perfs<<<blocks_for(c.topo.n_perfs, 64), 64, 0, c.stream>>>(
        c.fluid, c.topo.n_wells, c.topo.n_perfs, dt, c.d_perf_cell.p, c.d_perf_well.p, c.d_perf_inj.p,
        c.d_perf_has_wi.p, c.d_perf_wi.p, c.d_perf_head.p, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_bhp.p, c.d_q.p,
        c.d_diag.p, c.d_res.p, c.d_val.p, c.d_res_tail.p, c.d_jrw.p, c.d_jwr_perf.p, c.d_jww_perf_bhp.p);
    c.launches++;
  }
  if (c.topo.n_wells > 0) {
    k_wells<<<blocks_for(c.topo.n_wells, 32), 32, 0, c.stream>>>(
        c.fluid, c.topo.n_wells, c.d_ctrl.p, c.d_well_ptr.p, c.d_well_perfs.p, c.d_perf_cell.p, c.d_p.p, c.d_sw.p,
        c.d_hc.p, c.d_bhp.p, c.d_q.p, c.d_res_tail.p, c.d_jwr_ctrl.p, c.d_jww_ctrl_q.p, c.d_jww_ctrl_bhp.p);
    c.launches++;
  }
}

// Residual-only assembly shares k_cells (the Jacobian work is a small share of its cost); the
// well rows are refreshed the same way.
void launch_norms(Ctx& c, double dt, double* h_out /* kNormQ + 1 */) {
  const int n = c.n;
  int nb = blocks_for(n);
  if (nb > 4 * c.num_sms) nb = 4 * c.num_sms;
  if (c.fluid.three_phase) {
    launch_norm_partials3(c, dt, nb);
    c.launches--;  // counted below with the other three launches
  } else {
    k_norms_cells<<<nb, kBlock, 0, c.stream>>>(c.fluid, n, dt, c.d_pv.p, c.d_p.p, c.d_res.p, c.d_partials.p);
  }
  k_norms_final<<<1, 32, 0, c.stream>>>(nb, c.d_partials.p, c.d_scal.p);
  k_cnv_violation<<<nb, kBlock, 0, c.stream>>>(n, c.d_pv.p, c.d_res.p, c.d_scal.p, c.d_partials.p);
  k_sum_final<<<1, 32, 0, c.stream>>>(nb, c.d_partials.p, c.d_scal.p + kNormQ);
  c.launches += 4;
  d2h(c, h_out, c.d_scal.p, sizeof(double) * (kNormQ + 1));
  d2h_wait(c);
}

}  // namespace rf
