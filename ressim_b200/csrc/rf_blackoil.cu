// rf_blackoil.cu — device kernels of the three-phase black-oil mode.  They mirror the two-phase
// kernels of rf_assembly.cu / rf_state.cu with the black-oil physics of rf_blackoil.cuh:
//
// k_cells3      one thread per cell: accumulation (Dual<3>) and the six face fluxes (Dual<6> over
//               both neighbours' [p, sw, hc]), each in its cell's regime, written straight into
//               the cell's block row in the reference's triplet order (fim/assembly_ad.rs:782-983)
// k_perfs3      perforation source terms and rows (fim/assembly_ad.rs:239-577), gas injection
// k_wells3      control rows (fim/wells_ad.rs:345-378)
// k_norms3      scaled residual maxima and CNV/MB partials with Bo at the simulator's Rs and Bg
//               from the table (fim/scaling.rs:139-223, fim/newton/convergence.rs:3-26, 478-609)
// k_update3     OPM per-cell chop with the regime's implied dSg / dSo and the undersaturated Rs
//               floor (fim/newton/convergence.rs:648-708), then the raw update (fim/state.rs:597-715)
// k_from_sim3   regime classification and the hc primary at a substep start
//               (fim/state.rs:109-177, fim/flash.rs:13-40)
// k_derive3     write-back of So, Sg, Rs through the cell flash (fim/state.rs:823-914)
// k_sums3       relative change (fim/timestep.rs:436-467) and the component inventories
//               (fim/timestep.rs:1851-1888), reporting sums (reporting.rs:304-322)
#include "rf_blackoil_rows.cuh"
#include "rf_ops.hpp"
#include "rf_state.hpp"

namespace rf {

__global__ void __launch_bounds__(128) k_cells3(const __grid_constant__ Fluid f, int nx, int ny, int nz, double dt,
                                                 const double* __restrict__ pv, const double* __restrict__ tx,
                                                 const double* __restrict__ ty, const double* __restrict__ tz,
                                                 const double* __restrict__ depth, const int* __restrict__ reg,
                                                 const double* __restrict__ p, const double* __restrict__ sw,
                                                 const double* __restrict__ hc, const double* __restrict__ pp,
                                                 const double* __restrict__ psw, const double* __restrict__ phc,
                                                 const int* __restrict__ row_ptr, const int* __restrict__ stencil,
                                                 double* __restrict__ res, double* __restrict__ val,
                                                 const double* __restrict__ base_rs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nx * ny * nz) return;
  cell_row3(f, nx, ny, nz, i, dt, pv, tx, ty, tz, depth, reg, p, sw, hc, pp, psw, phc, row_ptr, stencil, res, val,
            base_rs);
}

__global__ void k_perfs3(const __grid_constant__ Fluid f, int n_wells, int n_perfs, double dt, const int* __restrict__ perf_cell,
                         const int* __restrict__ perf_inj, const int* __restrict__ perf_well,
                         const int* __restrict__ perf_has_wi, const double* __restrict__ perf_wi,
                         const double* __restrict__ perf_head, const int* __restrict__ reg,
                         const double* __restrict__ p, const double* __restrict__ sw, const double* __restrict__ hc,
                         const double* __restrict__ bhp, const double* __restrict__ q, const int* __restrict__ diag_pos,
                         double* __restrict__ res, double* __restrict__ val, double* __restrict__ res_tail,
                         double* __restrict__ jrw, double* __restrict__ jwr_perf, double* __restrict__ jww_perf_bhp,
                         const double* __restrict__ base_rs) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_perfs) return;
  perf_row3(f, n_wells, k, dt, perf_cell, perf_inj, perf_well, perf_has_wi, perf_wi, perf_head, reg, p, sw, hc, bhp,
            q, diag_pos, res, val, res_tail, jrw, jwr_perf, jww_perf_bhp, base_rs);
}

__global__ void k_wells3(const __grid_constant__ Fluid f, int n_wells, const WellControlH* __restrict__ ctrl, const int* __restrict__ well_ptr,
                         const int* __restrict__ well_perfs, const int* __restrict__ perf_cell,
                         const int* __restrict__ reg, const double* __restrict__ p, const double* __restrict__ sw,
                         const double* __restrict__ hc, const double* __restrict__ bhp, const double* __restrict__ q,
                         double* __restrict__ res_tail, double* __restrict__ jwr_ctrl, double* __restrict__ jww_ctrl_q,
                         double* __restrict__ jww_ctrl_bhp, const double* __restrict__ base_rs) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_wells) return;
  well_row3(f, w, ctrl[w], well_ptr, well_perfs, perf_cell, reg, p, sw, hc, bhp, q, res_tail, jwr_ctrl, jww_ctrl_q,
            jww_ctrl_bhp, base_rs);
}

// Scaled residual maxima, FVF sums, CNV maxima, residual sums and the pore-volume sum, as
// k_norms_cells; Bo is read at the simulator's Rs of the cell (get_b_o_cell) and Bg from the table.
constexpr int kNormQ3 = 13;
__global__ void __launch_bounds__(kBlock) k_norms3(const __grid_constant__ Fluid f, int n, double dt, const double* __restrict__ pv_ref,
                                                    const double* __restrict__ p, const double* __restrict__ rs_sim,
                                                    const double* __restrict__ res, double* __restrict__ partials) {
  __shared__ double sh[32];
  double q[kNormQ3];
#pragma unroll
  for (int k = 0; k < kNormQ3; ++k) q[k] = 0.0;
  const double dtc = fmax(dt, 1e-12);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double pvr = pv_ref[i];
    const double pod = fmax(fabs(pvr / dtc), 1.0);
    const double pr = p[i];
    const double bw = water_fvf(f, pr);
    const double bo = fmax(bo_for_rs(f, pr, rs_sim[i]), 1e-9);
    const double bg = fmax(get_b_g(f, pr), 1e-9);
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
  for (int k = 0; k < kNormQ3; ++k) {
    const bool is_max = (k <= 2) || (k >= 6 && k <= 8);
    const double r = is_max ? block_max<kBlock>(q[k], sh) : block_sum<kBlock>(q[k], sh);
    if (threadIdx.x == 0) partials[size_t(blockIdx.x) * kNormQ3 + k] = r;
  }
}

__global__ void __launch_bounds__(kBlock) k_update3(int n, double relax, const int* __restrict__ reg,
                                                     const double* __restrict__ dx, const double* __restrict__ p,
                                                     const double* __restrict__ sw, const double* __restrict__ hc,
                                                     double* __restrict__ cp, double* __restrict__ csw,
                                                     double* __restrict__ chc, double* __restrict__ partials) {
  __shared__ double sh[32];
  double pmax = -INFINITY, nonfinite = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double dp = dx[3 * i] * relax, dsw = dx[3 * i + 1] * relax, dhc = dx[3 * i + 2] * relax;
    const double pi = p[i], hci = hc[i];
    const bool sat = reg[i] == 0;
    const double dsg = sat ? dhc : 0.0, dso = sat ? -(dsw + dhc) : -dsw;
    const double mx = fmax(fmax(fabs(dsw), fabs(dso)), fabs(dsg));
    const double alpha = mx > 0.2 ? 0.2 / mx : 1.0;
    dsw = dsw * alpha;
    if (sat)
      dhc = dhc * alpha;
    else if (hci + dhc < 0.0)
      dhc = -hci;
    const double cap = 0.3 * fabs(pi);
    if (fabs(dp) > cap) dp = copysign(1.0, dp) * cap;
    double np = pi + 1.0 * dp;
    const double nsw = sw[i] + 1.0 * dsw;
    const double nhc = hci + 1.0 * dhc;
    np = fmax(np, 1e-6);
    cp[i] = np;
    csw[i] = nsw;
    chc[i] = nhc;
    pmax = fmax(pmax, np);
    if (!isfinite(np) || !isfinite(nsw) || !isfinite(nhc)) nonfinite = 1.0;
  }
  const double a = block_max<kBlock>(pmax, sh);
  const double b = block_max<kBlock>(nonfinite, sh);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

__global__ void __launch_bounds__(kBlock) k_from_sim3(const __grid_constant__ Fluid f, int n, const double* __restrict__ p,
                                                       const double* __restrict__ sg, const double* __restrict__ rs,
                                                       int* __restrict__ reg, double* __restrict__ hc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = classify_regime(f, p[i], sg[i], rs[i], rs[i]);
    reg[i] = r;
    hc[i] = r == 0 ? sg[i] : rs[i];
  }
}

__global__ void __launch_bounds__(kBlock) k_derive3(const __grid_constant__ Fluid f, int n, const double* __restrict__ p,
                                                     const double* __restrict__ sw, const double* __restrict__ hc,
                                                     const int* __restrict__ reg, double* __restrict__ so,
                                                     double* __restrict__ sg, double* __restrict__ rs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Derived3 d = derive_cell3(f, p[i], sw[i], hc[i], reg[i], rs[i]);  // base: Rs before the write
    so[i] = d.so;
    sg[i] = d.sg;
    rs[i] = d.rs;
  }
}

// 9 sums: rel-change delta and denom between (a) and (b) cell states sharing the regimes; then,
// over the simulator arrays (s*), water, oil and gas inventories, sum p*pv, sum pv, sum sw, sum sg
__global__ void __launch_bounds__(kBlock) k_sums3(const __grid_constant__ Fluid f, int n, const double* __restrict__ pv,
                                                   const int* __restrict__ reg, const double* __restrict__ ap,
                                                   const double* __restrict__ asw, const double* __restrict__ ahc,
                                                   const double* __restrict__ bp, const double* __restrict__ bsw,
                                                   const double* __restrict__ bhc, const double* __restrict__ sp,
                                                   const double* __restrict__ ssw, const double* __restrict__ sso,
                                                   const double* __restrict__ ssg, const double* __restrict__ srs,
                                                   double* __restrict__ partials) {
  __shared__ double sh[32];
  double q[kStateQ3] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double dp = bp[i] - ap[i];
    q[0] += dp * dp;
    q[1] += bp[i] * bp[i];
    const bool sat = reg[i] == 0;
    const double nsg = sat ? fmax(bhc[i], 0.0) : 0.0, osg = sat ? fmax(ahc[i], 0.0) : 0.0;
    const double nso = 1.0 - bsw[i] - nsg, oso = 1.0 - asw[i] - osg;
    const double ns[3] = {bsw[i], nsg, nso}, os[3] = {asw[i], osg, oso};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double ds = ns[k] - os[k];
      q[0] += ds * ds;
      q[1] += ns[k] * ns[k];
    }
    const double pvi = pv[i], pr = sp[i];
    q[2] += ssw[i] * pvi * inv_bw(f, pr);
    const double pvf = fmax(pvi, 1e-9);
    const double bo = fmax(bo_for_rs(f, pr, srs[i]), 1e-9);
    q[3] += sso[i] * pvf / bo;
    const double free_gas = ssg[i] * pvf / fmax(get_b_g(f, pr), 1e-9);
    const double dissolved = sso[i] * pvf * srs[i] / bo;
    q[4] += free_gas + dissolved;
    if (pvi > 0.0 && isfinite(pvi)) {
      q[5] += pr * pvi;
      q[6] += pvi;
    }
    q[7] += ssw[i];
    q[8] += ssg[i];
  }
#pragma unroll
  for (int k = 0; k < kStateQ3; ++k) {
    const double r = block_sum<kBlock>(q[k], sh);
    if (threadIdx.x == 0) partials[size_t(blockIdx.x) * kStateQ3 + k] = r;
  }
}

__global__ void k_fixed_sum_final(int nb, int nq, const double* __restrict__ partials, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= nq) return;
  double a = 0.0;
  for (int b = 0; b < nb; ++b) a += partials[size_t(b) * nq + k];
  out[k] = a;
}

// four values per perforation: (a, b, c) of the perforated cell and its regime
__global__ void k_gather_perf3(int n_perfs, const int* __restrict__ cells, const double* __restrict__ a,
                               const double* __restrict__ b, const double* __restrict__ c,
                               const int* __restrict__ reg, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_perfs) return;
  const int i = cells[k];
  out[4 * k] = a[i];
  out[4 * k + 1] = b[i];
  out[4 * k + 2] = c[i];
  out[4 * k + 3] = reg ? double(reg[i]) : 0.0;
}

// ---- host launchers ----
static int red_blocks3(const Ctx& c) {
  int nb = blocks_for(c.n);
  if (nb > 4 * c.num_sms) nb = 4 * c.num_sms;
  return nb;
}

void launch_assembly3(Ctx& c, double dt) {
  k_cells3<<<blocks_for(c.n, 128), 128, 0, c.stream>>>(c.fluid, c.nx, c.ny, c.nz, dt, c.d_pv.p, c.d_tx.p, c.d_ty.p,
                                                        c.d_tz.p, c.d_depth.p, c.d_reg.p, c.d_p.p, c.d_sw.p, c.d_hc.p,
                                                        c.d_pp.p, c.d_psw.p, c.d_phc.p, c.d_row_ptr.p, c.d_stencil.p,
                                                        c.d_res.p, c.d_val.p, c.d_rs.p);
  c.launches++;
  if (c.topo.n_perfs > 0) {
    k_perfs3<<<blocks_for(c.topo.n_perfs, 64), 64, 0, c.stream>>>(
        c.fluid, c.topo.n_wells, c.topo.n_perfs, dt, c.d_perf_cell.p, c.d_perf_inj.p, c.d_perf_well.p,
        c.d_perf_has_wi.p, c.d_perf_wi.p, c.d_perf_head.p, c.d_reg.p, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_bhp.p, c.d_q.p,
        c.d_diag.p, c.d_res.p, c.d_val.p, c.d_res_tail.p, c.d_jrw.p, c.d_jwr_perf.p, c.d_jww_perf_bhp.p, c.d_rs.p);
    c.launches++;
  }
  if (c.topo.n_wells > 0) {
    k_wells3<<<blocks_for(c.topo.n_wells, 32), 32, 0, c.stream>>>(
        c.fluid, c.topo.n_wells, c.d_ctrl.p, c.d_well_ptr.p, c.d_well_perfs.p, c.d_perf_cell.p, c.d_reg.p, c.d_p.p,
        c.d_sw.p, c.d_hc.p, c.d_bhp.p, c.d_q.p, c.d_res_tail.p, c.d_jwr_ctrl.p, c.d_jww_ctrl_q.p, c.d_jww_ctrl_bhp.p,
        c.d_rs.p);
    c.launches++;
  }
}

void launch_norm_partials3(Ctx& c, double dt, int nb) {
  k_norms3<<<nb, kBlock, 0, c.stream>>>(c.fluid, c.n, dt, c.d_pv.p, c.d_p.p, c.d_rs.p, c.d_res.p, c.d_partials.p);
  c.launches++;
}

void apply_cell_update3(Ctx& c, double relax, double& pmax, bool& finite) {
  const int nb = red_blocks3(c);
  k_update3<<<nb, kBlock, 0, c.stream>>>(c.n, relax, c.d_reg.p, c.d_x.p, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_cp.p,
                                         c.d_csw.p, c.d_chc.p, c.d_partials.p);
  c.launches++;
  max2_final(c, nb, pmax, finite);
}

void from_simulator3(Ctx& c) {
  k_from_sim3<<<red_blocks3(c), kBlock, 0, c.stream>>>(c.fluid, c.n, c.d_pp.p, c.d_sg.p, c.d_rs.p, c.d_reg.p,
                                                       c.d_phc.p);
  c.launches++;
}

void derive3(Ctx& c) {
  k_derive3<<<red_blocks3(c), kBlock, 0, c.stream>>>(c.fluid, c.n, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_reg.p, c.d_so.p,
                                                     c.d_sg.p, c.d_rs.p);
  c.launches++;
}

void state_sums3(Ctx& c, const double* ap, const double* asw, const double* ahc, const double* bp, const double* bsw,
                 const double* bhc, const double* sp, const double* ssw, double out[kStateQ3]) {
  const int nb = red_blocks3(c);
  k_sums3<<<nb, kBlock, 0, c.stream>>>(c.fluid, c.n, c.d_pv.p, c.d_reg.p, ap, asw, ahc, bp, bsw, bhc, sp, ssw,
                                       c.d_so.p, c.d_sg.p, c.d_rs.p, c.d_partials.p);
  k_fixed_sum_final<<<1, 32, 0, c.stream>>>(nb, kStateQ3, c.d_partials.p, c.d_scal.p + 220);
  c.launches += 2;
  d2h(c, out, c.d_scal.p + 220, sizeof(double) * kStateQ3);
  d2h_wait(c);
}

void gather_perf_cells3(Ctx& c, const double* a, const double* b, const double* cc, const int* reg,
                        std::vector<double>& out) {
  const int P = c.topo.n_perfs;
  out.assign(4 * size_t(P), 0.0);
  if (P == 0) return;
  double* d = c.d_scal.p + 1024;  // 4P <= 4096 doubles (checked at setup)
  k_gather_perf3<<<blocks_for(P, 64), 64, 0, c.stream>>>(P, c.d_perf_cell.p, a, b, cc, reg, d);
  c.launches++;
  d2h(c, out.data(), d, sizeof(double) * 4 * P);
  d2h_wait(c);
}

}  // namespace rf
