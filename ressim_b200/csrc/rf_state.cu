// rf_state.cu — per-cell update, bounds and substep-level reductions on the device.
//
//   k_apply_update   OPM per-cell chop of the relaxed Newton update (saturation scaling by
//                    0.2 / max|dS| including the implied dSo, relative pressure clamp 0.3 p) and
//                    its application with the pressure floor (fim/newton/convergence.rs:648-708,
//                    fim/state.rs:597-715)
//   k_state_sums     opm_relative_change terms, inventories, PV-weighted pressure
//                    (fim/timestep.rs:436-467, 1851-1885; reporting.rs:304-322)
#include "rf_ops.hpp"
#include "rf_state.hpp"

namespace rf {

__global__ void __launch_bounds__(kBlock) k_apply_update(int n, double relax, const double* __restrict__ dx,
                                                          const double* __restrict__ p, const double* __restrict__ sw,
                                                          const double* __restrict__ hc, double* __restrict__ cp,
                                                          double* __restrict__ csw, double* __restrict__ chc,
                                                          double* __restrict__ partials) {
  __shared__ double sh[32];
  double pmax = -INFINITY, nonfinite = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double dp = dx[3 * i] * relax, dsw = dx[3 * i + 1] * relax, dhc = dx[3 * i + 2] * relax;
    const double pi = p[i];
    // saturated regime (the two-phase third unknown is the gas saturation primary)
    const double dsg = dhc, dso = -(dsw + dhc);
    const double mx = fmax(fmax(fabs(dsw), fabs(dso)), fabs(dsg));
    const double alpha = mx > 0.2 ? 0.2 / mx : 1.0;
    dsw = dsw * alpha;
    dhc = dhc * alpha;
    const double cap = 0.3 * fabs(pi);
    if (fabs(dp) > cap) dp = copysign(1.0, dp) * cap;
    double np = pi + 1.0 * dp;
    const double nsw = sw[i] + 1.0 * dsw;
    const double nhc = hc[i] + 1.0 * dhc;
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

__global__ void k_max2_final(int nb, const double* __restrict__ partials, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double a = -INFINITY, b = 0.0;
  for (int k = 0; k < nb; ++k) {
    a = fmax(a, partials[2 * k]);
    b = fmax(b, partials[2 * k + 1]);
  }
  out[0] = a;
  out[1] = b;
}

// 7 sums: rel-change delta, rel-change denom, water inventory, oil inventory, sum p*pv, sum pv,
// sum sw.  (a = previous state, b = current state)
constexpr int kStateQ = 7;
__global__ void __launch_bounds__(kBlock) k_state_sums(Fluid f, int n, const double* __restrict__ pv,
                                                        const double* __restrict__ ap, const double* __restrict__ asw,
                                                        const double* __restrict__ ahc, const double* __restrict__ bp,
                                                        const double* __restrict__ bsw, const double* __restrict__ bhc,
                                                        double* __restrict__ partials) {
  __shared__ double sh[32];
  double q[kStateQ] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double dp = bp[i] - ap[i];
    q[0] += dp * dp;
    q[1] += bp[i] * bp[i];
    const double nsg = fmax(bhc[i], 0.0), osg = fmax(ahc[i], 0.0);
    const double nso = 1.0 - bsw[i] - nsg, oso = 1.0 - asw[i] - osg;
    const double ns[3] = {bsw[i], nsg, nso}, os[3] = {asw[i], osg, oso};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double ds = ns[k] - os[k];
      q[0] += ds * ds;
      q[1] += ns[k] * ns[k];
    }
    const double pvi = pv[i];
    q[2] += bsw[i] * pvi * inv_bw(f, bp[i]);
    const double so = fmax(1.0 - bsw[i], 0.0);
    q[3] += so * fmax(pvi, 1e-9) / fmax(oil_fvf_plain(f, bp[i]), 1e-9);
    if (pvi > 0.0 && isfinite(pvi)) {
      q[4] += bp[i] * pvi;
      q[5] += pvi;
    }
    q[6] += bsw[i];
  }
#pragma unroll
  for (int k = 0; k < kStateQ; ++k) {
    const double r = block_sum<kBlock>(q[k], sh);
    if (threadIdx.x == 0) partials[size_t(blockIdx.x) * kStateQ + k] = r;
  }
}
__global__ void k_state_final(int nb, const double* __restrict__ partials, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kStateQ) return;
  double a = 0.0;
  for (int b = 0; b < nb; ++b) a += partials[size_t(b) * kStateQ + k];
  out[k] = a;
}

__global__ void k_gather_perf(int n_perfs, const int* __restrict__ cells, const double* __restrict__ p,
                              const double* __restrict__ sw, const double* __restrict__ hc, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_perfs) return;
  const int c = cells[k];
  out[3 * k] = p[c];
  out[3 * k + 1] = sw[c];
  out[3 * k + 2] = hc[c];
}

static int red_blocks(Ctx& c) {
  int nb = blocks_for(c.n);
  if (nb > 4 * c.num_sms) nb = 4 * c.num_sms;
  return nb;
}

void apply_cell_update(Ctx& c, double relax, double& pmax, bool& finite) {
  const int nb = red_blocks(c);
  k_apply_update<<<nb, kBlock, 0, c.stream>>>(c.n, relax, c.d_x.p, c.d_p.p, c.d_sw.p, c.d_hc.p, c.d_cp.p, c.d_csw.p,
                                              c.d_chc.p, c.d_partials.p);
  k_max2_final<<<1, 32, 0, c.stream>>>(nb, c.d_partials.p, c.d_scal.p + 200);
  c.launches += 2;
  double h[2];
  d2h(c, h, c.d_scal.p + 200, sizeof(h));
  d2h_wait(c);
  pmax = h[0];
  finite = h[1] == 0.0;
}

void max2_final(Ctx& c, int nb, double& pmax, bool& finite) {
  k_max2_final<<<1, 32, 0, c.stream>>>(nb, c.d_partials.p, c.d_scal.p + 200);
  c.launches++;
  double h[2];
  d2h(c, h, c.d_scal.p + 200, sizeof(h));
  d2h_wait(c);
  pmax = h[0];
  finite = h[1] == 0.0;
}

void state_sums(Ctx& c, const double* ap, const double* asw, const double* ahc, const double* bp, const double* bsw,
                const double* bhc, double out[7]) {
  const int nb = red_blocks(c);
  k_state_sums<<<nb, kBlock, 0, c.stream>>>(c.fluid, c.n, c.d_pv.p, ap, asw, ahc, bp, bsw, bhc, c.d_partials.p);
  k_state_final<<<1, 32, 0, c.stream>>>(nb, c.d_partials.p, c.d_scal.p + 210);
  c.launches += 2;
  d2h(c, out, c.d_scal.p + 210, sizeof(double) * kStateQ);
  d2h_wait(c);
}

void gather_perf_cells(Ctx& c, const double* p, const double* sw, const double* hc, std::vector<double>& out) {
  const int P = c.topo.n_perfs;
  out.assign(3 * size_t(P), 0.0);
  if (P == 0) return;
  double* d = c.d_scal.p + 1024;  // 3P <= 3072 doubles (checked at setup)
  k_gather_perf<<<blocks_for(P, 64), 64, 0, c.stream>>>(P, c.d_perf_cell.p, p, sw, hc, d);
  c.launches++;
  d2h(c, out.data(), d, sizeof(double) * 3 * P);
  d2h_wait(c);
}

}  // namespace rf
