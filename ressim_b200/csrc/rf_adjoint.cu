// rf_adjoint.cu — device kernels of the discrete adjoint (backward pass) of the fully implicit
// step.  The reference has no adjoint; this is the differentiation form of the device path.
//
// For accepted substeps n = N..1 with converged states x_n and residuals
// R_n(x_n, x_{n-1}, theta) = 0, the adjoint states solve
//     (dR_n/dx_n)^T lambda_n = -(dJ/dx_n)^T + A_n^T lambda_{n+1},
// where A_n = d inventory(x_n) / d x_n is the block-diagonal accumulation derivative through which
// x_n enters R_{n+1} as its previous state; then dJ/dtheta = sum_n lambda_n^T dR_n/dtheta.
//
// k_bsr_transpose  the reduced (well-eliminated) matrix S in place into S^T: the well Schur
//                  complement of J^T is the transpose of J's, (A - B D^-1 C)^T
// k_adj_accum      rhs += A_n^T lambda_{n+1}, A_n per cell from the dual-number inventory
// k_adj_grad       lambda_n^T dR_n/dtheta_i for theta_i = ln of cell i's permeability multiplier
//                  (kx, ky, kz scaled together): every face flux is linear in its
//                  transmissibility, so each face adds (lambda_lo - lambda_hi) . flux dt
//                  dlnT/dtheta_i (harmonic mean in x and y, the dz-weighted form in z,
//                  grid.rs:47-80)
#include "rf_blackoil.cuh"
#include "rf_ops.hpp"

namespace rf {

__global__ void k_bsr_transpose(int nnzb, const int* __restrict__ tpos, double* __restrict__ val) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nnzb) return;
  const int t = tpos[b];
  if (t < b) return;  // the pair is handled by its lower position
  double* x = val + size_t(b) * 9;
  double* y = val + size_t(t) * 9;
  if (t == b) {
    double a[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) a[e] = x[e];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int v = 0; v < 3; ++v) x[3 * r + v] = a[3 * v + r];
    return;
  }
  double a[9], z[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) {
    a[e] = x[e];
    z[e] = y[e];
  }
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      x[3 * r + v] = z[3 * v + r];
      y[3 * r + v] = a[3 * v + r];
    }
}

__global__ void __launch_bounds__(kBlock) k_adj_accum(const __grid_constant__ Fluid f, int n,
                                                       const double* __restrict__ pv, const int* __restrict__ reg,
                                                       const double* __restrict__ p, const double* __restrict__ sw,
                                                       const double* __restrict__ hc, const double* __restrict__ lam,
                                                       double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Dual<3> cd[3];
    if (f.three_phase)
      inventory3<Dual<3>>(f, pv[i], reg[i], dvar<3>(p[i], 0), dvar<3>(sw[i], 1), dvar<3>(hc[i], 2), 0.0, cd);
    else
      inventory<Dual<3>>(f, pv[i], dvar<3>(p[i], 0), dvar<3>(sw[i], 1), dvar<3>(hc[i], 2), cd);
    const double l0 = lam[3 * i], l1 = lam[3 * i + 1], l2 = lam[3 * i + 2];
#pragma unroll
    for (int v = 0; v < 3; ++v) out[3 * i + v] += cd[0].d[v] * l0 + cd[1].d[v] * l1 + cd[2].d[v] * l2;
  }
}

__device__ __forceinline__ void face_flux_any(const Fluid& f, double t, double dlo, double dhi, int rlo, double plo,
                                              double swlo, double hclo, int rhi, double phi, double swhi,
                                              double hchi, double fv[3]) {
  if (f.three_phase)
    face_flux3<double>(f, t, dlo, dhi, rlo, plo, swlo, hclo, rhi, phi, swhi, hchi, fv);
  else
    face_flux<double>(f, t, dlo, dhi, plo, swlo, phi, swhi, fv);
}

__global__ void __launch_bounds__(128) k_adj_grad(const __grid_constant__ Fluid f, int nx, int ny, int nz, double dt,
                                                   const double* __restrict__ tx, const double* __restrict__ ty,
                                                   const double* __restrict__ tz, const double* __restrict__ kx,
                                                   const double* __restrict__ ky, const double* __restrict__ kz,
                                                   const double* __restrict__ dz, const double* __restrict__ depth,
                                                   const int* __restrict__ reg, const double* __restrict__ p,
                                                   const double* __restrict__ sw, const double* __restrict__ hc,
                                                   const double* __restrict__ lam, double* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nxy = nx * ny;
  if (i >= nxy * nz) return;
  const int ci = i % nx, cj = (i / nx) % ny, ck = i / nxy;
  const int ri = reg ? reg[i] : 0;
  double g = 0.0;
  // the six faces: neighbour, transmissibility index (lower cell), axis 0 x / 1 y / 2 z
  const int nb[6] = {ck > 0 ? i - nxy : -1, cj > 0 ? i - nx : -1, ci > 0 ? i - 1 : -1,
                     ci + 1 < nx ? i + 1 : -1, cj + 1 < ny ? i + nx : -1, ck + 1 < nz ? i + nxy : -1};
  const int axis[6] = {2, 1, 0, 0, 1, 2};
  for (int s = 0; s < 6; ++s) {
    const int j = nb[s];
    if (j < 0) continue;
    const int lo = j < i ? j : i, hi = j < i ? i : j;
    const double t = axis[s] == 0 ? tx[lo] : (axis[s] == 1 ? ty[lo] : tz[lo]);
    if (!(t > 0.0)) continue;
    const int klo = lo / nxy, khi = hi / nxy;
    const int rlo = reg ? reg[lo] : 0, rhi = reg ? reg[hi] : 0;
    (void)ri;
    double fv[3];
    face_flux_any(f, t, depth[klo], depth[khi], rlo, p[lo], sw[lo], hc[lo], rhi, p[hi], sw[hi], hc[hi], fv);
    double dl = 0.0;
#pragma unroll
    for (int e = 0; e < 3; ++e) dl += (lam[3 * lo + e] - lam[3 * hi + e]) * fv[e] * dt;
    double w;
    if (axis[s] == 2) {
      const double p1 = kz[lo], p2 = kz[hi], den = p2 * dz[klo] + p1 * dz[khi];
      w = den > 0.0 ? (i == lo ? p2 * dz[klo] : p1 * dz[khi]) / den : 0.0;
    } else {
      const double* k = axis[s] == 0 ? kx : ky;
      const double sum = k[lo] + k[hi];
      w = sum > 0.0 ? (i == lo ? k[hi] : k[lo]) / sum : 0.0;
    }
    g += dl * w;
  }
  grad[i] += g;
}

__global__ void k_add_at(int m, const int* __restrict__ idx, const double* __restrict__ v, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) out[idx[k]] += v[k];
}

__global__ void k_gather_at(int m, const int* __restrict__ idx, const double* __restrict__ v, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) out[k] = v[idx[k]];
}

// ---- host launchers ----
void adj_transpose(Ctx& c, const int* d_tpos) {
  k_bsr_transpose<<<blocks_for(c.nnzb), kBlock, 0, c.stream>>>(c.nnzb, d_tpos, c.d_val.p);
  c.launches++;
}

void adj_accum(Ctx& c, const double* lam_next, double* out) {
  int nb = blocks_for(c.n);
  if (nb > 4 * c.num_sms) nb = 4 * c.num_sms;
  k_adj_accum<<<nb, kBlock, 0, c.stream>>>(c.fluid, c.n, c.d_pv.p, c.fluid.three_phase ? c.d_reg.p : nullptr, c.d_p.p,
                                           c.d_sw.p, c.d_hc.p, lam_next, out);
  c.launches++;
}

void adj_grad(Ctx& c, double dt, const double* kx, const double* ky, const double* kz, const double* dz,
              const double* lam, double* grad) {
  k_adj_grad<<<blocks_for(c.n, 128), 128, 0, c.stream>>>(c.fluid, c.nx, c.ny, c.nz, dt, c.d_tx.p, c.d_ty.p, c.d_tz.p,
                                                         kx, ky, kz, dz, c.d_depth.p,
                                                         c.fluid.three_phase ? c.d_reg.p : nullptr, c.d_p.p, c.d_sw.p,
                                                         c.d_hc.p, lam, grad);
  c.launches++;
}

// out[idx[k]] += v[k] for m host values (staged through the scalar scratch: m <= 3000)
void adj_add_at(Ctx& c, const std::vector<int>& idx, const std::vector<double>& v, double* out, int* d_idx) {
  const int m = int(idx.size());
  if (m == 0) return;
  RF_CUDA(cudaMemcpyAsync(d_idx, idx.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c.stream));
  RF_CUDA(cudaMemcpyAsync(c.d_scal.p + 5120, v.data(), sizeof(double) * m, cudaMemcpyHostToDevice, c.stream));
  k_add_at<<<blocks_for(m, 64), 64, 0, c.stream>>>(m, d_idx, c.d_scal.p + 5120, out);
  c.launches++;
}

// host copy of v[idx[k]] for m device values (m <= 3000)
void adj_gather_at(Ctx& c, const std::vector<int>& idx, const double* v, std::vector<double>& out, int* d_idx) {
  const int m = int(idx.size());
  out.assign(m, 0.0);
  if (m == 0) return;
  RF_CUDA(cudaMemcpyAsync(d_idx, idx.data(), sizeof(int) * m, cudaMemcpyHostToDevice, c.stream));
  k_gather_at<<<blocks_for(m, 64), 64, 0, c.stream>>>(m, d_idx, v, c.d_scal.p + 5120);
  c.launches++;
  d2h(c, out.data(), c.d_scal.p + 5120, sizeof(double) * m);
  d2h_wait(c);
}

}  // namespace rf
