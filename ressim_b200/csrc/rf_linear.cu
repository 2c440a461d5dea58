// rf_linear.cu — the linear solve of one Newton iteration on the device.
//
//   well Schur elimination     k_schur / k_recover: one CTA per physical well, dense local
//                              inverse in shared memory (fim/linear/well_schur.rs:70-471)
//   CPR build                  k_cpr_weights (QuasiImpes: row 0 of the inverse diagonal block,
//                              normalised by its largest magnitude), k_pressure_matrix
//                              (A_p[i,j] = sum_l w_i[l] A[(i,l),(j,0)]), level-scheduled
//                              pressure ILU0 and block ILU0 factorisations in the reference's
//                              natural order (gmres_block_jacobi.rs:178-353, 746-808, 919-1363)
//   CPR apply                  restrict -> coarse solve (dense inverse when N <= 299, else a
//                              one-cluster persistent BiCGStab with pressure ILU0, at most 50
//                              iterations, tol 1e-6 relative) -> prolong -> r - A x_p ->
//                              block-ILU0 sweep -> add (gmres_block_jacobi.rs:471-729)
//   FGMRES(30)                 right-preconditioned flexible GMRES, x0 = 0, modified
//                              Gram-Schmidt, true residual of the candidate every inner step,
//                              tolerance 1e-12 + 5e-3 |b| (gmres_block_jacobi.rs:1470-1665)
//
// A block is "present" in the ILU pattern when any of its entries exceeds EPS in magnitude (the
// reference builds its ILU0 pattern that way); absent blocks are held as zeros and receive no
// fill.  Pressure-matrix entries with |v| <= 1e-14 are dropped, as the reference does.

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <cstdio>

#include "rf_fiber.hpp"
#include "rf_ops.hpp"

namespace rf {

constexpr double kEps = kF64Eps;

// ============================================================================================
// small dense helpers
// ============================================================================================
__device__ __forceinline__ void mat3_mul(const double* a, const double* b, double* c) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int k = 0; k < 3; ++k) c[3 * r + k] = a[3 * r] * b[k] + a[3 * r + 1] * b[3 + k] + a[3 * r + 2] * b[6 + k];
}
// 3x3 inverse by cofactors; fails only on an exactly zero determinant, then the diagonal
// reciprocal fallback (gmres_block_jacobi.rs:888-901) is used.
__host__ __device__ __forceinline__ void mat3_inverse_or_diag(const double* m, double* o) {
  const double m11 = m[0], m12 = m[1], m13 = m[2], m21 = m[3], m22 = m[4], m23 = m[5], m31 = m[6], m32 = m[7],
               m33 = m[8];
  const double c11 = m22 * m33 - m32 * m23;
  const double c21 = m21 * m33 - m31 * m23;
  const double c31 = m21 * m32 - m31 * m22;
  const double det = m11 * c11 - m12 * c21 + m13 * c31;
  if (det != 0.0) {
    o[0] = c11 / det;
    o[1] = (m13 * m32 - m33 * m12) / det;
    o[2] = (m12 * m23 - m22 * m13) / det;
    o[3] = -c21 / det;
    o[4] = (m11 * m33 - m31 * m13) / det;
    o[5] = (m13 * m21 - m23 * m11) / det;
    o[6] = c31 / det;
    o[7] = (m12 * m31 - m32 * m11) / det;
    o[8] = (m11 * m22 - m21 * m12) / det;
    return;
  }
  for (int k = 0; k < 9; ++k) o[k] = 0.0;
  for (int d = 0; d < 3; ++d) {
    const double v = m[4 * d];
    o[4 * d] = fabs(v) > kEps ? 1.0 / v : 1.0;
  }
}

// ============================================================================================
// BSR SpMV and vector kernels
// ============================================================================================
// y = A x (mode 0) or y = b - A x (mode 1), thread per block row, blocks in column order.
template <int MODE>
__global__ void __launch_bounds__(kBlock) k_spmv(int nb, const int* __restrict__ rp, const int* __restrict__ col,
                                                  const double* __restrict__ val, const double* __restrict__ x,
                                                  const double* __restrict__ b, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const double* a = val + size_t(k) * 9;
    const int j = col[k];
    const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
    s0 = s0 + a[0] * x0;
    s0 = s0 + a[1] * x1;
    s0 = s0 + a[2] * x2;
    s1 = s1 + a[3] * x0;
    s1 = s1 + a[4] * x1;
    s1 = s1 + a[5] * x2;
    s2 = s2 + a[6] * x0;
    s2 = s2 + a[7] * x1;
    s2 = s2 + a[8] * x2;
  }
  if (MODE == 0) {
    y[3 * i] = s0;
    y[3 * i + 1] = s1;
    y[3 * i + 2] = s2;
  } else {
    y[3 * i] = b[3 * i] - s0;
    y[3 * i + 1] = b[3 * i + 1] - s1;
    y[3 * i + 2] = b[3 * i + 2] - s2;
  }
}

// partial sums of a*b (or a*a when b == nullptr) per block, grid-stride; final pass in k_sum_final
__global__ void __launch_bounds__(kBlock) k_dot_partial(long long n, const double* __restrict__ a,
                                                         const double* __restrict__ b, double* __restrict__ partials) {
  __shared__ double sh[32];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s += a[i] * (b ? b[i] : a[i]);
  const double r = block_sum<kBlock>(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}
__global__ void k_reduce_to(int nblocks, const double* __restrict__ partials, double* __restrict__ out, int take_sqrt) {
  if (threadIdx.x != 0) return;
  double a = 0.0;
  for (int b = 0; b < nblocks; ++b) a += partials[b];
  *out = take_sqrt ? sqrt(a) : a;
}
// w -= h * v with h read from device memory
__global__ void k_axpy_dev(long long n, const double* __restrict__ h, const double* __restrict__ v, double* __restrict__ w) {
  const double c = *h;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    w[i] -= v[i] * c;
}
// out = w / nrm (nrm from device memory)
__global__ void k_scale_div(long long n, const double* __restrict__ w, const double* __restrict__ nrm,
                            double* __restrict__ out) {
  const double d = *nrm;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = w[i] / d;
}
// cand = origin + sum_c Z_c y_c (y on the device), update accumulated from zero in column order
__global__ void k_combine(long long n, int cols, const double* __restrict__ Z, long long ld, const double* __restrict__ y,
                          const double* __restrict__ origin, double* __restrict__ cand) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double u = 0.0;
    for (int c = 0; c < cols; ++c) u += Z[c * ld + i] * y[c];
    cand[i] = origin ? origin[i] + u : u;
  }
}
__global__ void k_copy(long long n, const double* __restrict__ a, double* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}
__global__ void k_neg(long long n, const double* __restrict__ a, double* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = -a[i];
}
__global__ void k_add_inplace(long long n, const double* __restrict__ a, double* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] += a[i];
}
__global__ void k_count_nonfinite(long long n, const double* __restrict__ a, int* __restrict__ flag) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!isfinite(a[i])) atomicExch(flag, 1);
}

// ============================================================================================
// Well Schur elimination (one CTA per physical well)
// ============================================================================================
struct SchurArgs {
  int n_wells;
  const int* well_ptr;
  const int* well_perfs;
  const int* perf_cell;
  const int* perf_has_wi;
  const double* jrw;
  const double* jwr_perf;
  const double* jwr_ctrl;
  const double* jww_perf_bhp;
  const double* jww_ctrl_q;
  const double* jww_ctrl_bhp;
  const double* res;       // cell residual (rhs = -res)
  const double* res_tail;  // W + P
  const int* tinv_off;
  double* tinv;
  const int* row_ptr;
  const int* fill_off;
  const int* fill_pos;
  const int* perf_row_off;
  double* val;
  double* jrr_perf;
  double* rhs_red;  // holds -res for every cell on entry; perforated rows corrected here
};

// Gauss-Jordan inverse with partial pivoting of the nt x nt matrix in shared memory.  Returns
// false on an exactly zero pivot.
__device__ bool smem_gauss_jordan(double* a, double* inv, int nt, int* s_piv, double* s_red) {
  const int t = threadIdx.x, nt_threads = blockDim.x;
  for (int k = t; k < nt * nt; k += nt_threads) inv[k] = (k / nt == k % nt) ? 1.0 : 0.0;
  __syncthreads();
  for (int c = 0; c < nt; ++c) {
    if (t == 0) {
      int piv = c;
      double best = fabs(a[c * nt + c]);
      for (int r = c + 1; r < nt; ++r)
        if (fabs(a[r * nt + c]) > best) {
          best = fabs(a[r * nt + c]);
          piv = r;
        }
      s_piv[0] = piv;
      s_red[0] = best;
    }
    __syncthreads();
    if (s_red[0] == 0.0) return false;
    const int piv = s_piv[0];
    if (piv != c)
      for (int k = t; k < nt; k += nt_threads) {
        double x = a[c * nt + k];
        a[c * nt + k] = a[piv * nt + k];
        a[piv * nt + k] = x;
        x = inv[c * nt + k];
        inv[c * nt + k] = inv[piv * nt + k];
        inv[piv * nt + k] = x;
      }
    __syncthreads();
    const double d = a[c * nt + c];
    __syncthreads();
    for (int k = t; k < nt; k += nt_threads) {
      a[c * nt + k] /= d;
      inv[c * nt + k] /= d;
    }
    __syncthreads();
    for (int idx = t; idx < nt * nt; idx += nt_threads) {
      const int r = idx / nt, k = idx % nt;
      if (r == c) continue;
      const double f = a[r * nt + c];
      if (k != c) a[r * nt + k] -= f * a[c * nt + k];
      inv[r * nt + k] -= f * inv[c * nt + k];
    }
    __syncthreads();
    for (int r = t; r < nt; r += nt_threads)
      if (r != c) a[r * nt + c] = 0.0;
    __syncthreads();
  }
  return true;
}

__global__ void k_schur(SchurArgs s) {
  extern __shared__ double sm[];
  __shared__ int s_piv[1];
  __shared__ double s_red[1];
  const int w = blockIdx.x;
  const int p0 = s.well_ptr[w], m = s.well_ptr[w + 1] - p0, nt = 1 + m;
  double* J = sm;
  double* I = sm + nt * nt;
  double* rw = I + nt * nt;  // local rhs tail (nt)
  double* tir = rw + nt;     // inv * rhs tail (nt)
  const int t = threadIdx.x;
  for (int k = t; k < nt * nt; k += blockDim.x) J[k] = 0.0;
  __syncthreads();
  if (t == 0) {
    J[0] = s.jww_ctrl_bhp[w];
    rw[0] = -s.res_tail[w];
    for (int a = 0; a < m; ++a) {
      const int k = s.well_perfs[p0 + a];
      J[1 + a] = s.jww_ctrl_q[k];
      J[(1 + a) * nt] = s.jww_perf_bhp[k];
      J[(1 + a) * nt + 1 + a] = s.perf_has_wi[k] ? 1.0 : 0.0;
      rw[1 + a] = -s.res_tail[s.n_wells + k];
    }
  }
  __syncthreads();
  // keep the assembled tail block's diagonal for the singular fallback
  __shared__ double s_diag[257];
  for (int r = t; r < nt && r < 257; r += blockDim.x) s_diag[r] = J[r * nt + r];
  __syncthreads();
  const bool ok = smem_gauss_jordan(J, I, nt, s_piv, s_red);
  __syncthreads();
  if (!ok) {
    for (int k = t; k < nt * nt; k += blockDim.x) I[k] = 0.0;
    __syncthreads();
    for (int r = t; r < nt && r < 257; r += blockDim.x) I[r * nt + r] = fabs(s_diag[r]) > kEps ? 1.0 / s_diag[r] : 1.0;
    __syncthreads();
  }
  double* tg = s.tinv + s.tinv_off[w];
  for (int k = t; k < nt * nt; k += blockDim.x) tg[k] = I[k];
  // inv * rhs_tail
  for (int r = t; r < nt; r += blockDim.x) {
    double acc = 0.0;
    for (int c = 0; c < nt; ++c) acc += I[r * nt + c] * rw[c];
    tir[r] = acc;
  }
  // save the original (pre-fill) blocks of every perforated row
  for (int a = 0; a < m; ++a) {
    const int k = s.well_perfs[p0 + a], cell = s.perf_cell[k];
    const int b0 = s.row_ptr[cell], b1 = s.row_ptr[cell + 1];
    double* dst = s.jrr_perf + size_t(s.perf_row_off[k]) * 9;
    for (int e = t; e < (b1 - b0) * 9; e += blockDim.x) dst[e] = s.val[size_t(b0) * 9 + e];
  }
  __syncthreads();
  // fill: block(a, b) -= jrw_a * inv[1+a][.] * J_WR[., b]
  for (int pr = t; pr < m * m * 9; pr += blockDim.x) {
    const int a = pr / (m * 9), b = (pr / 9) % m, e = pr % 9, r = e / 3, v = e % 3;
    const int ka = s.well_perfs[p0 + a], kb = s.well_perfs[p0 + b];
    const double j = s.jrw[3 * ka + r];
    if (fabs(j) <= kEps) continue;
    const double wc = 0.0 + j * I[(1 + a) * nt + 0];
    const double wp = 0.0 + j * I[(1 + a) * nt + 1 + b];
    const int pos = s.fill_pos[s.fill_off[w] + a * m + b];
    double* blk = s.val + size_t(pos) * 9;
    double x = blk[e];
    const double jc = s.jwr_ctrl[3 * kb + v], jp = s.jwr_perf[3 * kb + v];
    if (fabs(wc) > kEps && fabs(jc) > kEps) x += -wc * jc;
    if (fabs(wp) > kEps && fabs(jp) > kEps) x += -wp * jp;
    blk[e] = x;
  }
  // reduced rhs of the perforated rows
  for (int idx = t; idx < m * 3; idx += blockDim.x) {
    const int a = idx / 3, r = idx % 3;
    const int k = s.well_perfs[p0 + a], cell = s.perf_cell[k];
    const double j = s.jrw[3 * k + r];
    if (fabs(j) <= kEps) continue;
    const double corr = 0.0 + j * tir[1 + a];
    s.rhs_red[3 * cell + r] -= corr;
  }
}

struct RecoverArgs {
  int n_wells;
  const int* well_ptr;
  const int* well_perfs;
  const int* perf_cell;
  const int* perf_has_wi;
  const double* jrw;
  const double* jwr_perf;
  const double* jwr_ctrl;
  const double* jww_perf_bhp;
  const double* jww_ctrl_q;
  const double* jww_ctrl_bhp;
  const double* res;
  const double* res_tail;
  const int* tinv_off;
  const double* tinv;
  const double* x;  // reduced solution
  double* dx_tail;  // W + P
  const int* row_ptr;
  const int* col;
  const int* perf_row_off;
  const double* jrr_perf;
  double* full;       // full-system residual of the reservoir rows (perforated rows rewritten)
  double* tail_sq;    // per well: sum of squared full-system residual of its tail rows
};

__global__ void k_recover(RecoverArgs s) {
  const int w = blockIdx.x;
  if (threadIdx.x != 0) return;
  const int p0 = s.well_ptr[w], m = s.well_ptr[w + 1] - p0, nt = 1 + m;
  const double* I = s.tinv + s.tinv_off[w];
  double rt[257];
  const int ntc = nt < 257 ? nt : 257;
  {
    double acc = 0.0;
    for (int a = 0; a < m; ++a) {
      const int k = s.well_perfs[p0 + a], c = s.perf_cell[k];
      for (int v = 0; v < 3; ++v) {
        const double j = s.jwr_ctrl[3 * k + v];
        if (fabs(j) > kEps) acc += j * s.x[3 * c + v];
      }
    }
    rt[0] = -s.res_tail[w] - acc;
  }
  for (int a = 0; a < m && a + 1 < ntc; ++a) {
    const int k = s.well_perfs[p0 + a], c = s.perf_cell[k];
    double acc = 0.0;
    for (int v = 0; v < 3; ++v) {
      const double j = s.jwr_perf[3 * k + v];
      if (fabs(j) > kEps) acc += j * s.x[3 * c + v];
    }
    rt[1 + a] = -s.res_tail[s.n_wells + k] - acc;
  }
  double dx[257];
  for (int r = 0; r < ntc; ++r) {
    double acc = 0.0;
    for (int c = 0; c < ntc; ++c) acc += I[r * nt + c] * rt[c];
    dx[r] = acc;
  }
  s.dx_tail[w] = dx[0];
  for (int a = 0; a < m && a + 1 < ntc; ++a) s.dx_tail[s.n_wells + s.well_perfs[p0 + a]] = dx[1 + a];
  // full-system residual of this well's perforated rows and tail rows
  double sq = 0.0;
  {
    double acc = 0.0;
    for (int a = 0; a < m; ++a) {
      const int k = s.well_perfs[p0 + a], c = s.perf_cell[k];
      for (int v = 0; v < 3; ++v) acc += s.jwr_ctrl[3 * k + v] * s.x[3 * c + v];
    }
    acc += s.jww_ctrl_bhp[w] * dx[0];
    for (int a = 0; a < m && a + 1 < ntc; ++a) acc += s.jww_ctrl_q[s.well_perfs[p0 + a]] * dx[1 + a];
    const double r = -s.res_tail[w] - acc;
    sq += r * r;
  }
  for (int a = 0; a < m && a + 1 < ntc; ++a) {
    const int k = s.well_perfs[p0 + a], c = s.perf_cell[k];
    double acc = 0.0;
    for (int v = 0; v < 3; ++v) acc += s.jwr_perf[3 * k + v] * s.x[3 * c + v];
    acc += s.jww_perf_bhp[k] * dx[0];
    acc += (s.perf_has_wi[k] ? 1.0 : 0.0) * dx[1 + a];
    const double r = -s.res_tail[s.n_wells + k] - acc;
    sq += r * r;
    // reservoir rows of the perforated cell, from the original (pre-fill) blocks
    const int b0 = s.row_ptr[c], b1 = s.row_ptr[c + 1];
    const double* blk0 = s.jrr_perf + size_t(s.perf_row_off[k]) * 9;
    for (int e = 0; e < 3; ++e) {
      double acc2 = 0.0;
      for (int b = b0; b < b1; ++b) {
        const double* blk = blk0 + size_t(b - b0) * 9;
        const int j = s.col[b];
        acc2 += blk[3 * e] * s.x[3 * j];
        acc2 += blk[3 * e + 1] * s.x[3 * j + 1];
        acc2 += blk[3 * e + 2] * s.x[3 * j + 2];
      }
      acc2 += s.jrw[3 * k + e] * dx[1 + a];
      s.full[3 * c + e] = -s.res[3 * c + e] - acc2;
    }
  }
  s.tail_sq[w] = sq;
}

// ============================================================================================
// CPR build
// ============================================================================================
// QuasiImpes restriction weights from the diagonal block and the block presence mask
__global__ void k_cpr_weights(int nb, const int* __restrict__ rp, const int* __restrict__ diag,
                              const double* __restrict__ val, double* __restrict__ w,
                              unsigned char* __restrict__ mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  double inv[9];
  mat3_inverse_or_diag(val + size_t(diag[i]) * 9, inv);
  double r0 = inv[0], r1 = inv[1], r2 = inv[2];
  const double mx = fmax(fmax(fmax(0.0, fabs(r0)), fabs(r1)), fabs(r2));
  if (mx > kEps) {
    r0 /= mx;
    r1 /= mx;
    r2 /= mx;
  }
  w[3 * i] = r0;
  w[3 * i + 1] = r1;
  w[3 * i + 2] = r2;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const double* a = val + size_t(k) * 9;
    bool present = (k == diag[i]);
    for (int e = 0; e < 9; ++e) present = present || fabs(a[e]) > kEps;
    mask[k] = present ? 1 : 0;
  }
}

// Transposed-system CPR (the adjoint's solves on S^T): the transpose of the forward two-stage
// operator's coarse correction, P A_p^-1 R -> R^T A_p^-T P^T, with the forward weights.  The
// weights of S (row 0 of S_ii^-1) are column 0 of (S^T)_ii^-1; the coarse matrix is
// A_p^T[i, j] = sum_l S^T[(i,0),(j,l)] w_j[l]; restriction takes the pressure component and
// prolongation spreads the correction with the weights.  The block-ILU0 smoother factors S^T.
__global__ void k_cpr_weights_t(int nb, const int* __restrict__ rp, const int* __restrict__ diag,
                                const double* __restrict__ val, double* __restrict__ w,
                                unsigned char* __restrict__ mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  double inv[9];
  mat3_inverse_or_diag(val + size_t(diag[i]) * 9, inv);
  double r0 = inv[0], r1 = inv[3], r2 = inv[6];
  const double mx = fmax(fmax(fmax(0.0, fabs(r0)), fabs(r1)), fabs(r2));
  if (mx > kEps) {
    r0 /= mx;
    r1 /= mx;
    r2 /= mx;
  }
  w[3 * i] = r0;
  w[3 * i + 1] = r1;
  w[3 * i + 2] = r2;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const double* a = val + size_t(k) * 9;
    bool present = (k == diag[i]);
    for (int e = 0; e < 9; ++e) present = present || fabs(a[e]) > kEps;
    mask[k] = present ? 1 : 0;
  }
}
__global__ void k_pressure_matrix_t(int nb, const int* __restrict__ rp, const int* __restrict__ col,
                                    const double* __restrict__ val, const double* __restrict__ w,
                                    double* __restrict__ pval) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const double* a = val + size_t(k) * 9;
    const int j = col[k];
    const double s = a[0] * w[3 * j] + a[1] * w[3 * j + 1] + a[2] * w[3 * j + 2];
    pval[k] = fabs(s) > 1e-14 ? s : 0.0;
  }
}

// A_p[i, j] = ((0 + w0 A[(i,0),(j,0)]) + w1 A[(i,1),(j,0)]) + w2 A[(i,2),(j,0)]; |A_p| <= 1e-14 -> 0
__global__ void k_pressure_matrix(int nb, const int* __restrict__ rp, const double* __restrict__ val,
                                  const double* __restrict__ w, double* __restrict__ pval) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const double w0 = w[3 * i], w1 = w[3 * i + 1], w2 = w[3 * i + 2];
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const double* a = val + size_t(k) * 9;
    double s = 0.0;
    // entries whose row weight is <= EPS are skipped, and so are zero matrix entries (absent from
    // the reference's CSR)
    if (fabs(w0) > kEps && a[0] != 0.0) s += w0 * a[0] * 1.0;
    if (fabs(w1) > kEps && a[3] != 0.0) s += w1 * a[3] * 1.0;
    if (fabs(w2) > kEps && a[6] != 0.0) s += w2 * a[6] * 1.0;
    pval[k] = fabs(s) > 1e-14 ? s : 0.0;
  }
}

// Pressure ILU0, one row (factorize_pressure_ilu0's up-looking order).  `plu` holds L in the
// lower positions and U in the upper positions; absent entries (A_p == 0) stay zero.
__device__ __forceinline__ double upper_entry(const int* rp, const int* col, const int* diag, const double* plu,
                                              int k, int c) {
  int lo = diag[k] + 1, hi = rp[k + 1] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int cm = col[mid];
    if (cm == c) return plu[mid];
    if (cm < c)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return 0.0;
}
__device__ void pressure_ilu_row(int r, const int* rp, const int* col, const int* diag, const double* pval,
                                 double* plu, double* pdiag) {
  const int b0 = rp[r], dp = diag[r], b1 = rp[r + 1];
  for (int kp = b0; kp < dp; ++kp) {
    if (pval[kp] == 0.0) {
      plu[kp] = 0.0;
      continue;
    }
    const int c = col[kp];
    double s = pval[kp];
    for (int lp = b0; lp < kp; ++lp) {
      if (pval[lp] == 0.0) continue;
      s -= plu[lp] * upper_entry(rp, col, diag, plu, col[lp], c);
    }
    const double d = pdiag[c];
    plu[kp] = fabs(d) > kEps ? s / d : 0.0;
  }
  const double de = pval[dp];
  double ud = de;
  for (int lp = b0; lp < dp; ++lp) {
    if (pval[lp] == 0.0) continue;
    ud -= plu[lp] * upper_entry(rp, col, diag, plu, col[lp], r);
  }
  if (fabs(ud) <= kEps) ud = fabs(de) > kEps ? de : 1.0;
  pdiag[r] = ud;
  plu[dp] = 0.0;
  for (int up = dp + 1; up < b1; ++up) {
    if (pval[up] == 0.0) {
      plu[up] = 0.0;
      continue;
    }
    const int c = col[up];
    double s = pval[up];
    for (int lp = b0; lp < dp; ++lp) {
      if (pval[lp] == 0.0) continue;
      s -= plu[lp] * upper_entry(rp, col, diag, plu, col[lp], c);
    }
    plu[up] = s;
  }
}

// Block ILU0, one row (factorize_block_ilu0's IKJ order).
__device__ void block_ilu_row(int i, const int* rp, const int* col, const int* diag, const double* val,
                              const unsigned char* mask, double* lu, double* dinv) {
  const int b0 = rp[i], dp = diag[i], b1 = rp[i + 1];
  for (int k = b0; k < b1; ++k)
    for (int e = 0; e < 9; ++e) lu[size_t(k) * 9 + e] = mask[k] ? val[size_t(k) * 9 + e] : 0.0;
  for (int kp = b0; kp < dp; ++kp) {
    if (!mask[kp]) continue;
    const int kr = col[kp];
    double lik[9];
    mat3_mul(lu + size_t(kp) * 9, dinv + size_t(kr) * 9, lik);
    // U-row of kr: present blocks right of its diagonal; merge with row i's present blocks
    int ip = kp + 1;
    for (int up = diag[kr] + 1; up < rp[kr + 1]; ++up) {
      if (!mask[up]) continue;
      const int j = col[up];
      while (ip < b1 && col[ip] < j) ++ip;
      if (ip >= b1) break;
      if (col[ip] != j || !mask[ip]) continue;
      double prod[9];
      mat3_mul(lik, lu + size_t(up) * 9, prod);
      double* t = lu + size_t(ip) * 9;
      for (int e = 0; e < 9; ++e) t[e] -= prod[e];
    }
    for (int e = 0; e < 9; ++e) lu[size_t(kp) * 9 + e] = lik[e];
  }
  mat3_inverse_or_diag(lu + size_t(dp) * 9, dinv + size_t(i) * 9);
}

// Both ILU0 rows of a long row (a perforated cell's row with its well's fill) by one warp.  Its
// work grows with the square of its length, so one thread per row made these rows the longest
// step of their levels.  Every element gets the same operations in the same order as in
// block_ilu_row / pressure_ilu_row:
//  - block: for each present lower block kp in turn (all lanes form L_ik from the row's current
//    block, the same value in every lane), the lanes share the U-row of col[kp]; each U entry
//    updates at most one block of row i, so one kp's updates are independent;
//  - pressure, lower part: for each kp in turn the lanes look up the terms plu[lp] U(col[lp], c)
//    of all earlier lp in parallel and lane 0 sums them in lp order (rows of at most 32 lower
//    entries; longer ones are done by lane 0 alone); the diagonal likewise; upper entries: one
//    lane per entry, each summing over lp in order.
__device__ void ilu_rows_warp(int i, const int* rp, const int* col, const int* diag, const double* val,
                              const unsigned char* mask, double* lu, double* dinv, const double* pval, double* plu,
                              double* pdiag) {
  const int lane = threadIdx.x & 31;
  const int b0 = rp[i], dp = diag[i], b1 = rp[i + 1];
  for (int k = b0 + lane; k < b1; k += 32)
    for (int e = 0; e < 9; ++e) lu[size_t(k) * 9 + e] = mask[k] ? val[size_t(k) * 9 + e] : 0.0;
  __syncwarp();
  for (int kp = b0; kp < dp; ++kp) {
    if (!mask[kp]) continue;
    const int kr = col[kp];
    double lik[9];
    mat3_mul(lu + size_t(kp) * 9, dinv + size_t(kr) * 9, lik);
    __syncwarp();
    for (int up = diag[kr] + 1 + lane; up < rp[kr + 1]; up += 32) {
      if (!mask[up]) continue;
      const int j = col[up];
      int lo = kp + 1, hi = b1 - 1, t = -1;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int cm = col[mid];
        if (cm == j) {
          t = mid;
          break;
        }
        if (cm < j)
          lo = mid + 1;
        else
          hi = mid - 1;
      }
      if (t < 0 || !mask[t]) continue;
      double prod[9];
      mat3_mul(lik, lu + size_t(up) * 9, prod);
      double* tb = lu + size_t(t) * 9;
      for (int e = 0; e < 9; ++e) tb[e] -= prod[e];
    }
    __syncwarp();
    if (lane == 0)
      for (int e = 0; e < 9; ++e) lu[size_t(kp) * 9 + e] = lik[e];
    __syncwarp();
  }
  if (lane == 0) mat3_inverse_or_diag(lu + size_t(dp) * 9, dinv + size_t(i) * 9);
  // pressure ILU0
  if (dp - b0 > 32) {
    if (lane == 0) pressure_ilu_row(i, rp, col, diag, pval, plu, pdiag);
    __syncwarp();
    return;
  }
  for (int kp = b0; kp < dp; ++kp) {
    if (pval[kp] == 0.0) {
      if (lane == 0) plu[kp] = 0.0;
      __syncwarp();
      continue;
    }
    const int c = col[kp];
    const int lp = b0 + lane;
    double term = 0.0;
    if (lp < kp && pval[lp] != 0.0) term = plu[lp] * upper_entry(rp, col, diag, plu, col[lp], c);
    double sum = pval[kp];
    for (int q = b0; q < kp; ++q) {
      const double tq = __shfl_sync(0xffffffffu, term, q - b0);
      if (pval[q] != 0.0) sum -= tq;
    }
    if (lane == 0) {
      const double d = pdiag[c];
      plu[kp] = fabs(d) > kEps ? sum / d : 0.0;
    }
    __syncwarp();
  }
  {
    const double de = pval[dp];
    const int lp = b0 + lane;
    double term = 0.0;
    if (lp < dp && pval[lp] != 0.0) term = plu[lp] * upper_entry(rp, col, diag, plu, col[lp], i);
    double ud = de;
    for (int q = b0; q < dp; ++q) {
      const double tq = __shfl_sync(0xffffffffu, term, q - b0);
      if (pval[q] != 0.0) ud -= tq;
    }
    if (lane == 0) {
      if (fabs(ud) <= kEps) ud = fabs(de) > kEps ? de : 1.0;
      pdiag[i] = ud;
      plu[dp] = 0.0;
    }
  }
  for (int up = dp + 1 + lane; up < b1; up += 32) {
    if (pval[up] == 0.0) {
      plu[up] = 0.0;
      continue;
    }
    const int c = col[up];
    double s = pval[up];
    for (int lp = b0; lp < dp; ++lp) {
      if (pval[lp] == 0.0) continue;
      s -= plu[lp] * upper_entry(rp, col, diag, plu, col[lp], c);
    }
    plu[up] = s;
  }
  __syncwarp();
}

// Level-scheduled triangular work: rows of level l depend only on rows of lower levels, so each
// level is one parallel pass followed by a barrier.  The row arithmetic is the reference's, in the
// reference's order, so factors and solves equal the natural-order sequential ones.
//
// These kernels run as ONE thread-block cluster (up to 16 CTAs of 512-1024 threads) and separate
// the levels with the hardware cluster barrier (barrier.cluster arrive.release / wait.acquire):
// a level of a 7-point grid holds at most a few thousand rows, so a cluster covers it in one pass,
// and the per-level cost is the cluster barrier instead of a grid-wide software barrier through
// L2.  Every thread of every CTA takes the same number of barriers (loop bounds are uniform), so no
// wait can be left open.  Vectors written by other CTAs inside the same launch are read with
// ld.global.cg (L2), never from a possibly stale L1 line.
constexpr int kCBlock = 1024;      // threads per CTA: sweeps and BiCGStab
constexpr int kFBlock = 512;       // threads per CTA: factorisation (more registers per row)
constexpr int kSmemLevels = 4096;  // level pointers staged in shared memory up to this many levels

struct LevelSched {
  int n_levels;
  const int* lvl_rows;
  const int* lvl_ptr;
  const int* rp;
  const int* col;
  const int* diag;
  const int* long_rows;  // rows of more than kLongRowBlocks blocks, per level (factorisation only)
  const int* long_ptr;
};

__device__ __forceinline__ void cluster_barrier() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ unsigned cluster_nblocks() {
  unsigned v;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(v));
  return v;
}

// level pointers from shared memory when they fit (one fewer dependent global load per level)
__device__ __forceinline__ const int* stage_levels(const LevelSched& L, int* s_ptr) {
  if (L.n_levels + 1 <= kSmemLevels) {
    for (int i = threadIdx.x; i <= L.n_levels; i += blockDim.x) s_ptr[i] = L.lvl_ptr[i];
    __syncthreads();
    return s_ptr;
  }
  return L.lvl_ptr;
}

// Precomputed update lists of the factorisation (built once per pattern): for each lower entry kp
// of a row, the pairs (up, ip) of the U-row of col[kp] whose column the row also holds (the
// merge block_ilu_row performs); for each entry k of a row, the terms (lp, ue) of the pressure ILU
// (pressure_ilu_row's lower entries lp before it whose row holds the column of k above its
// diagonal, at entry ue).  Present-entry checks on the values stay at run time.
struct FacRecipes {
  const int* tri_ptr;  // [nnzb + 1]
  const int* tri_up;
  const int* tri_ip;
  const int* pt_ptr;   // [nnzb + 1]
  const int* pt_lp;
  const int* pt_ue;
  const unsigned char* simple;  // [n] 1: the row takes ilu_row_simple
};

struct FacArgs {
  LevelSched L;
  const double* val;
  const unsigned char* mask;
  double* lu;
  double* dinv;
  const double* pval;
  double* plu;
  double* pdiag;
  FacRecipes R;  // tri_ptr == nullptr: search as block_ilu_row / pressure_ilu_row do
};

// Both ILU0 rows of row i from the update lists: the same operations in the same order as
// block_ilu_row and pressure_ilu_row.
__device__ void ilu_row_recipe(int i, const FacArgs& a) {
  const int* rp = a.L.rp;
  const int* col = a.L.col;
  const int b0 = rp[i], dp = a.L.diag[i], b1 = rp[i + 1];
  const FacRecipes& R = a.R;
  for (int k = b0; k < b1; ++k) {
    const bool m = a.mask[k];
    for (int e = 0; e < 9; ++e) a.lu[size_t(k) * 9 + e] = m ? a.val[size_t(k) * 9 + e] : 0.0;
  }
  for (int kp = b0; kp < dp; ++kp) {
    if (!a.mask[kp]) continue;
    double lik[9];
    mat3_mul(a.lu + size_t(kp) * 9, a.dinv + size_t(col[kp]) * 9, lik);
    for (int e = R.tri_ptr[kp]; e < R.tri_ptr[kp + 1]; ++e) {
      const int up = R.tri_up[e], ip = R.tri_ip[e];
      if (!a.mask[up] || !a.mask[ip]) continue;
      double prod[9];
      mat3_mul(lik, a.lu + size_t(up) * 9, prod);
      double* t = a.lu + size_t(ip) * 9;
      for (int q = 0; q < 9; ++q) t[q] -= prod[q];
    }
    for (int q = 0; q < 9; ++q) a.lu[size_t(kp) * 9 + q] = lik[q];
  }
  mat3_inverse_or_diag(a.lu + size_t(dp) * 9, a.dinv + size_t(i) * 9);
  // pressure ILU0
  auto terms = [&](int k, double s) {
    for (int e = R.pt_ptr[k]; e < R.pt_ptr[k + 1]; ++e) {
      const int lp = R.pt_lp[e];
      if (a.pval[lp] == 0.0) continue;
      s -= a.plu[lp] * a.plu[R.pt_ue[e]];
    }
    return s;
  };
  for (int kp = b0; kp < dp; ++kp) {
    if (a.pval[kp] == 0.0) {
      a.plu[kp] = 0.0;
      continue;
    }
    const double s = terms(kp, a.pval[kp]);
    const double d = a.pdiag[col[kp]];
    a.plu[kp] = fabs(d) > kEps ? s / d : 0.0;
  }
  const double de = a.pval[dp];
  double ud = terms(dp, de);
  if (fabs(ud) <= kEps) ud = fabs(de) > kEps ? de : 1.0;
  a.pdiag[i] = ud;
  a.plu[dp] = 0.0;
  for (int up = dp + 1; up < b1; ++up) {
    if (a.pval[up] == 0.0) {
      a.plu[up] = 0.0;
      continue;
    }
    a.plu[up] = terms(up, a.pval[up]);
  }
}
// Both ILU0 rows of a "simple" row, the shape of every 7-point stencil row: at most kSimpleLower
// lower entries, each updating only the diagonal block (at most one pair per lower entry, its
// target the diagonal), and pressure terms only on the diagonal.  Then no lower entry changes
// before it is used, so the row's inputs (its own values, the lower columns' inverse diagonal
// blocks and pivots, the U blocks and pressure factors the updates read) are all loaded first, in
// a few independent rounds, instead of the chain of dependent loads the general walk takes.  The
// arithmetic is ilu_row_recipe's, in its order: L_ik = lu_kp Dinv_col[kp], the diagonal minus
// L_ik U_up in kp order, the pressure lower entries s / d, the diagonal's terms in list order.
constexpr int kSimpleLower = 4;
__device__ void ilu_row_simple(int i, const FacArgs& a) {
  const int* rp = a.L.rp;
  const int* col = a.L.col;
  const FacRecipes& R = a.R;
  const int b0 = __ldg(rp + i), dp = __ldg(a.L.diag + i), b1 = __ldg(rp + i + 1);
  const int nl = dp - b0;
  // structure (read-only in this kernel)
  int ck[kSimpleLower], up[kSimpleLower];
  bool mk[kSimpleLower];
  double pv[kSimpleLower];
#pragma unroll
  for (int j = 0; j < kSimpleLower; ++j) {
    ck[j] = 0;
    up[j] = -1;
    mk[j] = false;
    pv[j] = 0.0;
    if (j < nl) {
      const int k = b0 + j;
      ck[j] = __ldg(col + k);
      mk[j] = __ldg(a.mask + k) != 0;
      pv[j] = __ldg(a.pval + k);
      const int e0 = __ldg(R.tri_ptr + k), e1 = __ldg(R.tri_ptr + k + 1);
      if (e1 > e0) up[j] = __ldg(R.tri_up + e0);
    }
  }
  const bool md = __ldg(a.mask + dp) != 0;
  double D[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) D[e] = md ? __ldg(a.val + size_t(dp) * 9 + e) : 0.0;
  // block ILU0: each present lower entry's L_ik, and its update of the diagonal in kp order; the
  // row's stores wait until all its loads are issued
  double lik[kSimpleLower][9];
#pragma unroll
  for (int j = 0; j < kSimpleLower; ++j) {
#pragma unroll
    for (int e = 0; e < 9; ++e) lik[j][e] = 0.0;
    if (j >= nl || !mk[j]) continue;
    const int k = b0 + j;
    double lk[9], dk[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      lk[e] = __ldg(a.val + size_t(k) * 9 + e);
      dk[e] = a.dinv[size_t(ck[j]) * 9 + e];
    }
    mat3_mul(lk, dk, lik[j]);
    if (up[j] >= 0 && md && __ldg(a.mask + up[j])) {
      double u[9], prod[9];
#pragma unroll
      for (int e = 0; e < 9; ++e) u[e] = a.lu[size_t(up[j]) * 9 + e];
      mat3_mul(lik[j], u, prod);
#pragma unroll
      for (int e = 0; e < 9; ++e) D[e] -= prod[e];
    }
  }
#pragma unroll
  for (int j = 0; j < kSimpleLower; ++j)
    if (j < nl) {
#pragma unroll
      for (int e = 0; e < 9; ++e) a.lu[size_t(b0 + j) * 9 + e] = lik[j][e];
    }
  for (int k = dp + 1; k < b1; ++k) {
    const bool m = __ldg(a.mask + k) != 0;
#pragma unroll
    for (int e = 0; e < 9; ++e) a.lu[size_t(k) * 9 + e] = m ? __ldg(a.val + size_t(k) * 9 + e) : 0.0;
  }
#pragma unroll
  for (int e = 0; e < 9; ++e) a.lu[size_t(dp) * 9 + e] = D[e];
  mat3_inverse_or_diag(D, a.dinv + size_t(i) * 9);
  // pressure ILU0: lower entries (no terms), the diagonal's terms in list order, upper entries
  double pl[kSimpleLower];
#pragma unroll
  for (int j = 0; j < kSimpleLower; ++j) {
    pl[j] = 0.0;
    if (j < nl && pv[j] != 0.0) {
      const double d = a.pdiag[ck[j]];
      pl[j] = fabs(d) > kEps ? pv[j] / d : 0.0;
    }
    if (j < nl) a.plu[b0 + j] = pl[j];
  }
  const double de = __ldg(a.pval + dp);
  double ud = de;
  for (int e = __ldg(R.pt_ptr + dp); e < __ldg(R.pt_ptr + dp + 1); ++e) {
    const int jl = __ldg(R.pt_lp + e) - b0;
    double plp = 0.0, pvl = 0.0;
#pragma unroll
    for (int j = 0; j < kSimpleLower; ++j)
      if (j == jl) {
        plp = pl[j];
        pvl = pv[j];
      }
    if (pvl == 0.0) continue;
    ud -= plp * a.plu[__ldg(R.pt_ue + e)];
  }
  if (fabs(ud) <= kEps) ud = fabs(de) > kEps ? de : 1.0;
  a.pdiag[i] = ud;
  a.plu[dp] = 0.0;
  for (int k = dp + 1; k < b1; ++k) {
    const double v = __ldg(a.pval + k);
    a.plu[k] = v == 0.0 ? 0.0 : v;
  }
}

// Both ILU0 rows of a row of at most 32 blocks (a perforated cell's row with its well's fill) by
// one warp, from the update lists: lane j holds entry b0 + j of the row in registers, so the
// sequential walk over the row's lower entries costs shuffles instead of global round trips.
// Every element gets the operations of block_ilu_row / pressure_ilu_row in their order:
//  - block: for each present lower entry kp in turn, every lane forms L_ik = lu_kp Dinv_col[kp]
//    (both shuffled from lane kp); lane e takes the e-th pair (up, ip) of kp's list and forms
//    L_ik U_up; lane ip - b0 subtracts it from its block (each pair updates a different block);
//    lane kp's block becomes L_ik;
//  - pressure: each lower entry in turn, its terms plu[lp] U(col[lp], c) formed by one lane each
//    and summed in list order; then the diagonal; the upper entries each by their own lane.
// s_src and s_pl are this warp's 32-entry shared-memory scratch.
__device__ void ilu_rows_lanes(int i, const FacArgs& a, int* s_src, double* s_pl) {
  constexpr unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int* rp = a.L.rp;
  const int* col = a.L.col;
  const FacRecipes& R = a.R;
  const int b0 = rp[i], dp = a.L.diag[i], b1 = rp[i + 1];
  const int len = b1 - b0, nl = dp - b0;
  const int k = b0 + lane;
  const bool own = lane < len;
  const bool m = own && a.mask[k];
  double blk[9], dv[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) blk[e] = m ? a.val[size_t(k) * 9 + e] : 0.0;
  const int ck = own ? col[k] : 0;
#pragma unroll
  for (int e = 0; e < 9; ++e) dv[e] = lane < nl ? a.dinv[size_t(ck) * 9 + e] : 0.0;
  const unsigned present = __ballot_sync(kAll, m);
  for (int kp = 0; kp < nl; ++kp) {
    if (!((present >> kp) & 1u)) continue;  // uniform over the warp
    double lk[9], dk[9], lik[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      lk[e] = __shfl_sync(kAll, blk[e], kp);
      dk[e] = __shfl_sync(kAll, dv[e], kp);
    }
    mat3_mul(lk, dk, lik);
    const int e0 = R.tri_ptr[b0 + kp], np = R.tri_ptr[b0 + kp + 1] - e0;
    int tgt = -1;
    double prod[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) prod[e] = 0.0;
    if (lane < np) {
      const int up = R.tri_up[e0 + lane], ip = R.tri_ip[e0 + lane];
      if (a.mask[up] && a.mask[ip]) {
        double u[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) u[e] = a.lu[size_t(up) * 9 + e];
        mat3_mul(lik, u, prod);
        tgt = ip - b0;
      }
    }
    s_src[lane] = -1;
    __syncwarp();
    if (tgt >= 0) s_src[tgt] = lane;
    __syncwarp();
    const int src = s_src[lane];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      const double v = __shfl_sync(kAll, prod[e], src >= 0 ? src : lane);
      if (src >= 0) blk[e] -= v;
    }
    if (lane == kp) {
#pragma unroll
      for (int e = 0; e < 9; ++e) blk[e] = lik[e];
    }
  }
  if (lane == nl) mat3_inverse_or_diag(blk, a.dinv + size_t(i) * 9);
  if (own) {
#pragma unroll
    for (int e = 0; e < 9; ++e) a.lu[size_t(k) * 9 + e] = blk[e];
  }
  // pressure ILU0
  const double pv = own ? a.pval[k] : 0.0;
  const double pdg = lane < nl ? a.pdiag[ck] : 0.0;
  const unsigned pnz = __ballot_sync(kAll, own && pv != 0.0);
  double pl = 0.0;
  // s0 minus the terms of entry kk in list order (entries whose lp has a zero value skipped)
  auto terms = [&](int kk, double s0) {
    const int e0 = R.pt_ptr[kk], nt = R.pt_ptr[kk + 1] - e0;
    int lpl = lane;
    double ue = 0.0;
    if (lane < nt) {
      lpl = R.pt_lp[e0 + lane] - b0;
      ue = a.plu[R.pt_ue[e0 + lane]];
    }
    const double plp = __shfl_sync(kAll, pl, lpl);
    const bool valid = lane < nt && ((pnz >> lpl) & 1u);
    const double term = valid ? plp * ue : 0.0;
    double s = s0;
    for (int q = 0; q < nt; ++q) {
      const double tq = __shfl_sync(kAll, term, q);
      if (__shfl_sync(kAll, int(valid), q)) s -= tq;
    }
    return s;
  };
  for (int kp = 0; kp < nl; ++kp) {
    if (!((pnz >> kp) & 1u)) continue;  // plu stays 0
    const double s = terms(b0 + kp, __shfl_sync(kAll, pv, kp));
    const double d = __shfl_sync(kAll, pdg, kp);
    if (lane == kp) pl = fabs(d) > kEps ? s / d : 0.0;
  }
  {
    const double de = __shfl_sync(kAll, pv, nl);
    double ud = terms(dp, de);
    if (fabs(ud) <= kEps) ud = fabs(de) > kEps ? de : 1.0;
    if (lane == 0) a.pdiag[i] = ud;
  }
  // upper entries: each lane its own, reading the row's lower values from shared memory
  s_pl[lane] = pl;
  __syncwarp();
  if (own && lane > nl && pv != 0.0) {
    double s = pv;
    for (int e = R.pt_ptr[k]; e < R.pt_ptr[k + 1]; ++e) {
      const int lpl = R.pt_lp[e] - b0;
      if (!((pnz >> lpl) & 1u)) continue;
      s -= s_pl[lpl] * a.plu[R.pt_ue[e]];
    }
    pl = s;
  }
  if (own) a.plu[k] = lane == nl ? 0.0 : pl;
  __syncwarp();
}

// One factorisation on one thread-block cluster: each level's short rows spread over all CTAs'
// threads, the rows with a well's fill over their warps, one cluster barrier per level.
__global__ void __launch_bounds__(kFBlock, 1) k_factor_cluster(const __grid_constant__ FacArgs a) {
  __shared__ int s_ptr[kSmemLevels];
  __shared__ int s_src[kFBlock];
  __shared__ double s_pl[kFBlock];
  const LevelSched& L = a.L;
  const int* lp = stage_levels(L, s_ptr);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const int warp = tid >> 5, nwarps = nth >> 5, lw = threadIdx.x >> 5;
  for (int l = 0; l < L.n_levels; ++l) {
    for (int q = lp[l] + tid; q < lp[l + 1]; q += nth) {
      const int r = L.lvl_rows[q];
      if (L.rp[r + 1] - L.rp[r] > kLongRowBlocks) continue;  // a warp takes it below
      if (a.R.tri_ptr) {
        if (a.R.simple[r])
          ilu_row_simple(r, a);
        else
          ilu_row_recipe(r, a);
      } else {
        block_ilu_row(r, L.rp, L.col, L.diag, a.val, a.mask, a.lu, a.dinv);
        pressure_ilu_row(r, L.rp, L.col, L.diag, a.pval, a.plu, a.pdiag);
      }
    }
    __syncwarp();
    for (int q = L.long_ptr[l] + warp; q < L.long_ptr[l + 1]; q += nwarps) {
      const int r = L.long_rows[q];
      if (a.R.tri_ptr && L.rp[r + 1] - L.rp[r] <= 32)
        ilu_rows_lanes(r, a, s_src + 32 * lw, s_pl + 32 * lw);
      else
        ilu_rows_warp(r, L.rp, L.col, L.diag, a.val, a.mask, a.lu, a.dinv, a.pval, a.plu, a.pdiag);
    }
    cluster_barrier();
  }
}

// The same factorisation for many contexts in one launch (the ensemble's batched stepping, and
// the level-order path with one item): thread block b factors item b's matrices alone, level by
// level, with block barriers.  Every row gets the operations of k_factor_cluster, so the factors
// do not depend on the launch.
struct FacBatch {
  int count;
  FacArgs item[kBatchItems];
};
__global__ void __launch_bounds__(kFBlock, 1) k_factor_batch(const __grid_constant__ FacBatch b) {
  if (blockIdx.x >= unsigned(b.count)) return;  // uniform over the block
  const FacArgs& a = b.item[blockIdx.x];
  const LevelSched& L = a.L;
  __shared__ int s_ptr[kSmemLevels];
  const int* lp = stage_levels(L, s_ptr);
  __shared__ int s_src[kFBlock];
  __shared__ double s_pl[kFBlock];
  const int tid = threadIdx.x, nth = blockDim.x;
  const int warp = tid >> 5, nwarps = nth >> 5;
  for (int l = 0; l < L.n_levels; ++l) {
    for (int q = lp[l] + tid; q < lp[l + 1]; q += nth) {
      const int r = L.lvl_rows[q];
      if (L.rp[r + 1] - L.rp[r] > kLongRowBlocks) continue;  // a warp takes it below
      if (a.R.tri_ptr) {
        if (a.R.simple[r])
          ilu_row_simple(r, a);
        else
          ilu_row_recipe(r, a);
      } else {
        block_ilu_row(r, L.rp, L.col, L.diag, a.val, a.mask, a.lu, a.dinv);
        pressure_ilu_row(r, L.rp, L.col, L.diag, a.pval, a.plu, a.pdiag);
      }
    }
    __syncwarp();
    for (int q = L.long_ptr[l] + warp; q < L.long_ptr[l + 1]; q += nwarps) {
      const int r = L.long_rows[q];
      if (a.R.tri_ptr && L.rp[r + 1] - L.rp[r] <= 32)
        ilu_rows_lanes(r, a, s_src + 32 * warp, s_pl + 32 * warp);
      else
        ilu_rows_warp(r, L.rp, L.col, L.diag, a.val, a.mask, a.lu, a.dinv, a.pval, a.plu, a.pdiag);
    }
    __syncthreads();
  }
}
static_assert(sizeof(FacArgs) <= kBatchArgBytes, "factorisation arguments must fit a batch item");

bool launch_factor_batch(const BatchItem* const* items, int count, cudaStream_t stream) {
  FacBatch b;
  b.count = count;
  for (int i = 0; i < count; ++i) std::memcpy(&b.item[i], items[i]->args, sizeof(FacArgs));
  void* args[] = {&b};
  return cudaLaunchKernel((const void*)k_factor_batch, dim3(count), dim3(kFBlock), args, 0, stream) == cudaSuccess;
}

// ============================================================================================
// ILU sweeps
// ============================================================================================
// Storage type T of factors and work vectors: double for the FP64 path, float for the mixed form
// (FP32 block-ILU0 and pressure stage under the FP64 FGMRES).  Inputs and outputs at the FGMRES
// boundary stay double; row sums run in T.
//
// block: y_i = r_i - sum L_ik y_k (forward); x_i = Dinv_i (y_i - sum U_ij x_j) (backward)
template <class T>
__device__ __forceinline__ void block_fwd_row(int i, const int* rp, const int* col, const int* diag, const T* lu,
                                              const double* r, T* y) {
  T b0 = T(__ldcg(r + 3 * i)), b1 = T(__ldcg(r + 3 * i + 1)), b2 = T(__ldcg(r + 3 * i + 2));
  for (int k = rp[i]; k < diag[i]; ++k) {
    const T* Lb = lu + size_t(k) * 9;
    const int j = col[k];
    const T y0 = __ldcg(y + 3 * j), y1 = __ldcg(y + 3 * j + 1), y2 = __ldcg(y + 3 * j + 2);
    b0 -= Lb[0] * y0 + Lb[1] * y1 + Lb[2] * y2;
    b1 -= Lb[3] * y0 + Lb[4] * y1 + Lb[5] * y2;
    b2 -= Lb[6] * y0 + Lb[7] * y1 + Lb[8] * y2;
  }
  y[3 * i] = b0;
  y[3 * i + 1] = b1;
  y[3 * i + 2] = b2;
}
template <class T>
__device__ __forceinline__ void block_bwd_row(int i, const int* rp, const int* col, const int* diag, const T* lu,
                                              const T* dinv, const T* y, T* xt, double* x) {
  T b0 = __ldcg(y + 3 * i), b1 = __ldcg(y + 3 * i + 1), b2 = __ldcg(y + 3 * i + 2);
  for (int k = diag[i] + 1; k < rp[i + 1]; ++k) {
    const T* U = lu + size_t(k) * 9;
    const int j = col[k];
    const T x0 = __ldcg(xt + 3 * j), x1 = __ldcg(xt + 3 * j + 1), x2 = __ldcg(xt + 3 * j + 2);
    b0 -= U[0] * x0 + U[1] * x1 + U[2] * x2;
    b1 -= U[3] * x0 + U[4] * x1 + U[5] * x2;
    b2 -= U[6] * x0 + U[7] * x1 + U[8] * x2;
  }
  const T* D = dinv + size_t(i) * 9;
  const T o0 = D[0] * b0 + D[1] * b1 + D[2] * b2;
  const T o1 = D[3] * b0 + D[4] * b1 + D[5] * b2;
  const T o2 = D[6] * b0 + D[7] * b1 + D[8] * b2;
  xt[3 * i] = o0;
  xt[3 * i + 1] = o1;
  xt[3 * i + 2] = o2;
  if (x != nullptr && (const void*)x != (const void*)xt) {
    x[3 * i] = double(o0);
    x[3 * i + 1] = double(o1);
    x[3 * i + 2] = double(o2);
  }
}

// x = BlockILU(cr)   [one cluster: forward levels, then backward levels].  For T = double the
// backward sweep works in x itself (xt == x); for T = float it works in xt and writes x too.
template <class T>
__global__ void __launch_bounds__(kCBlock, 1) k_block_sweep_cluster(LevelSched L, const T* __restrict__ lu,
                                                                     const T* __restrict__ dinv,
                                                                     const double* __restrict__ cr, T* y, T* xt,
                                                                     double* x) {
  __shared__ int s_ptr[kSmemLevels];
  const int* lp = stage_levels(L, s_ptr);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int l = 0; l < L.n_levels; ++l) {
    for (int q = lp[l] + tid; q < lp[l + 1]; q += nth) block_fwd_row(L.lvl_rows[q], L.rp, L.col, L.diag, lu, cr, y);
    cluster_barrier();
  }
  for (int l = L.n_levels - 1; l >= 0; --l) {
    for (int q = lp[l] + tid; q < lp[l + 1]; q += nth)
      block_bwd_row(L.lvl_rows[q], L.rp, L.col, L.diag, lu, dinv, y, xt, x);
    if (l > 0) cluster_barrier();
  }
}

// scalar pressure ILU rows
template <class T>
__device__ __forceinline__ void p_fwd_row(int r, const int* rp, const int* col, const int* diag, const T* plu,
                                          const T* rhs, T* y) {
  T s = __ldcg(rhs + r);
  for (int k = rp[r]; k < diag[r]; ++k) s -= plu[k] * __ldcg(y + col[k]);
  y[r] = s;
}
template <class T>
__device__ __forceinline__ void p_bwd_row(int r, const int* rp, const int* col, const int* diag, const T* plu,
                                          const T* pdiag, const T* y, T* x) {
  T s = __ldcg(y + r);
  for (int k = diag[r] + 1; k < rp[r + 1]; ++k) s -= plu[k] * __ldcg(x + col[k]);
  const T d = pdiag[r];
  x[r] = fabs(double(d)) > kEps ? s / d : s;
}

// ============================================================================================
// BiCGStab on the pressure system (solve_pressure_with_bicgstab), one cluster
// ============================================================================================
template <class T>
struct BicgArgs {
  LevelSched L;
  int n;
  const T* pval;
  const T* plu;
  const T* pdiag;
  const double* rhs;
  double* x;
  T* r;
  T* rh;
  T* p;
  T* v;
  T* ph;
  T* s;
  T* sh;
  T* t;
  T* y;
  int max_iters;
  long long* iter_counter;  // incremented by the iterations this solve ran
};

// Cluster-wide sums of up to 4 per-thread values; every CTA ends with the same totals (each CTA
// adds the CTAs' partials in rank order from distributed shared memory, so the result is
// deterministic and identical everywhere).  The partials alternate between two slots (`parity`,
// advanced identically by every CTA): a CTA may run ahead into the next reduction and overwrite
// its own slot while a slower CTA is still reading this reduction's partials, but it cannot reach
// the reduction after that before the slower CTA has passed the barrier in between.
template <int BLOCK = kCBlock>
__device__ void cluster_sums(double* red /* shared [2][4] */, int& parity, int nq, const double* vals, double* out,
                             double* sh) {
  double* buf = red + (parity & 1) * 4;
  ++parity;
  for (int q = 0; q < nq; ++q) {
    const double r = block_sum<BLOCK>(vals[q], sh);
    if (threadIdx.x == 0) buf[q] = r;
  }
  cluster_barrier();
  __shared__ double tot[4];
  if (threadIdx.x < nq) {
    double a = 0.0;
    const unsigned nb = cluster_nblocks();
    const unsigned addr = static_cast<unsigned>(__cvta_generic_to_shared(buf + threadIdx.x));
    for (unsigned b = 0; b < nb; ++b) {
      unsigned remote;
      double v;
      asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(addr), "r"(b));
      asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(remote) : "memory");
      a += v;
    }
    tot[threadIdx.x] = a;
  }
  __syncthreads();
  for (int q = 0; q < nq; ++q) out[q] = tot[q];
  __syncthreads();
}

template <class T>
__device__ __forceinline__ void pressure_spmv(const LevelSched& L, const T* pval, const T* x, T* y, int n) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int r = tid; r < n; r += nth) {
    T s = T(0);
    for (int k = L.rp[r]; k < L.rp[r + 1]; ++k) s += pval[k] * __ldcg(x + L.col[k]);
    y[r] = s;
  }
}

// out = PressureILU(rhs): forward levels, backward levels, each level ended by a cluster barrier
// (the last one also publishes `out` to the SpMV that follows).
template <class T>
__device__ void pressure_ilu_apply(const BicgArgs<T>& a, const int* lp, const T* rhs, T* out) {
  const LevelSched& L = a.L;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int l = 0; l < L.n_levels; ++l) {
    for (int q = lp[l] + tid; q < lp[l + 1]; q += nth)
      p_fwd_row(L.lvl_rows[q], L.rp, L.col, L.diag, a.plu, rhs, a.y);
    cluster_barrier();
  }
  for (int l = L.n_levels - 1; l >= 0; --l) {
    for (int q = lp[l] + tid; q < lp[l + 1]; q += nth)
      p_bwd_row(L.lvl_rows[q], L.rp, L.col, L.diag, a.plu, a.pdiag, a.y, out);
    cluster_barrier();
  }
}

// The whole BiCGStab solve in one launch.  tol = max(|rhs|, EPS) * 1e-6 is formed from the first
// reduction (r0 = rhs - A*0 = rhs), as the reference forms it from the right-hand side.  Dot
// products accumulate in double and the iterate x is kept in double for either storage type.
template <class T>
__global__ void __launch_bounds__(kCBlock, 1) k_bicgstab_cluster(BicgArgs<T> a) {
  __shared__ double sh[32];
  __shared__ double red[8];
  __shared__ int s_ptr[kSmemLevels];
  const int* lp = stage_levels(a.L, s_ptr);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const int n = a.n;
  double v3[3], o3[3];
  int parity = 0;
  v3[0] = 0.0;
  for (int i = tid; i < n; i += nth) {
    const double ri = a.rhs[i] - 0.0;
    const T rt = T(ri);
    a.x[i] = 0.0;
    a.r[i] = rt;
    a.rh[i] = rt;
    a.v[i] = T(0);
    a.p[i] = T(0);
    v3[0] += double(rt) * double(rt);
  }
  cluster_sums(red, parity, 1, v3, o3, sh);
  const double rnorm0 = sqrt(o3[0]);
  const double tol = fmax(rnorm0, kEps) * 1e-6;
  const int max_iters = rnorm0 <= tol ? 0 : a.max_iters;
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  int started = 0;
  for (int it = 0; it < max_iters; ++it) {
    started = it + 1;
    v3[0] = 0.0;
    for (int i = tid; i < n; i += nth) v3[0] += double(a.rh[i]) * double(a.r[i]);
    cluster_sums(red, parity, 1, v3, o3, sh);
    const double rho = o3[0];
    if (!isfinite(rho) || fabs(rho) < kEps) break;
    if (it == 0) {
      for (int i = tid; i < n; i += nth) a.p[i] = a.r[i];
    } else {
      const double beta = (rho / rho_prev) * (alpha / omega);
      for (int i = tid; i < n; i += nth)
        a.p[i] = T(double(a.r[i]) + beta * (double(a.p[i]) - omega * double(a.v[i])));
    }
    cluster_barrier();
    pressure_ilu_apply(a, lp, a.p, a.ph);
    pressure_spmv(a.L, a.pval, a.ph, a.v, n);
    v3[0] = 0.0;
    for (int i = tid; i < n; i += nth) v3[0] += double(a.rh[i]) * double(a.v[i]);
    cluster_sums(red, parity, 1, v3, o3, sh);
    const double vd = o3[0];
    if (!isfinite(vd) || fabs(vd) < kEps) break;
    alpha = rho / vd;
    v3[0] = 0.0;
    for (int i = tid; i < n; i += nth) {
      const T si = T(double(a.r[i]) - alpha * double(a.v[i]));
      a.s[i] = si;
      v3[0] += double(si) * double(si);
    }
    cluster_sums(red, parity, 1, v3, o3, sh);
    if (sqrt(o3[0]) <= tol) {
      for (int i = tid; i < n; i += nth) a.x[i] += alpha * double(__ldcg(a.ph + i));
      break;
    }
    pressure_ilu_apply(a, lp, a.s, a.sh);
    pressure_spmv(a.L, a.pval, a.sh, a.t, n);
    v3[0] = 0.0;
    v3[1] = 0.0;
    for (int i = tid; i < n; i += nth) {
      const double ti = double(a.t[i]);
      v3[0] += ti * ti;
      v3[1] += ti * double(a.s[i]);
    }
    cluster_sums(red, parity, 2, v3, o3, sh);
    const double tt = o3[0];
    if (!isfinite(tt) || tt <= kEps) break;
    omega = o3[1] / tt;
    if (!isfinite(omega) || fabs(omega) < kEps) break;
    v3[0] = 0.0;
    for (int i = tid; i < n; i += nth) {
      a.x[i] += alpha * double(__ldcg(a.ph + i)) + omega * double(__ldcg(a.sh + i));
      const T ri = T(double(a.s[i]) - omega * double(a.t[i]));
      a.r[i] = ri;
      v3[0] += double(ri) * double(ri);
    }
    cluster_sums(red, parity, 1, v3, o3, sh);
    if (sqrt(o3[0]) <= tol) break;
    rho_prev = rho;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.iter_counter)
    atomicAdd((unsigned long long*)a.iter_counter, (unsigned long long)started);
  // no CTA may leave while another can still read its shared partials
  cluster_barrier();
}

// ============================================================================================
// BiCGStab with the vectors the level sweeps exchange held in distributed shared memory
// ============================================================================================
// Used when the pressure system fits the cluster's shared memory.  CTA b of the cluster owns the
// contiguous rows [b*S, b*S + S) ("slice"): it computes every row of its slice in every phase, so
// all vectors that are only read at a row's own index (r, rh, p, v, s, t, x) stay in global memory
// touched by one SM, and the three vectors read at neighbour indices (the forward-sweep result y
// and the sweep outputs ph and sh, which the SpMV reads next) live in the owners' shared memory.
// A neighbour in another slice is read through the cluster's distributed shared memory
// (mapa + ld.shared::cluster), so a level costs a cluster barrier plus one on-chip round trip
// instead of an L2 round trip after a release of global stores.  Within each slice the rows keep
// the level order, so every row still sees exactly the values the sequential sweep would.
constexpr int kDBlock = 256;

struct OwnedLevels {
  int slice;        // rows per CTA (the last CTA may own fewer)
  const int* rows;  // [n]: CTA b's rows in level order at [b*slice, b*slice + count_b)
  const int* ptr;   // [cs * (n_levels + 1)]: per-CTA level pointers, relative to b*slice
};

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned v;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(v));
  return v;
}
// Remote shared-memory loads.  They carry no "memory" clobber, so the compiler may overlap them
// with other loads; they stay ordered against the barriers and progress waits, which are volatile
// asm statements with a memory clobber.
__device__ __forceinline__ double dsm_load(const double* p, unsigned rank) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  unsigned r;
  double v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(r));
  return v;
}
__device__ __forceinline__ float dsm_load(const float* p, unsigned rank) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  unsigned r;
  float v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(r));
  return v;
}
// element `idx` of a slice-distributed vector whose local slice starts at `local`
template <class T>
__device__ __forceinline__ T slice_read(const T* local, int idx, int slice, unsigned me) {
  const unsigned owner = unsigned(idx / slice);
  const T* p = local + (idx - int(owner) * slice);
  return owner == me ? *p : dsm_load(p, owner);
}

// Level-ordered packed rows of each CTA's slice (index g = position in the ownership order,
// the same order as OwnedLevels::rows): for the forward (L) and backward (U) parts, the number of
// entries (-1 when more than kPackK: that row takes the CSR path), each entry's column as
// (owner CTA << 24) | index within the owner's slice, and the factor values in column order.
// The structure is fixed per pattern; the values are repacked after every factorisation.
constexpr int kPackK = 4;
template <class T>
struct PackedSweep {
  const int* cnt;  // [n]
  const int* dep;  // [kPackK][n]
  const T* val;    // [kPackK][n]
};

// sum -= plu[k] * src[col[k]] for k in [k0, k1), in k order, with the loads of each batch of
// eight entries issued together (rows of a well's clique have up to ~20 entries)
template <class T>
__device__ __noinline__ T csr_subtract(T sum, int k0, int k1, const int* col, const T* val, const T* src, int slice,
                                       unsigned me) {
  for (int k = k0; k < k1; k += 8) {
    T v[8], d[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (k + j < k1) {
        v[j] = val[k + j];
        d[j] = slice_read(src, col[k + j], slice, me);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (k + j < k1) sum -= v[j] * d[j];
  }
  return sum;
}
template <class T>
__device__ __forceinline__ T csr_dot(int k0, int k1, const int* col, const T* val, const T* src, int slice,
                                     unsigned me) {
  T s = T(0);
  for (int k = k0; k < k1; k += 8) {
    T v[8], d[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (k + j < k1) {
        v[j] = val[k + j];
        d[j] = slice_read(src, col[k + j], slice, me);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (k + j < k1) s += v[j] * d[j];
  }
  return s;
}

template <class T>
struct DsmBicgArgs {
  int n, n_levels;
  OwnedLevels own;
  const int* rp;
  const int* col;
  const int* diag;
  const T* pval;
  const T* plu;
  const T* pdiag;
  PackedSweep<T> fw, bw;
  const T* dval;  // [n] pivots in ownership order
  // [cs][L][cs]: progress (in positions) CTA b needs from CTA b' before a position, 0 = none
  const unsigned short* reqf;
  const unsigned short* reqb;
  const unsigned* cons_f;  // [cs]: bit j set when CTA j reads this CTA's rows in the forward sweep
  const unsigned* cons_b;  // [cs]: the same for the backward sweep
  int* status;
  const double* rhs;
  double* x;
  T* r;
  T* rh;
  T* p;
  T* v;
  T* s;
  T* t;
  int max_iters;
  long long* iter_counter;
};

__device__ __forceinline__ void cluster_arrive_release() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

template <class T>
__device__ __forceinline__ T dep_read(const T* slice_base, int dep, unsigned me) {
  const unsigned owner = unsigned(dep) >> 24;
  const T* p = slice_base + (dep & 0xffffff);
  return owner == me ? *p : dsm_load(p, owner);
}

// One row's packed data, loaded one level ahead.
template <class T>
struct PackedRow {
  int g, r, cnt;
  int dep[kPackK];
  T val[kPackK];
  T extra;  // forward: rhs[r]; backward: pivot
};

template <class T>
__device__ __forceinline__ void load_packed(PackedRow<T>& pr, const PackedSweep<T>& ps, int n, int g, int r,
                                            const T* extra_src, int extra_idx) {
  pr.g = g;
  pr.r = r;
  pr.cnt = ps.cnt[g];
#pragma unroll
  for (int j = 0; j < kPackK; ++j) {
    pr.dep[j] = ps.dep[size_t(j) * n + g];
    pr.val[j] = ps.val[size_t(j) * n + g];
  }
  pr.extra = extra_src[extra_idx];
}

// s - sum_j val_j * src[dep_j] over the row's entries in column order; the dependency loads are
// issued together, the subtractions keep the sequential order.
template <class T>
__device__ __forceinline__ T packed_subtract(T s, const PackedRow<T>& pr, const T* src, unsigned me) {
  T d[kPackK];
#pragma unroll
  for (int j = 0; j < kPackK; ++j) d[j] = j < pr.cnt ? dep_read(src, pr.dep[j], me) : T(0);
#pragma unroll
  for (int j = 0; j < kPackK; ++j)
    if (j < pr.cnt) s -= pr.val[j] * d[j];
  return s;
}

// Pipelined triangular sweeps on slices.  A CTA walks its own rows in level order ("positions":
// the levels for the forward sweep, the levels from the top for the backward one), separating
// its positions with __syncthreads only.  After each position it pushes how far it has got into
// an inbox word in the shared memory of each CTA that reads its rows (st.release.cluster to
// distributed shared memory); before a position it waits on its own inbox (ld.acquire.cluster on
// local shared memory) for the CTAs its rows read from, up to the position those rows need (a
// per-CTA table built with the schedule).  A CTA whose inputs are ready runs ahead instead of
// meeting every other CTA at a barrier each level, and the waits poll on-chip local memory.
// Progress values only grow within a launch: sweep number k counts from k * (L + 1).  Every wait
// is bounded; a wait that gives up sets the status word (2) and marks the CTA so it waits no more,
// which ends the launch with wrong values that the host then rejects.
constexpr long long kProgressPollLimit = 1ll << 24;

struct PipeSync {
  unsigned* inbox;        // [cs] in this CTA's shared memory: progress pushed by each producer
  volatile int* abort_s;  // shared: a wait of this CTA gave up
  int* status;            // global status word, read by the host after the solve
  unsigned epoch;         // progress value at the start of the current sweep
  unsigned level;         // positions processed so far in this launch (selects the barrier pair)
  unsigned cons_f, cons_b;  // CTAs that read this CTA's rows in the forward / backward sweep
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned read_inbox(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.cluster.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
  return v;
}

// Lane j of the signalling warp: push `value` into inbox[me] of consumer CTA j.  The compute
// warps' rows of the positions it covers were ordered before this store by the named barrier the
// signalling warp waited on.
__device__ __forceinline__ void push_progress(const PipeSync& ps, unsigned consumers, unsigned me, unsigned lane,
                                              unsigned value) {
  if ((consumers >> lane) & 1u) {
    unsigned addr;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(addr) : "r"(smem_u32(ps.inbox + me)), "r"(lane));
    asm volatile("st.release.cluster.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(value) : "memory");
  }
}

// Named barriers of the pipelined sweeps (0 is __syncthreads), used in two alternating pairs by
// the running count i of processed positions, so that no barrier instance can collect arrivals
// from two positions:
//   compute warps, position i: sync kBarCompute + (i & 1) (with the signalling warp's arrival),
//     handle the rows, arrive (no wait) on kBarSignal + (i & 1);
//   signalling warp, position i: sync kBarSignal + (i & 1), push the progress, arrive on
//     kBarCompute + (i & 1) -- the compute barrier of position i + 2.
// The signalling warp arrives on both compute barriers once at kernel start (for positions 0 and
// 1), and the compute warps sync on both once at kernel end, which leaves every instance complete.
constexpr int kBarCompute = 1;  // and 2
constexpr int kBarSignal = 3;   // and 4
__device__ __forceinline__ void named_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}
__device__ __forceinline__ void named_arrive(int id, int threads) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Warp 0 waits until every CTA that position `pos` of this CTA reads from has pushed the
// progress the table asks for; the other compute warps meet it at the named barrier that follows.
__device__ __forceinline__ void wait_inputs(PipeSync& ps, const unsigned short* req_s, int pos, int cs, unsigned me,
                                            int all_threads) {
  const int j = threadIdx.x;
  if (j < cs && j != int(me) && !*ps.abort_s) {
    const unsigned need = req_s[pos * cs + j];
    if (need != 0) {
      const unsigned target = ps.epoch + need;
      long long polls = 0;
      while (read_inbox(ps.inbox + j) < target) {
        if (++polls > kProgressPollLimit) {
          *ps.abort_s = 1;
          atomicExch(ps.status, 2);
          break;
        }
      }
    }
  }
  named_sync(kBarCompute + int(ps.level & 1u), all_threads);
}

// The last warp of the CTA only signals: it waits for the compute warps to finish each position
// and pushes the progress, so the release stores stay off the compute warps' path.  The compute
// warps (all but the last) handle the rows.
template <class T, bool FWD>
__device__ void pipe_sweep(const DsmBicgArgs<T>& a, const int* lrows, const int* lptr, const unsigned short* req_s,
                           int base, unsigned me, int cs, PipeSync& ps, const T* rhs, T* y_s, T* out_s) {
  const int S = a.own.slice, n = a.n, L = a.n_levels, t = threadIdx.x;
  const int B = blockDim.x - 32;  // compute threads
  const PackedSweep<T>& pk = FWD ? a.fw : a.bw;
  auto level_of = [&](int pos) { return FWD ? pos : L - 1 - pos; };
  auto empty = [&](int pos) {
    const int l = level_of(pos);
    return lptr[l] == lptr[l + 1];
  };
  auto prefetch = [&](PackedRow<T>& pr, int pos) {
    pr.cnt = -2;
    if (pos >= L) return;
    const int l = level_of(pos);
    const int q = lptr[l] + t;
    if (q < lptr[l + 1]) {
      if (FWD)
        load_packed(pr, pk, n, base + q, lrows[q], rhs, lrows[q]);
      else
        load_packed(pr, pk, n, base + q, lrows[q], a.dval, base + q);
    }
  };
  const unsigned consumers = FWD ? ps.cons_f : ps.cons_b;
  int pos = 0;
  while (pos < L && empty(pos)) ++pos;
  if (t >= B) {
    // signalling warp: the same sequence of positions as the compute warps
    const unsigned lane = unsigned(t - B);
    push_progress(ps, consumers, me, lane, ps.epoch + unsigned(pos));
    while (pos < L) {
      int next = pos + 1;
      while (next < L && empty(next)) ++next;
      named_sync(kBarSignal + int(ps.level & 1u), B + 32);
      push_progress(ps, consumers, me, lane, ps.epoch + unsigned(next));
      named_arrive(kBarCompute + int(ps.level & 1u), B + 32);
      ++ps.level;
      pos = next;
    }
    ps.epoch += unsigned(L) + 1u;
    return;
  }
  PackedRow<T> cur;
  prefetch(cur, pos);
  while (pos < L) {
    wait_inputs(ps, req_s, pos, cs, me, B + 32);
    const int l = level_of(pos);
    const int q0 = lptr[l] + t, qe = lptr[l + 1];
    if (q0 < qe) {
      const int r = cur.r;
      if (FWD) {
        if (cur.cnt >= 0) {
          y_s[r - base] = packed_subtract(cur.extra, cur, y_s, me);
        } else {
          y_s[r - base] = csr_subtract(cur.extra, a.rp[r], a.diag[r], a.col, a.plu, y_s, S, me);
        }
      } else {
        T sum = y_s[r - base];
        if (cur.cnt >= 0)
          sum = packed_subtract(sum, cur, out_s, me);
        else
          sum = csr_subtract(sum, a.diag[r] + 1, a.rp[r + 1], a.col, a.plu, out_s, S, me);
        const T d = cur.extra;
        out_s[r - base] = fabs(double(d)) > kEps ? sum / d : sum;
      }
    }
    for (int q = q0 + B; q < qe; q += B) {
      const int r = lrows[q];
      if (FWD) {
        y_s[r - base] = csr_subtract(rhs[r], a.rp[r], a.diag[r], a.col, a.plu, y_s, S, me);
      } else {
        const T sum = csr_subtract(y_s[r - base], a.diag[r] + 1, a.rp[r + 1], a.col, a.plu, out_s, S, me);
        const T d = a.pdiag[r];
        out_s[r - base] = fabs(double(d)) > kEps ? sum / d : sum;
      }
    }
    int next = pos + 1;
    while (next < L && empty(next)) ++next;
    named_arrive(kBarSignal + int(ps.level & 1u), B + 32);
    ++ps.level;
    prefetch(cur, next);
    pos = next;
  }
  ps.epoch += unsigned(L) + 1u;
}

// out = PressureILU(rhs) on slices: the pipelined forward sweep into y_s, the pipelined backward
// sweep into out_s, then one cluster barrier so the SpMV that follows sees all of out_s.
template <class T>
__device__ void dsm_ilu_apply(const DsmBicgArgs<T>& a, const int* lrows, const int* lptr,
                              const unsigned short* reqf_s, const unsigned short* reqb_s, int base, unsigned me,
                              int cs, PipeSync& ps, const T* rhs, T* y_s, T* out_s) {
  pipe_sweep<T, true>(a, lrows, lptr, reqf_s, base, me, cs, ps, rhs, y_s, out_s);
  pipe_sweep<T, false>(a, lrows, lptr, reqb_s, base, me, cs, ps, rhs, y_s, out_s);
  cluster_barrier();
}

// Values of the packed sweeps after a factorisation (ownership order, column order per row).
template <class T>
__global__ void k_pack_sweeps(int n, const int* __restrict__ own_rows, const int* __restrict__ rp,
                              const int* __restrict__ diag, const int* __restrict__ fcnt, const int* __restrict__ bcnt,
                              const double* __restrict__ plu, const double* __restrict__ pdiag, T* __restrict__ fval,
                              T* __restrict__ bval, T* __restrict__ dval) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const int r = own_rows[g];
  const int fc = fcnt[g], bc = bcnt[g];
#pragma unroll
  for (int j = 0; j < kPackK; ++j) {
    fval[size_t(j) * n + g] = j < fc ? T(plu[rp[r] + j]) : T(0);
    bval[size_t(j) * n + g] = j < bc ? T(plu[diag[r] + 1 + j]) : T(0);
  }
  dval[g] = T(pdiag[r]);
}

template <class T>
__device__ __forceinline__ void dsm_spmv(const DsmBicgArgs<T>& a, int base, int cnt, unsigned me, const T* in_s,
                                         T* out) {
  const int S = a.own.slice;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    const int r = base + i;
    out[r] = csr_dot(a.rp[r], a.rp[r + 1], a.col, a.pval, in_s, S, me);
  }
}

template <class T>
__global__ void __launch_bounds__(kDBlock, 1) k_bicgstab_dsmem(DsmBicgArgs<T> a) {
  extern __shared__ __align__(16) unsigned char dsm_raw[];
  __shared__ double sh[32];
  __shared__ double red[8];
  const int S = a.own.slice, n = a.n;
  T* y_s = reinterpret_cast<T*>(dsm_raw);
  T* ph_s = y_s + S;
  T* sh_s = ph_s + S;
  int* lrows = reinterpret_cast<int*>(sh_s + S);
  int* lptr = lrows + S;
  const int L = a.n_levels;
  const int cs = int(cluster_nblocks());
  unsigned short* reqf_s = reinterpret_cast<unsigned short*>(lptr + L + 1);
  unsigned short* reqb_s = reqf_s + size_t(L) * cs;
  __shared__ unsigned s_inbox[16];
  __shared__ int s_abort;
  const unsigned me = cluster_rank();
  const int base = int(me) * S;
  const int cnt = max(0, min(S, n - base));
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) lrows[i] = a.own.rows[base + i];
  for (int l = threadIdx.x; l <= L; l += blockDim.x) lptr[l] = a.own.ptr[size_t(me) * (L + 1) + l];
  for (int i = threadIdx.x; i < L * cs; i += blockDim.x) {
    reqf_s[i] = a.reqf[size_t(me) * L * cs + i];
    reqb_s[i] = a.reqb[size_t(me) * L * cs + i];
  }
  if (threadIdx.x < 16) s_inbox[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_abort = 0;
  PipeSync ps;
  ps.inbox = s_inbox;
  ps.abort_s = &s_abort;
  ps.status = a.status;
  ps.epoch = 0;
  ps.level = 0;
  ps.cons_f = a.cons_f[me];
  ps.cons_b = a.cons_b[me];
  if (threadIdx.x >= blockDim.x - 32) {  // signalling warp: release the compute barriers of positions 0 and 1
    named_arrive(kBarCompute, blockDim.x);
    named_arrive(kBarCompute + 1, blockDim.x);
  }
  double v3[3], o3[3];
  int parity = 0;
  v3[0] = 0.0;
  for (int i = base + threadIdx.x; i < base + cnt; i += blockDim.x) {
    const double ri = a.rhs[i] - 0.0;
    const T rt = T(ri);
    a.x[i] = 0.0;
    a.r[i] = rt;
    a.rh[i] = rt;
    a.v[i] = T(0);
    a.p[i] = T(0);
    v3[0] += double(rt) * double(rt);
  }
  cluster_sums<kDBlock>(red, parity, 1, v3, o3, sh);
  const double rnorm0 = sqrt(o3[0]);
  const double tol = fmax(rnorm0, kEps) * 1e-6;
  const int max_iters = rnorm0 <= tol ? 0 : a.max_iters;
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  int started = 0;
  for (int it = 0; it < max_iters; ++it) {
    started = it + 1;
    v3[0] = 0.0;
    for (int i = base + threadIdx.x; i < base + cnt; i += blockDim.x) v3[0] += double(a.rh[i]) * double(a.r[i]);
    cluster_sums<kDBlock>(red, parity, 1, v3, o3, sh);
    const double rho = o3[0];
    if (!isfinite(rho) || fabs(rho) < kEps) break;
    if (it == 0) {
      for (int i = base + threadIdx.x; i < base + cnt; i += blockDim.x) a.p[i] = a.r[i];
    } else {
      const double beta = (rho / rho_prev) * (alpha / omega);
      for (int i = base + threadIdx.x; i < base + cnt; i += blockDim.x)
        a.p[i] = T(double(a.r[i]) + beta * (double(a.p[i]) - omega * double(a.v[i])));
    }
    __syncthreads();
    dsm_ilu_apply(a, lrows, lptr, reqf_s, reqb_s, base, me, cs, ps, a.p, y_s, ph_s);
    dsm_spmv(a, base, cnt, me, ph_s, a.v);
    v3[0] = 0.0;
    for (int i = base + threadIdx.x; i < base + cnt; i += blockDim.x) v3[0] += double(a.rh[i]) * double(a.v[i]);
    cluster_sums<kDBlock>(red, parity, 1, v3, o3, sh);
    const double vd = o3[0];
    if (!isfinite(vd) || fabs(vd) < kEps) break;
    alpha = rho / vd;
    v3[0] = 0.0;
    for (int i = base + threadIdx.x; i < base + cnt; i += blockDim.x) {
      const T si = T(double(a.r[i]) - alpha * double(a.v[i]));
      a.s[i] = si;
      v3[0] += double(si) * double(si);
    }
    cluster_sums<kDBlock>(red, parity, 1, v3, o3, sh);
    if (sqrt(o3[0]) <= tol) {
      for (int i = threadIdx.x; i < cnt; i += blockDim.x) a.x[base + i] += alpha * double(ph_s[i]);
      break;
    }
    dsm_ilu_apply(a, lrows, lptr, reqf_s, reqb_s, base, me, cs, ps, a.s, y_s, sh_s);
    dsm_spmv(a, base, cnt, me, sh_s, a.t);
    v3[0] = 0.0;
    v3[1] = 0.0;
    for (int i = base + threadIdx.x; i < base + cnt; i += blockDim.x) {
      const double ti = double(a.t[i]);
      v3[0] += ti * ti;
      v3[1] += ti * double(a.s[i]);
    }
    cluster_sums<kDBlock>(red, parity, 2, v3, o3, sh);
    const double tt = o3[0];
    if (!isfinite(tt) || tt <= kEps) break;
    omega = o3[1] / tt;
    if (!isfinite(omega) || fabs(omega) < kEps) break;
    v3[0] = 0.0;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
      const int g = base + i;
      a.x[g] += alpha * double(ph_s[i]) + omega * double(sh_s[i]);
      const T ri = T(double(a.s[g]) - omega * double(a.t[g]));
      a.r[g] = ri;
      v3[0] += double(ri) * double(ri);
    }
    cluster_sums<kDBlock>(red, parity, 1, v3, o3, sh);
    if (sqrt(o3[0]) <= tol) break;
    rho_prev = rho;
  }
  if (me == 0 && threadIdx.x == 0 && a.iter_counter)
    atomicAdd((unsigned long long*)a.iter_counter, (unsigned long long)started);
  if (threadIdx.x < blockDim.x - 32) {  // complete the compute-barrier instances the signalling warp opened last
    named_sync(kBarCompute + int(ps.level & 1u), blockDim.x);
    named_sync(kBarCompute + int((ps.level + 1u) & 1u), blockDim.x);
  }
  // no CTA may leave while another can still read its shared memory
  cluster_barrier();
}

// FP32 copies of the factors and the pressure matrix for the mixed form (one pass over each).
__global__ void k_factors_to_f32(long long n_lu, const double* __restrict__ lu, float* __restrict__ lu32,
                                 long long n_dinv, const double* __restrict__ dinv, float* __restrict__ dinv32,
                                 long long nnzb, const double* __restrict__ plu, float* __restrict__ plu32,
                                 const double* __restrict__ pval, float* __restrict__ pval32, long long nb,
                                 const double* __restrict__ pdiag, float* __restrict__ pdiag32) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_lu; i += stride) lu32[i] = float(lu[i]);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_dinv; i += stride)
    dinv32[i] = float(dinv[i]);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nnzb; i += stride) {
    plu32[i] = float(plu[i]);
    pval32[i] = float(pval[i]);
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb; i += stride)
    pdiag32[i] = float(pdiag[i]);
}

// ============================================================================================
// CPR apply pieces
// ============================================================================================
__global__ void k_restrict(int nb, const double* __restrict__ w, const double* __restrict__ v, double* __restrict__ pr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  double s = 0.0;
  s += w[3 * i] * v[3 * i];
  s += w[3 * i + 1] * v[3 * i + 1];
  s += w[3 * i + 2] * v[3 * i + 2];
  pr[i] = s;
}
__global__ void k_prolong(int nb, const double* __restrict__ corr, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  out[3 * i] = 0.0 + 1.0 * corr[i];
  out[3 * i + 1] = 0.0;
  out[3 * i + 2] = 0.0;
}
__global__ void k_restrict_t(int nb, const double* __restrict__ v, double* __restrict__ pr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) pr[i] = v[3 * i];
}
__global__ void k_prolong_t(int nb, const double* __restrict__ w, const double* __restrict__ corr,
                            double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const double c = corr[i];
  out[3 * i] = w[3 * i] * c;
  out[3 * i + 1] = w[3 * i + 1] * c;
  out[3 * i + 2] = w[3 * i + 2] * c;
}
// y = a x for a dense row-major n x n matrix.  When `ok` is given and holds 0 (the inverse that
// produced `a` hit an exactly zero pivot), y is left untouched.
__global__ void k_dense_matvec(int n, const double* __restrict__ a, const double* __restrict__ x, double* __restrict__ y,
                               const int* __restrict__ ok) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || (ok != nullptr && *ok == 0)) return;
  double s = 0.0;
  for (int c = 0; c < n; ++c) s += a[size_t(r) * n + c] * x[c];
  y[r] = s;
}
// dense pressure matrix (N <= 299) from the block-pattern values
__global__ void k_dense_build(int nb, const int* __restrict__ rp, const int* __restrict__ col,
                              const double* __restrict__ pval, double* __restrict__ a) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nb) return;
  for (int c = 0; c < nb; ++c) a[size_t(r) * nb + c] = 0.0;
  for (int k = rp[r]; k < rp[r + 1]; ++k) a[size_t(r) * nb + col[k]] = pval[k];
}
// Dense inverse by LU with partial pivoting in nalgebra's operation order (linalg/lu.rs
// `try_invert_to` and `gauss_step`, linalg/solve.rs triangular solves).  Every step updates each
// element once, so spreading a step over threads keeps the sequential rounding: the first largest
// |pivot| of the column wins, multipliers are scaled by the pivot's reciprocal, updates are
// y = (-p) * c + y, the forward solve has a unit diagonal and the back substitution applies the
// columns from the last one down.  Two kernels:
//   k_dense_lu: one 1024-thread block factors `a` in place (row-major).  A warp owns a row of the
//     trailing matrix at each step, its lanes the columns; while updating, lane 0 of each warp
//     also tracks the largest |a_r,c+1| of its rows, so the next pivot is a reduction over 32
//     partials (value descending, row ascending: the sequential scan's first maximum) instead of
//     a pass over the column.  ok[0] = 0 when a pivot is exactly zero, else 1.
//   k_dense_inv_cols: thread block b solves for the 32 columns 32b.. of the inverse with them held
//     in shared memory (lane = column, warp = row), the factors read from global memory.
// `perm` holds n ints.
constexpr int kDenseColsPerBlock = 32;

__device__ __forceinline__ void piv_better(double v, int r, double& bv, int& br) {
  if (br < 0 || v > bv || (v == bv && r < br)) {
    bv = v;
    br = r;
  }
}

__global__ void __launch_bounds__(1024) k_dense_lu(int n, double* a, int* perm, int* ok) {
  __shared__ double s_val[32];
  __shared__ int s_row[32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = blockDim.x >> 5;
  for (int r = t; r < n; r += blockDim.x) perm[r] = r;
  // partial pivots of column 0
  {
    double bv = 0.0;
    int br = -1;
    for (int r = t; r < n; r += blockDim.x) piv_better(fabs(a[size_t(r) * n]), r, bv, br);
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, bv, o);
      const int orr = __shfl_down_sync(0xffffffffu, br, o);
      if (orr >= 0) piv_better(ov, orr, bv, br);
    }
    if (lane == 0) {
      s_val[warp] = bv;
      s_row[warp] = br;
    }
  }
  __syncthreads();
  for (int c = 0; c < n; ++c) {
    // every warp reduces the warps' partials (lane w takes warp w's) by the same butterfly and
    // takes lane 0's result: the same pivot everywhere.  piv_better is a total order (largest
    // value, then smallest row), so the order of the reduction does not change the pivot.
    double bv = 0.0;
    int piv = -1;
    if (lane < nwarps && s_row[lane] >= 0) {
      bv = s_val[lane];
      piv = s_row[lane];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int orr = __shfl_xor_sync(0xffffffffu, piv, o);
      if (orr >= 0) piv_better(ov, orr, bv, piv);
    }
    bv = __shfl_sync(0xffffffffu, bv, 0);
    piv = __shfl_sync(0xffffffffu, piv, 0);
    if (piv < 0 || bv == 0.0) {  // |a_piv,c| of the partials: an exactly zero pivot
      if (t == 0) ok[0] = 0;
      return;  // uniform: every thread saw the same partials
    }
    if (piv != c) {
      for (int k = t; k < n; k += blockDim.x) {
        const double x = a[size_t(c) * n + k];
        a[size_t(c) * n + k] = a[size_t(piv) * n + k];
        a[size_t(piv) * n + k] = x;
      }
      if (t == 0) {
        const int q = perm[c];
        perm[c] = perm[piv];
        perm[piv] = q;
      }
    }
    __syncthreads();  // swapped rows visible; every thread is done reading this step's partials
    const double inv_pivot = 1.0 / a[size_t(c) * n + c];
    double wv = 0.0;
    int wr = -1;
    for (int r = c + 1 + warp; r < n; r += nwarps) {
      double* row = a + size_t(r) * n;
      const double m = row[c] * inv_pivot;
      __syncwarp();
      if (lane == 0) row[c] = m;
      for (int k = c + 1 + lane; k < n; k += 32) {
        const double p = -a[size_t(c) * n + k];
        row[k] = p * m + row[k];
      }
      if (lane == 0 && c + 1 < n) piv_better(fabs(row[c + 1]), r, wv, wr);
    }
    if (lane == 0) {
      s_val[warp] = wv;
      s_row[warp] = wr;
    }
    __syncthreads();
  }
  if (t == 0) ok[0] = 1;
}

__global__ void __launch_bounds__(1024) k_dense_inv_cols(int n, const double* __restrict__ lu,
                                                         const int* __restrict__ perm, const int* __restrict__ ok,
                                                         double* __restrict__ inv) {
  extern __shared__ double X[];  // [n][32]
  if (*ok == 0) return;          // the factorisation failed: leave the inverse untouched
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int j = blockIdx.x * kDenseColsPerBlock + lane;
  const bool active = j < n;
  for (int r = warp; r < n; r += nwarps) X[r * 32 + lane] = (active && perm[r] == j) ? 1.0 : 0.0;
  __syncthreads();
  for (int i = 0; i + 1 < n; ++i) {  // unit-lower forward solve
    const double coeff = -X[i * 32 + lane];
    for (int r = i + 1 + warp; r < n; r += nwarps) X[r * 32 + lane] = coeff * lu[size_t(r) * n + i] + X[r * 32 + lane];
    __syncthreads();
  }
  for (int i = n - 1; i >= 0; --i) {  // back substitution, columns from the last one down
    if (warp == 0) X[i * 32 + lane] = X[i * 32 + lane] / lu[size_t(i) * n + i];
    __syncthreads();
    const double coeff = X[i * 32 + lane];
    for (int r = warp; r < i; r += nwarps) X[r * 32 + lane] = (-coeff) * lu[size_t(r) * n + i] + X[r * 32 + lane];
    __syncthreads();
  }
  if (active)
    for (int r = warp; r < n; r += nwarps) inv[size_t(r) * n + j] = X[r * 32 + lane];
}

void dense_invert_launch(int n, double* a, double* inv, int* perm, int* ok, cudaStream_t stream) {
  const size_t smem = sizeof(double) * size_t(n) * kDenseColsPerBlock;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute((const void*)k_dense_inv_cols, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(sizeof(double) * 299 * kDenseColsPerBlock));
  });
  k_dense_lu<<<1, 1024, 0, stream>>>(n, a, perm, ok);
  k_dense_inv_cols<<<(n + kDenseColsPerBlock - 1) / kDenseColsPerBlock, 1024, smem, stream>>>(n, a, perm, ok, inv);
}

// ============================================================================================
// host side
// ============================================================================================
static int reduce_blocks(Ctx& c, long long n) {
  long long b = (n + kBlock - 1) / kBlock;
  const long long cap = 4ll * c.num_sms;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return int(b);
}

static void dot_dev(Ctx& c, long long n, const double* a, const double* b, double* out, bool take_sqrt) {
  const int nb = reduce_blocks(c, n);
  k_dot_partial<<<nb, kBlock, 0, c.stream>>>(n, a, b, c.d_partials.p);
  k_reduce_to<<<1, 32, 0, c.stream>>>(nb, c.d_partials.p, out, take_sqrt ? 1 : 0);
  c.launches += 2;
}

static void spmv_res(Ctx& c, const double* x, const double* b, double* y) {
  k_spmv<1><<<blocks_for(c.n), kBlock, 0, c.stream>>>(c.n, c.d_row_ptr.p, c.d_col.p, c.d_val.p, x, b, y);
  c.launches++;
}
static void spmv(Ctx& c, const double* x, double* y) {
  k_spmv<0><<<blocks_for(c.n), kBlock, 0, c.stream>>>(c.n, c.d_row_ptr.p, c.d_col.p, c.d_val.p, x, nullptr, y);
  c.launches++;
}

static LevelSched level_sched(Ctx& c) {
  LevelSched L;
  L.n_levels = c.levels.n_levels;
  L.lvl_rows = c.levels.d_rows;
  L.lvl_ptr = c.levels.d_ptr;
  L.long_rows = c.levels.d_long_rows;
  L.long_ptr = c.levels.d_long_ptr;
  L.rp = c.d_row_ptr.p;
  L.col = c.d_col.p;
  L.diag = c.d_diag.p;
  return L;
}

// one cluster of c.cluster_size CTAs
static void cluster_launch(Ctx& c, const void* fn, int block, void** args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(c.cluster_size);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c.stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = c.cluster_size;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  RF_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
  c.launches++;
}

// CPR preconditioner build on the current reduced matrix
static void cpr_build(Ctx& c) {
  PhaseScope ps(c, kPhCprBuild);
  const int n = c.n;
  if (c.cpr_transposed) {
    k_cpr_weights_t<<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_row_ptr.p, c.d_diag.p, c.d_val.p, c.d_cpr_w.p,
                                                             c.d_bmask.p);
    k_pressure_matrix_t<<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_row_ptr.p, c.d_col.p, c.d_val.p, c.d_cpr_w.p,
                                                                 c.d_pval.p);
  } else {
    k_cpr_weights<<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_row_ptr.p, c.d_diag.p, c.d_val.p, c.d_cpr_w.p,
                                                           c.d_bmask.p);
    k_pressure_matrix<<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_row_ptr.p, c.d_val.p, c.d_cpr_w.p, c.d_pval.p);
  }
  c.launches += 2;
  LevelSched L = level_sched(c);
  const double* val = c.d_val.p;
  const unsigned char* mask = c.d_bmask.p;
  double* lu = c.d_lu.p;
  double* dinv = c.d_dinv.p;
  const double* pval = c.d_pval.p;
  double* plu = c.d_plu.p;
  double* pdiag = c.d_pdiag.p;
  FacRecipes rec{c.d_tri_ptr.p, c.d_tri_up.p, c.d_tri_ip.p, c.d_pt_ptr.p, c.d_pt_lp.p, c.d_pt_ue.p, c.d_fac_simple.p};
  const FacArgs fa{L, val, mask, lu, dinv, pval, plu, pdiag, rec};
  if (c.batched && fiber_file(kBatchFactor, 0, &fa, sizeof(fa), kFBlock, 0)) {
    // filed with the group's batched launch
  } else if (level_solver_active(c)) {
    // the level-order path: one thread block with the update lists
    FacBatch fb;
    fb.count = 1;
    fb.item[0] = fa;
    k_factor_batch<<<1, kFBlock, 0, c.stream>>>(fb);
    c.launches++;
  } else {
    void* args[] = {(void*)&fa};
    cluster_launch(c, (const void*)k_factor_cluster, kFBlock, args);
  }
  c.lvl.packed = -1;
  const bool level = level_solver_active(c);
  if (level) level_pack(c);
  if (!level && c.dsm_bytes[c.precision == 1 ? 1 : 0] != 0) {
    if (c.precision == 1)
      k_pack_sweeps<float><<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_own_rows.p, c.d_row_ptr.p, c.d_diag.p,
                                                                   c.d_fcnt.p, c.d_bcnt.p, c.d_plu.p, c.d_pdiag.p,
                                                                   c.d_fval32.p, c.d_bval32.p, c.d_dval32.p);
    else
      k_pack_sweeps<double><<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_own_rows.p, c.d_row_ptr.p, c.d_diag.p,
                                                                    c.d_fcnt.p, c.d_bcnt.p, c.d_plu.p, c.d_pdiag.p,
                                                                    c.d_fval.p, c.d_bval.p, c.d_dval.p);
    c.launches++;
  }
  if (c.precision == 1) {
    k_factors_to_f32<<<4 * c.num_sms, kBlock, 0, c.stream>>>(
        9ll * c.nnzb, c.d_lu.p, c.d_lu32.p, 9ll * n, c.d_dinv.p, c.d_dinv32.p, c.nnzb, c.d_plu.p, c.d_plu32.p,
        c.d_pval.p, c.d_pval32.p, n, c.d_pdiag.p, c.d_pdiag32.p);
    c.launches++;
  }
  c.dense_ok = 0;
  if (n <= 299) {
    k_dense_build<<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_row_ptr.p, c.d_col.p, c.d_pval.p, c.d_tmp2.p);
    dense_invert_launch(n, c.d_tmp2.p, c.d_dense.p, c.d_dense_perm.p, c.d_flag_dense.p, c.stream);
    c.launches += 2;
    int ok = 0;
    d2h(c, &ok, c.d_flag_dense.p, sizeof(int));
    d2h_wait(c);
    c.dense_ok = ok;
  }
}

template <class T>
static bool launch_bicgstab_dsmem(Ctx& c, const T* pval, const T* plu, const T* pdiag, const double* rhs, double* x,
                                  T* base) {
  const size_t bytes = c.dsm_bytes[sizeof(T) == 4 ? 1 : 0];
  if (bytes == 0) return false;
  const size_t n = c.n;
  DsmBicgArgs<T> a;
  a.n = c.n;
  a.n_levels = c.levels.n_levels;
  a.own.slice = c.own_slice;
  a.own.rows = c.d_own_rows.p;
  a.own.ptr = c.d_own_ptr.p;
  a.rp = c.d_row_ptr.p;
  a.col = c.d_col.p;
  a.diag = c.d_diag.p;
  a.pval = pval;
  a.plu = plu;
  a.pdiag = pdiag;
  a.reqf = c.d_reqf.p;
  a.reqb = c.d_reqb.p;
  a.cons_f = c.d_cons.p;
  a.cons_b = c.d_cons.p + c.cluster_size;
  a.status = c.d_pipe_status.p;
  a.fw.cnt = c.d_fcnt.p;
  a.fw.dep = c.d_fdep.p;
  a.bw.cnt = c.d_bcnt.p;
  a.bw.dep = c.d_bdep.p;
  if constexpr (sizeof(T) == 4) {
    a.fw.val = c.d_fval32.p;
    a.bw.val = c.d_bval32.p;
    a.dval = c.d_dval32.p;
  } else {
    a.fw.val = c.d_fval.p;
    a.bw.val = c.d_bval.p;
    a.dval = c.d_dval.p;
  }
  a.rhs = rhs;
  a.x = x;
  a.r = base;
  a.rh = base + n;
  a.p = base + 2 * n;
  a.v = base + 3 * n;
  a.s = base + 5 * n;
  a.t = base + 7 * n;
  a.max_iters = 50;
  a.iter_counter = c.d_bicg_iters;
  void* args[] = {&a};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(c.cluster_size);
  cfg.blockDim = dim3(kDBlock);
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = c.stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = c.cluster_size;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  RF_CUDA(cudaLaunchKernelExC(&cfg, (const void*)k_bicgstab_dsmem<T>, args));
  c.launches++;
  return true;
}

template <class T>
static void launch_bicgstab(Ctx& c, const T* pval, const T* plu, const T* pdiag, const double* rhs, double* x,
                            T* base) {
  if (level_solver_active(c)) {
    launch_bicgstab_level(c, rhs, x);
    return;
  }
  if (launch_bicgstab_dsmem<T>(c, pval, plu, pdiag, rhs, x, base)) return;
  const size_t n = c.n;
  BicgArgs<T> a;
  a.L = level_sched(c);
  a.n = c.n;
  a.pval = pval;
  a.plu = plu;
  a.pdiag = pdiag;
  a.rhs = rhs;
  a.x = x;
  a.r = base;
  a.rh = base + n;
  a.p = base + 2 * n;
  a.v = base + 3 * n;
  a.ph = base + 4 * n;
  a.s = base + 5 * n;
  a.sh = base + 6 * n;
  a.t = base + 7 * n;
  a.y = base + 8 * n;
  a.max_iters = 50;
  a.iter_counter = c.d_bicg_iters;
  void* args[] = {&a};
  cluster_launch(c, (const void*)k_bicgstab_cluster<T>, kCBlock, args);
}

// z = CPR(v)
static void cpr_apply(Ctx& c, const double* v, double* z) {
  const int n = c.n;
  double* prhs = c.d_pvec.p + size_t(10) * n;
  double* corr = c.d_pvec.p + size_t(11) * n;
  {
  PhaseScope ps(c, kPhCoarse);
  if (c.cpr_transposed)
    k_restrict_t<<<blocks_for(n), kBlock, 0, c.stream>>>(n, v, prhs);
  else
    k_restrict<<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_cpr_w.p, v, prhs);
  c.launches++;
  if (c.dense_ok) {
    k_dense_matvec<<<blocks_for(n, 64), 64, 0, c.stream>>>(n, c.d_dense.p, prhs, corr, nullptr);
    c.launches++;
  } else {
    PhaseScope pk(c, kPhBicgKernel);
    if (c.precision == 1)
      launch_bicgstab<float>(c, c.d_pval32.p, c.d_plu32.p, c.d_pdiag32.p, prhs, corr, c.d_pvec32.p);
    else
      launch_bicgstab<double>(c, c.d_pval.p, c.d_plu.p, c.d_pdiag.p, prhs, corr, c.d_pvec.p);
  }
  if (c.cpr_transposed)
    k_prolong_t<<<blocks_for(n), kBlock, 0, c.stream>>>(n, c.d_cpr_w.p, corr, z);
  else
    k_prolong<<<blocks_for(n), kBlock, 0, c.stream>>>(n, corr, z);
  c.launches++;
  }
  PhaseScope ps(c, kPhSmoother);
  // cr = v - A z_p ; sm = ILU(cr) ; z += sm
  double* cr = c.d_tmp.p;
  double* ysw = c.d_tmp2.p;
  spmv_res(c, z, v, cr);
  LevelSched L = level_sched(c);
  const double* crp = cr;
  double* xo = c.d_w.p;
  if (level_block_sweep_active(c)) {
    if (c.precision == 1)
      launch_block_sweep_level(c, crp, xo, c.d_lu32.p, c.d_dinv32.p);
    else
      launch_block_sweep_level(c, crp, xo, c.d_lu.p, c.d_dinv.p);
  } else if (c.precision == 1) {
    const float* lu = c.d_lu32.p;
    const float* dinv = c.d_dinv32.p;
    float* y32 = c.d_sweep32.p;
    float* x32 = c.d_sweep32.p + 3 * size_t(n);
    void* args[] = {&L, (void*)&lu, (void*)&dinv, (void*)&crp, &y32, &x32, &xo};
    cluster_launch(c, (const void*)k_block_sweep_cluster<float>, kCBlock, args);
  } else {
    const double* lu = c.d_lu.p;
    const double* dinv = c.d_dinv.p;
    void* args[] = {&L, (void*)&lu, (void*)&dinv, (void*)&crp, &ysw, &xo, &xo};
    cluster_launch(c, (const void*)k_block_sweep_cluster<double>, kCBlock, args);
  }
  k_add_inplace<<<reduce_blocks(c, 3ll * n), kBlock, 0, c.stream>>>(3ll * n, c.d_w.p, z);
  c.launches++;
}

static inline void givens(double a, double b, double& cs, double& sn) {
  const double rad = std::hypot(a, b);
  if (rad <= kEps) {
    cs = 1.0;
    sn = 0.0;
  } else {
    cs = a / rad;
    sn = b / rad;
  }
}

LinResult linear_solve_reduced(Ctx& c, bool rebuild) {
  LinResult out;
  const long long n3 = 3ll * c.n;
  const int R = Ctx::kRestart;
  double* V = c.d_V.p;
  double* Z = c.d_Z.p;
  double* b = c.d_rhs_red.p;
  double* hbuf = c.d_scal.p + 32;  // H column (R+2)
  if (rebuild) cpr_build(c);
  dot_dev(c, n3, b, nullptr, c.d_scal.p + 21, true);
  double rhs_norm = 0.0;
  d2h(c, &rhs_norm, c.d_scal.p + 21, sizeof(double));
  d2h_wait(c);
  out.rhs_norm = rhs_norm;
  const double tol = 1e-12 + 5e-3 * fmax(rhs_norm, kEps);
  // x0 = 0: r = b - A*0, computed explicitly as the reference does
  RF_CUDA(cudaMemsetAsync(c.d_x.p, 0, sizeof(double) * n3, c.stream));
  spmv_res(c, c.d_x.p, b, c.d_cres.p);
  dot_dev(c, n3, c.d_cres.p, nullptr, c.d_scal.p + 22, true);
  double rn = 0.0;
  d2h(c, &rn, c.d_scal.p + 22, sizeof(double));
  d2h_wait(c);
  if (rn <= tol) {
    out.converged = true;
    out.iterations = 0;
    out.final_residual_norm = rn;
    return out;
  }
  const double beta = rn;
  // V0 = r / beta
  k_scale_div<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, c.d_cres.p, c.d_scal.p + 22, V);
  c.launches++;
  std::vector<double> H((R + 1) * R, 0.0), cs(R, 0.0), sn(R, 0.0), g(R + 1, 0.0), hcol(R + 2);
  g[0] = beta;
  int iters = 0;
  for (int j = 0; j < R; ++j) {
    double* vj = V + size_t(j) * n3;
    double* zj = Z + size_t(j) * n3;
    double* w = c.d_cand.p;
    cpr_apply(c, vj, zj);
    PhaseScope ps(c, kPhKrylov);
    spmv(c, zj, w);
    for (int p = 0; p <= j; ++p) {
      double* vp = V + size_t(p) * n3;
      dot_dev(c, n3, vp, w, hbuf + p, false);
      k_axpy_dev<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, hbuf + p, vp, w);
      c.launches++;
    }
    dot_dev(c, n3, w, nullptr, hbuf + j + 1, true);
    d2h(c, hcol.data(), hbuf, sizeof(double) * (j + 2));
    d2h_wait(c);
    const double nn = hcol[j + 1];
    auto Hc = [&](int r, int cc) -> double& { return H[size_t(r) * R + cc]; };
    for (int p = 0; p <= j + 1; ++p) Hc(p, j) = hcol[p];
    if (nn > kEps && j + 1 <= R) {
      k_scale_div<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, w, hbuf + j + 1, V + size_t(j + 1) * n3);
      c.launches++;
    }
    for (int p = 0; p < j; ++p) {
      const double a = Hc(p, j), bb = Hc(p + 1, j);
      Hc(p, j) = cs[p] * a + sn[p] * bb;
      Hc(p + 1, j) = -sn[p] * a + cs[p] * bb;
    }
    double cc, ss;
    givens(Hc(j, j), Hc(j + 1, j), cc, ss);
    cs[j] = cc;
    sn[j] = ss;
    {
      const double a = Hc(j, j), bb = Hc(j + 1, j);
      Hc(j, j) = cc * a + ss * bb;
      Hc(j + 1, j) = -ss * a + cc * bb;
      const double g0 = g[j], g1 = g[j + 1];
      g[j] = cc * g0 + ss * g1;
      g[j + 1] = -ss * g0 + cc * g1;
    }
    ++iters;
    const int cols = j + 1;
    std::vector<double> y(cols, 0.0);
    for (int r = cols - 1; r >= 0; --r) {
      double sum = g[r];
      for (int k = r + 1; k < cols; ++k) sum -= Hc(r, k) * y[k];
      const double d = Hc(r, r);
      y[r] = std::fabs(d) > kEps ? sum / d : 0.0;
    }
    RF_CUDA(cudaMemcpyAsync(c.d_scal.p + 64, y.data(), sizeof(double) * cols, cudaMemcpyHostToDevice, c.stream));
    k_combine<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, cols, Z, n3, c.d_scal.p + 64, nullptr, c.d_x.p);
    spmv_res(c, c.d_x.p, b, c.d_cres.p);
    dot_dev(c, n3, c.d_cres.p, nullptr, c.d_scal.p + 23, true);
    c.launches++;
    double trn = 0.0;
    d2h(c, &trn, c.d_scal.p + 23, sizeof(double));
    d2h_wait(c);
    if (trn <= tol) {
      out.converged = true;
      out.iterations = iters;
      out.final_residual_norm = trn;
      break;
    }
    if (nn <= kEps || iters >= std::max(20, R)) {
      out.converged = false;
      out.iterations = iters;
      out.final_residual_norm = trn;
      break;
    }
  }
  RF_CUDA(cudaGetLastError());
  if (c.d_pipe_status.p) {
    int st = 0;
    d2h(c, &st, c.d_pipe_status.p, sizeof(int));
    d2h_wait(c);
    if (st != 0) throw CudaError("device status " + std::to_string(st) + ": a pressure-sweep wait gave up");
  }
  return out;
}

void schur_eliminate(Ctx& c) {
  const long long n3 = 3ll * c.n;
  // rhs_red = -res (cell rows); Schur corrects the perforated rows and adds the fill
  k_neg<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, c.d_res.p, c.d_rhs_red.p);
  c.launches++;
  const int W = c.topo.n_wells;
  if (W > 0) {
    PhaseScope ps(c, kPhSchur);
    SchurArgs s;
    s.n_wells = W;
    s.well_ptr = c.d_well_ptr.p;
    s.well_perfs = c.d_well_perfs.p;
    s.perf_cell = c.d_perf_cell.p;
    s.perf_has_wi = c.d_perf_has_wi.p;
    s.jrw = c.d_jrw.p;
    s.jwr_perf = c.d_jwr_perf.p;
    s.jwr_ctrl = c.d_jwr_ctrl.p;
    s.jww_perf_bhp = c.d_jww_perf_bhp.p;
    s.jww_ctrl_q = c.d_jww_ctrl_q.p;
    s.jww_ctrl_bhp = c.d_jww_ctrl_bhp.p;
    s.res = c.d_res.p;
    s.res_tail = c.d_res_tail.p;
    s.tinv_off = c.d_tinv_off.p;
    s.tinv = c.d_tinv.p;
    s.row_ptr = c.d_row_ptr.p;
    s.fill_off = c.d_fill_off.p;
    s.fill_pos = c.d_fill_pos.p;
    s.perf_row_off = c.d_perf_row_off.p;
    s.val = c.d_val.p;
    s.jrr_perf = c.d_jrr_perf.p;
    s.rhs_red = c.d_rhs_red.p;
    const int nt = 1 + c.topo.max_perfs_per_well;
    const size_t smem = sizeof(double) * (2 * size_t(nt) * nt + 2 * nt);
    k_schur<<<W, kBlock, smem, c.stream>>>(s);
    c.launches++;
  }
}

LinResult solve_reduced_accurate(Ctx& c, const double* b, double* x, double rtol, int max_passes,
                                 bool allow_direct) {
  // iterative refinement over the path's own inner solve (direct LU for small systems when
  // allowed, else CPR-FGMRES at its 5e-3 relative tolerance): x += solve(b - A x) until
  // |b - A x| <= rtol |b|
  const long long n3 = 3ll * c.n;
  LinResult out;
  dot_dev(c, n3, b, nullptr, c.d_scal.p + 26, true);
  double bn = 0.0;
  d2h(c, &bn, c.d_scal.p + 26, sizeof(double));
  d2h_wait(c);
  out.rhs_norm = bn;
  RF_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n3, c.stream));
  const bool direct = allow_direct && direct_rows(c, false) <= kDirectSolveRows;
  for (int pass = 0; pass <= max_passes; ++pass) {
    spmv_res(c, x, b, c.d_rhs_red.p);
    dot_dev(c, n3, c.d_rhs_red.p, nullptr, c.d_scal.p + 27, true);
    double rn = 0.0;
    d2h(c, &rn, c.d_scal.p + 27, sizeof(double));
    d2h_wait(c);
    out.final_residual_norm = rn;
    out.finite = std::isfinite(rn);
    if (!out.finite) return out;
    if (rn <= rtol * bn || bn == 0.0) {
      out.converged = true;
      return out;
    }
    if (pass == max_passes) break;
    LinResult inner;
    if (direct) inner = linear_solve_direct(c, false, nullptr);
    // the matrix is the same in every pass: the CPR factors of the first pass are reused
    if (!direct || !inner.converged) inner = linear_solve_reduced(c, pass == 0 || direct);
    out.iterations += inner.iterations;
    k_add_inplace<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, c.d_x.p, x);
    c.launches++;
  }
  return out;
}

LinResult linear_solve_full(Ctx& c, std::vector<double>& h_dx_tail) {
  // small systems go to the direct LU first; CPR-FGMRES runs when it does not converge
  // (fim/linear/mod.rs:279-300)
  bool fell_back = false;
  if (direct_rows(c, true) <= kDirectSolveRows) {
    LinResult d = linear_solve_direct(c, true, &h_dx_tail);
    if (d.converged) return d;
    fell_back = true;
  }
  const int n = c.n;
  const long long n3 = 3ll * n;
  schur_eliminate(c);
  const int W = c.topo.n_wells;
  LinResult lin;
  if (c.lin_refine_rtol > 0.0) {
    // refined solve (rf_set_linear_refinement): the reduced system's b and x kept aside while
    // the passes use the solver's own buffers; d_cres ends as the reduced residual of x
    const size_t bytes = sizeof(double) * size_t(n3);
    RF_CUDA(cudaMemcpyAsync(c.d_ref_b.p, c.d_rhs_red.p, bytes, cudaMemcpyDeviceToDevice, c.stream));
    lin = solve_reduced_accurate(c, c.d_ref_b.p, c.d_ref_x.p, c.lin_refine_rtol, c.lin_refine_passes, false);
    RF_CUDA(cudaMemcpyAsync(c.d_x.p, c.d_ref_x.p, bytes, cudaMemcpyDeviceToDevice, c.stream));
    RF_CUDA(cudaMemcpyAsync(c.d_rhs_red.p, c.d_ref_b.p, bytes, cudaMemcpyDeviceToDevice, c.stream));
    spmv_res(c, c.d_x.p, c.d_rhs_red.p, c.d_cres.p);
  } else {
    lin = linear_solve_reduced(c);
  }
  h_dx_tail.assign(size_t(W) + c.topo.n_perfs, 0.0);
  // full-system residual: reduced residual for unperforated rows, direct rows elsewhere
  k_copy<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, c.d_cres.p, c.d_full.p);
  c.launches++;
  double tail_sq_sum = 0.0;
  if (W > 0) {
    PhaseScope ps(c, kPhSchur);
    RecoverArgs r;
    r.n_wells = W;
    r.well_ptr = c.d_well_ptr.p;
    r.well_perfs = c.d_well_perfs.p;
    r.perf_cell = c.d_perf_cell.p;
    r.perf_has_wi = c.d_perf_has_wi.p;
    r.jrw = c.d_jrw.p;
    r.jwr_perf = c.d_jwr_perf.p;
    r.jwr_ctrl = c.d_jwr_ctrl.p;
    r.jww_perf_bhp = c.d_jww_perf_bhp.p;
    r.jww_ctrl_q = c.d_jww_ctrl_q.p;
    r.jww_ctrl_bhp = c.d_jww_ctrl_bhp.p;
    r.res = c.d_res.p;
    r.res_tail = c.d_res_tail.p;
    r.tinv_off = c.d_tinv_off.p;
    r.tinv = c.d_tinv.p;
    r.x = c.d_x.p;
    r.dx_tail = c.d_dx_tail.p;
    r.row_ptr = c.d_row_ptr.p;
    r.col = c.d_col.p;
    r.perf_row_off = c.d_perf_row_off.p;
    r.jrr_perf = c.d_jrr_perf.p;
    r.full = c.d_full.p;
    r.tail_sq = c.d_scal.p + 4096;
    k_recover<<<W, 32, 0, c.stream>>>(r);
    c.launches++;
    d2h(c, h_dx_tail.data(), c.d_dx_tail.p, sizeof(double) * h_dx_tail.size());
    std::vector<double> tsq(W);
    d2h(c, tsq.data(), c.d_scal.p + 4096, sizeof(double) * W);
    d2h_wait(c);
    for (double v : tsq) tail_sq_sum += v;
  }
  dot_dev(c, n3, c.d_full.p, nullptr, c.d_scal.p + 24, false);
  double sq = 0.0;
  d2h(c, &sq, c.d_scal.p + 24, sizeof(double));
  // rhs norm of the full system: |[-res; -res_tail]|
  dot_dev(c, n3, c.d_res.p, nullptr, c.d_scal.p + 25, false);
  double rsq = 0.0;
  d2h(c, &rsq, c.d_scal.p + 25, sizeof(double));
  std::vector<double> rt(size_t(W) + c.topo.n_perfs);
  if (!rt.empty())
    d2h(c, rt.data(), c.d_res_tail.p, sizeof(double) * rt.size());
  // finiteness of the solution
  RF_CUDA(cudaMemsetAsync(c.d_flag_dense.p + 1, 0, sizeof(int), c.stream));
  k_count_nonfinite<<<reduce_blocks(c, n3), kBlock, 0, c.stream>>>(n3, c.d_x.p, c.d_flag_dense.p + 1);
  c.launches++;
  int nonfinite = 0;
  d2h(c, &nonfinite, c.d_flag_dense.p + 1, sizeof(int));
  d2h_wait(c);
  for (double v : rt) rsq += v * v;
  for (double v : h_dx_tail)
    if (!std::isfinite(v)) nonfinite = 1;
  const double full_norm = std::sqrt(sq + tail_sq_sum);
  const double rhs_norm = std::sqrt(rsq);
  const double tol = 1e-12 + 5e-3 * fmax(rhs_norm, kEps);
  LinResult out;
  out.iterations = lin.iterations;
  out.rhs_norm = rhs_norm;
  out.final_residual_norm = full_norm;
  out.converged = lin.converged && full_norm <= tol;
  out.finite = nonfinite == 0;
  out.used_fallback = fell_back;
  return out;
}

// ---- one-time setup ----
// Update lists of the factorisation (FacRecipes) for the current pattern.
void build_factor_recipes(Ctx& c) {
  // RESSIM_FACTOR_RECIPES=0 (read when a context is set up) keeps the searching forms of the
  // factorisation instead; the two give identical factors, which the tests check through it
  const char* env = std::getenv("RESSIM_FACTOR_RECIPES");
  if (env && std::strcmp(env, "0") == 0) return;
  const int n = c.n, nnzb = c.nnzb;
  std::vector<int> tri_ptr(nnzb + 1, 0), tri_up, tri_ip, pt_ptr(nnzb + 1, 0), pt_lp, pt_ue;
  auto find_in_row_upper = [&](int row, int colj) -> int {
    const int lo = c.h_diag[row] + 1, hi = c.h_row_ptr[row + 1];
    auto b = c.h_col.begin() + lo, e = c.h_col.begin() + hi;
    auto it = std::lower_bound(b, e, colj);
    return (it != e && *it == colj) ? int(it - c.h_col.begin()) : -1;
  };
  for (int i = 0; i < n; ++i) {
    const int b0 = c.h_row_ptr[i], dp = c.h_diag[i], b1 = c.h_row_ptr[i + 1];
    for (int k = b0; k < b1; ++k) {
      if (k < dp) {  // block ILU: U-row of col[k] against row i's later entries
        const int kr = c.h_col[k];
        int ip = k + 1;
        for (int up = c.h_diag[kr] + 1; up < c.h_row_ptr[kr + 1]; ++up) {
          const int j = c.h_col[up];
          while (ip < b1 && c.h_col[ip] < j) ++ip;
          if (ip >= b1) break;
          if (c.h_col[ip] != j) continue;
          tri_up.push_back(up);
          tri_ip.push_back(ip);
        }
      }
      tri_ptr[k + 1] = int(tri_up.size());
      // pressure ILU: earlier lower entries lp whose row holds col[k] above its diagonal
      const int lp_end = k < dp ? k : dp;
      for (int lp = b0; lp < lp_end; ++lp) {
        const int ue = find_in_row_upper(c.h_col[lp], c.h_col[k]);
        if (ue < 0) continue;
        pt_lp.push_back(lp);
        pt_ue.push_back(ue);
      }
      pt_ptr[k + 1] = int(pt_lp.size());
    }
  }
  auto up = [](DBuf<int>& b, const std::vector<int>& h) {
    b.free();
    b.alloc(h.size());
    if (!h.empty()) RF_CUDA(cudaMemcpy(b.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
  };
  // rows of the simple shape (ilu_row_simple): few lower entries, each updating only the
  // diagonal, and pressure terms only on the diagonal
  std::vector<unsigned char> simple(n, 0);
  for (int i = 0; i < n; ++i) {
    const int b0 = c.h_row_ptr[i], dp = c.h_diag[i], b1 = c.h_row_ptr[i + 1];
    bool ok = dp - b0 <= 4 && b1 - b0 <= kLongRowBlocks;  // kSimpleLower
    for (int k = b0; ok && k < dp; ++k) {
      const int cnt = tri_ptr[k + 1] - tri_ptr[k];
      if (cnt > 1 || (cnt == 1 && tri_ip[tri_ptr[k]] != dp)) ok = false;
    }
    for (int k = b0; ok && k < b1; ++k)
      if (k != dp && pt_ptr[k + 1] != pt_ptr[k]) ok = false;
    simple[i] = ok ? 1 : 0;
  }
  c.d_fac_simple.free();
  c.d_fac_simple.alloc(size_t(n));
  RF_CUDA(cudaMemcpy(c.d_fac_simple.p, simple.data(), size_t(n), cudaMemcpyHostToDevice));
  up(c.d_tri_ptr, tri_ptr);
  up(c.d_tri_up, tri_up);
  up(c.d_tri_ip, tri_ip);
  up(c.d_pt_ptr, pt_ptr);
  up(c.d_pt_lp, pt_lp);
  up(c.d_pt_ue, pt_ue);
}

void build_levels(Ctx& c) {
  const int n = c.n;
  std::vector<int> lvl(n, 0);
  int maxl = 0;
  for (int i = 0; i < n; ++i) {
    int l = 0;
    for (int k = c.h_row_ptr[i]; k < c.h_diag[i]; ++k) l = std::max(l, lvl[c.h_col[k]] + 1);
    lvl[i] = l;
    maxl = std::max(maxl, l);
  }
  c.levels.n_levels = maxl + 1;
  c.levels.h_ptr.assign(c.levels.n_levels + 1, 0);
  for (int i = 0; i < n; ++i) c.levels.h_ptr[lvl[i] + 1]++;
  for (int l = 0; l < c.levels.n_levels; ++l) c.levels.h_ptr[l + 1] += c.levels.h_ptr[l];
  std::vector<int> rows(n), fillp(c.levels.h_ptr.begin(), c.levels.h_ptr.end() - 1);
  for (int i = 0; i < n; ++i) rows[fillp[lvl[i]]++] = i;
  c.levels.h_rows = rows;
  RF_CUDA(cudaMalloc(&c.levels.d_rows, sizeof(int) * n));
  RF_CUDA(cudaMalloc(&c.levels.d_ptr, sizeof(int) * (c.levels.n_levels + 1)));
  RF_CUDA(cudaMemcpy(c.levels.d_rows, rows.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.levels.d_ptr, c.levels.h_ptr.data(), sizeof(int) * (c.levels.n_levels + 1),
                     cudaMemcpyHostToDevice));
  std::vector<int> lptr(c.levels.n_levels + 1, 0), lrows;
  for (int l = 0; l < c.levels.n_levels; ++l) {
    for (int q = c.levels.h_ptr[l]; q < c.levels.h_ptr[l + 1]; ++q) {
      const int r = rows[q];
      if (c.h_row_ptr[r + 1] - c.h_row_ptr[r] > kLongRowBlocks) lrows.push_back(r);
    }
    lptr[l + 1] = int(lrows.size());
  }
  lrows.push_back(0);
  RF_CUDA(cudaMalloc(&c.levels.d_long_rows, sizeof(int) * lrows.size()));
  RF_CUDA(cudaMalloc(&c.levels.d_long_ptr, sizeof(int) * lptr.size()));
  RF_CUDA(cudaMemcpy(c.levels.d_long_rows, lrows.data(), sizeof(int) * lrows.size(), cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.levels.d_long_ptr, lptr.data(), sizeof(int) * lptr.size(), cudaMemcpyHostToDevice));
}

// Automatic cluster size: the smallest power of two (<= 16) whose slices fit the FP64
// distributed-shared-memory BiCGStab (three vectors, the row list and the level and progress
// tables per CTA) and that gives every row of the widest level its own thread in the
// global-memory kernels (1024 threads per CTA); 16 when no size fits.  Fewer CTAs per cluster
// leave more SMs to other work, which matters when many decks run at once.
int auto_cluster_size(const Ctx& c) {
  int widest = 1;
  for (int l = 0; l < c.levels.n_levels; ++l)
    widest = std::max(widest, c.levels.h_ptr[l + 1] - c.levels.h_ptr[l]);
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device) != cudaSuccess) optin = 0;
  const size_t budget = optin > 4096 ? size_t(optin) - 4096 : 0;  // static shared memory and slack
  const size_t L = size_t(c.levels.n_levels);
  for (int cs = 1; cs <= 16; cs *= 2) {
    const size_t S = (size_t(c.n) + cs - 1) / cs;
    const size_t bytes = 3 * S * sizeof(double) + sizeof(int) * (S + L + 1) + 2 * sizeof(unsigned short) * L * cs;
    if (bytes <= budget && cs * kCBlock >= widest) return cs;
  }
  return 16;
}

// Dynamic shared memory limits are attributes of a kernel, shared by every context in the process:
// only ever raise them, so a context created later with smaller needs cannot undercut an earlier
// one's launches.
void raise_dynamic_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  cudaFuncAttributes fa;
  RF_CUDA(cudaFuncGetAttributes(&fa, fn));
  if (size_t(fa.maxDynamicSharedSizeBytes) < bytes)
    RF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}

// Slice ownership for the distributed-shared-memory BiCGStab at the current cluster size: CTA b
// owns rows [b*S, b*S + S), listed in level order (ties in row order), with per-CTA level
// pointers.  Records, per value type, the dynamic shared memory the kernel needs, or 0 when the
// slices do not fit (the global-memory cluster kernel runs instead).
static void build_owned_levels(Ctx& c) {
  const int n = c.n, cs = c.cluster_size, L = c.levels.n_levels;
  const int S = (n + cs - 1) / cs;
  std::vector<int> lvl(n);
  for (int l = 0; l < L; ++l)
    for (int q = c.levels.h_ptr[l]; q < c.levels.h_ptr[l + 1]; ++q) lvl[c.levels.h_rows[q]] = l;
  std::vector<int> rows(n), ptr(size_t(cs) * (L + 1), 0);
  for (int b = 0; b < cs; ++b) {
    const int lo = b * S, hi = std::min(n, lo + S);
    int* bp = ptr.data() + size_t(b) * (L + 1);
    for (int r = lo; r < hi; ++r) bp[lvl[r] + 1]++;
    for (int l = 0; l < L; ++l) bp[l + 1] += bp[l];
    std::vector<int> fill(bp, bp + L);
    for (int r = lo; r < hi; ++r) rows[lo + fill[lvl[r]]++] = r;
  }
  // packed sweep structure: entry counts (-1 above kPackK) and (owner << 24 | local) columns
  std::vector<int> fcnt(n), bcnt(n), fdep(size_t(kPackK) * n, 0), bdep(size_t(kPackK) * n, 0);
  auto packdep = [&](int col) { return ((col / S) << 24) | (col - (col / S) * S); };
  for (int g = 0; g < n; ++g) {
    const int r = rows[g];
    const int lo = c.h_row_ptr[r], d = c.h_diag[r], hi = c.h_row_ptr[r + 1];
    fcnt[g] = d - lo <= kPackK ? d - lo : -1;
    bcnt[g] = hi - d - 1 <= kPackK ? hi - d - 1 : -1;
    for (int j = 0; j < kPackK; ++j) {
      if (j < fcnt[g]) fdep[size_t(j) * n + g] = packdep(c.h_col[lo + j]);
      if (j < bcnt[g]) bdep[size_t(j) * n + g] = packdep(c.h_col[d + 1 + j]);
    }
  }
  // progress tables of the pipelined sweeps: before position p (forward: level p; backward:
  // level L-1-p) CTA b needs, from each other CTA b', every position that holds a column its rows
  // at that level read, i.e. progress >= (forward) level(col) + 1 or (backward) L - level(col)
  std::vector<unsigned short> reqf(size_t(cs) * L * cs, 0), reqb(size_t(cs) * L * cs, 0);
  bool req_fits = L + 1 <= 65535;
  for (int r = 0; r < n && req_fits; ++r) {
    const int b = r / S, l = lvl[r];
    for (int k = c.h_row_ptr[r]; k < c.h_row_ptr[r + 1]; ++k) {
      const int col = c.h_col[k], ob = col / S;
      if (ob == b || col == r) continue;
      if (k < c.h_diag[r]) {
        unsigned short& q = reqf[(size_t(b) * L + l) * cs + ob];
        q = std::max<unsigned short>(q, static_cast<unsigned short>(lvl[col] + 1));
      } else {
        unsigned short& q = reqb[(size_t(b) * L + (L - 1 - l)) * cs + ob];
        q = std::max<unsigned short>(q, static_cast<unsigned short>(L - lvl[col]));
      }
    }
  }
  c.own_slice = S;
  for (auto* b : {&c.d_own_rows, &c.d_own_ptr, &c.d_fcnt, &c.d_bcnt, &c.d_fdep, &c.d_bdep}) b->free();
  // consumers of each CTA: the CTAs whose progress tables wait on it
  std::vector<unsigned> cons(2 * size_t(cs), 0u);
  for (int b = 0; b < cs; ++b)
    for (int p = 0; p < L; ++p)
      for (int ob = 0; ob < cs; ++ob) {
        if (reqf[(size_t(b) * L + p) * cs + ob]) cons[ob] |= 1u << b;
        if (reqb[(size_t(b) * L + p) * cs + ob]) cons[cs + ob] |= 1u << b;
      }
  c.d_cons.free();
  c.d_cons.alloc(cons.size());
  RF_CUDA(cudaMemcpy(c.d_cons.p, cons.data(), sizeof(unsigned) * cons.size(), cudaMemcpyHostToDevice));
  c.d_reqf.free();
  c.d_reqb.free();
  c.d_reqf.alloc(reqf.size());
  c.d_reqb.alloc(reqb.size());
  RF_CUDA(cudaMemcpy(c.d_reqf.p, reqf.data(), sizeof(unsigned short) * reqf.size(), cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.d_reqb.p, reqb.data(), sizeof(unsigned short) * reqb.size(), cudaMemcpyHostToDevice));
  if (c.d_pipe_status.p == nullptr) {
    c.d_pipe_status.alloc(1);
    RF_CUDA(cudaMemset(c.d_pipe_status.p, 0, sizeof(int)));
  }
  c.d_own_rows.alloc(n);
  c.d_own_ptr.alloc(ptr.size());
  c.d_fcnt.alloc(n);
  c.d_bcnt.alloc(n);
  c.d_fdep.alloc(size_t(kPackK) * n);
  c.d_bdep.alloc(size_t(kPackK) * n);
  RF_CUDA(cudaMemcpy(c.d_own_rows.p, rows.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.d_own_ptr.p, ptr.data(), sizeof(int) * ptr.size(), cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.d_fcnt.p, fcnt.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.d_bcnt.p, bcnt.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.d_fdep.p, fdep.data(), sizeof(int) * fdep.size(), cudaMemcpyHostToDevice));
  RF_CUDA(cudaMemcpy(c.d_bdep.p, bdep.data(), sizeof(int) * bdep.size(), cudaMemcpyHostToDevice));
  if (c.d_fval.p == nullptr) {
    c.d_fval.alloc(size_t(kPackK) * n);
    c.d_bval.alloc(size_t(kPackK) * n);
    c.d_dval.alloc(n);
  }
  if (c.precision == 1 && c.d_fval32.p == nullptr) {
    c.d_fval32.alloc(size_t(kPackK) * n);
    c.d_bval32.alloc(size_t(kPackK) * n);
    c.d_dval32.alloc(n);
  }
  int optin = 0;
  RF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
  const void* fns[2] = {(const void*)k_bicgstab_dsmem<double>, (const void*)k_bicgstab_dsmem<float>};
  const size_t tsz[2] = {sizeof(double), sizeof(float)};
  for (int f = 0; f < 2; ++f) {
    c.dsm_bytes[f] = 0;
    cudaFuncAttributes fa;
    RF_CUDA(cudaFuncGetAttributes(&fa, fns[f]));
    const size_t bytes = 3 * size_t(S) * tsz[f] + sizeof(int) * (size_t(S) + L + 1) +
                         2 * sizeof(unsigned short) * size_t(L) * cs;
    if (!req_fits || bytes + fa.sharedSizeBytes > size_t(optin)) continue;
    raise_dynamic_smem(fns[f], bytes);
    if (cs > 8) RF_CUDA(cudaFuncSetAttribute(fns[f], cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kDBlock);
    cfg.dynamicSmemBytes = bytes;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, fns[f], &cfg) == cudaSuccess && ncl >= 1) c.dsm_bytes[f] = bytes;
    cudaGetLastError();
  }
}

// The largest cluster size <= `want` (a power of two, 1..16) that every level-scheduled kernel
// can launch with (16 needs the non-portable cluster attribute).
int set_cluster_size(Ctx& c, int want) {
  const void* fns[5] = {(const void*)k_factor_cluster, (const void*)k_block_sweep_cluster<double>,
                        (const void*)k_bicgstab_cluster<double>, (const void*)k_block_sweep_cluster<float>,
                        (const void*)k_bicgstab_cluster<float>};
  const int blocks[5] = {kFBlock, kCBlock, kCBlock, kCBlock, kCBlock};
  for (int cs = 16; cs >= 1; cs /= 2) {
    if (cs > want) continue;
    bool ok = true;
    for (int f = 0; f < 5 && ok; ++f) {
      if (cs > 8) RF_CUDA(cudaFuncSetAttribute(fns[f], cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(cs);
      cfg.blockDim = dim3(blocks[f]);
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = cs;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      int nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, fns[f], &cfg) != cudaSuccess || nclusters < 1) ok = false;
    }
    cudaGetLastError();
    if (ok) {
      c.cluster_size = cs;
      build_owned_levels(c);
      return cs;
    }
  }
  throw CudaError("no thread-block cluster shape fits the level-scheduled kernels");
}

// FP32 factors and work vectors of the mixed form, allocated on first use.
void set_linear_precision(Ctx& c, int mode) {
  if (mode == 1 && c.d_fval32.p == nullptr) {
    const size_t n = c.n;
    c.d_fval32.alloc(size_t(kPackK) * n);
    c.d_bval32.alloc(size_t(kPackK) * n);
    c.d_dval32.alloc(n);
  }
  if (mode == 1 && c.d_lu32.p == nullptr) {
    const size_t n = c.n;
    c.d_lu32.alloc(size_t(c.nnzb) * 9);
    c.d_dinv32.alloc(n * 9);
    c.d_plu32.alloc(c.nnzb);
    c.d_pval32.alloc(c.nnzb);
    c.d_pdiag32.alloc(n);
    c.d_pvec32.alloc(10 * n);
    c.d_sweep32.alloc(6 * n);
  }
  c.precision = mode;
}

void setup_linear_workspace(Ctx& c) {
  const size_t n = c.n, n3 = 3 * n;
  const int R = Ctx::kRestart;
  c.d_V.alloc((R + 1) * n3);
  c.d_Z.alloc(R * n3);
  c.d_w.alloc(n3);
  c.d_x.alloc(n3);
  c.d_tmp.alloc(n3);
  c.d_tmp2.alloc(n <= 299 && n * n > n3 ? n * n : n3);  // also the dense pressure matrix when N <= 299
  c.d_cand.alloc(n3);
  c.d_cres.alloc(n3);
  c.d_full.alloc(n3);
  c.d_cpr_w.alloc(n3);
  c.d_pval.alloc(c.nnzb);
  c.d_plu.alloc(c.nnzb);
  c.d_pdiag.alloc(n);
  c.d_lu.alloc(size_t(c.nnzb) * 9);
  c.d_dinv.alloc(n * 9);
  c.d_bmask.alloc(c.nnzb);
  if (n <= 299) {
    c.d_dense.alloc(n * n);
    c.d_dense_perm.alloc(n);
  }
  c.d_pvec.alloc(12 * n);
  c.d_partials.alloc(4 * 4096);
  c.d_scal.alloc(8192);
  c.d_flag_dense.alloc(4);
  RF_CUDA(cudaMalloc(&c.d_bicg_iters, sizeof(long long)));
  RF_CUDA(cudaMemset(c.d_bicg_iters, 0, sizeof(long long)));
  // the largest cluster (16 CTAs, non-portable; else 8) that every level-scheduled kernel can run
  set_cluster_size(c, auto_cluster_size(c));
  build_level_plan(c);
  build_factor_recipes(c);
  const int nt = 1 + c.topo.max_perfs_per_well;
  const size_t smem = sizeof(double) * (2 * size_t(nt) * nt + 2 * nt);
  if (smem > 48 * 1024) raise_dynamic_smem((const void*)k_schur, smem);
}

}  // namespace rf
