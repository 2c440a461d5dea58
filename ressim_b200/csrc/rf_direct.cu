// rf_direct.cu — the direct route for small systems.
//
// The reference solves a full Newton system of at most 512 rows (3 unknowns per cell, one BHP per
// well, one rate per perforation) with a sparse direct LU instead of CPR-FGMRES
// (fim/linear/mod.rs:15, 56-67, 262-300; sparse_lu_debug.rs:148-232): one factorisation, one
// solve, then at most two refinement solves that are kept only while each cuts the residual below
// 95 % of the previous one; the solve counts as converged when |b - J x| <= 1e-12 + 5e-3 |b|.
// When it does not converge the iterative route runs instead.
//
// On the device the system is small enough to factor densely:
//   k_direct_build_*  scatter the assembled Jacobian (cell blocks, well rows and columns) into a
//                     dense column-major matrix and the right-hand side.
//   k_direct_lu       one thread-block cluster; the columns are dealt round-robin to the CTAs and
//                     stay in their shared memory (at 512 rows, 32 columns x 512 rows = 128 KB per
//                     CTA of a 16-CTA cluster).  At step k the owner of column k picks the pivot,
//                     forms the multipliers and stores them into every CTA's shared memory; after
//                     one cluster barrier each CTA swaps the two rows and updates its own columns.
//                     Partial pivoting takes the first largest |a_ik|; an exactly zero pivot
//                     column is a failed factorisation.
//   k_direct_solve    one CTA: x = U^-1 L^-1 P b column by column, factor columns read from L2
//                     eight steps ahead.
//   k_direct_residual one CTA: r = b - A x and |r|, summed left to right.
// Every element is updated in the same order, with the same operations and skip rules, as the
// oracle's dense restatement, so both produce the same factors and solutions bit for bit.
#include <cmath>
#include <vector>

#include "rf_ops.hpp"

namespace rf {

namespace {

constexpr int kDirThreads = 512;

__device__ __forceinline__ unsigned dir_cta_rank() {
  unsigned v;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(v));
  return v;
}
__device__ __forceinline__ void dir_cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned dir_remote(const void* local, unsigned rank) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(local));
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void dir_store_remote(unsigned addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
__device__ __forceinline__ void dir_store_remote(unsigned addr, int v) {
  asm volatile("st.shared::cluster.s32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// Dense column-major A (n x n) and b from the cell blocks of the block pattern: one thread per
// cell row.  Unset entries were zeroed by the caller.
__global__ void k_direct_build_cells(int n_cells, int nf, const int* __restrict__ rp, const int* __restrict__ col,
                                     const double* __restrict__ val, const double* __restrict__ rhs_cells,
                                     double rhs_sign, double* __restrict__ a, double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_cells) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = col[k];
    for (int r = 0; r < 3; ++r)
      for (int v = 0; v < 3; ++v) a[size_t(3 * j + v) * nf + 3 * i + r] = 0.0 + val[size_t(k) * 9 + 3 * r + v];
  }
  for (int r = 0; r < 3; ++r) b[3 * i + r] = rhs_sign * rhs_cells[3 * i + r];
}

// The well tail: one thread per physical well writes its control row and the rows and columns of
// its perforations (unknowns ordered cells, BHP per well, rate per perforation).
__global__ void k_direct_build_wells(int n_cells, int n_wells, int nf, const int* __restrict__ well_ptr,
                                     const int* __restrict__ well_perfs, const int* __restrict__ perf_cell,
                                     const int* __restrict__ perf_has_wi, const double* __restrict__ jrw,
                                     const double* __restrict__ jwr_perf, const double* __restrict__ jwr_ctrl,
                                     const double* __restrict__ jww_perf_bhp, const double* __restrict__ jww_ctrl_q,
                                     const double* __restrict__ jww_ctrl_bhp, const double* __restrict__ res_tail,
                                     double* __restrict__ a, double* __restrict__ b) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_wells) return;
  const int n3 = 3 * n_cells, wrow = n3 + w;
  a[size_t(wrow) * nf + wrow] = 0.0 + jww_ctrl_bhp[w];
  b[wrow] = -res_tail[w];
  for (int e = well_ptr[w]; e < well_ptr[w + 1]; ++e) {
    const int k = well_perfs[e], cell = perf_cell[k], q = n3 + n_wells + k;
    for (int r = 0; r < 3; ++r) a[size_t(q) * nf + 3 * cell + r] = 0.0 + jrw[3 * k + r];
    a[size_t(q) * nf + wrow] = 0.0 + jww_ctrl_q[k];
    for (int v = 0; v < 3; ++v) {
      double& x = a[size_t(3 * cell + v) * nf + wrow];
      x = x + jwr_ctrl[3 * k + v];
    }
    a[size_t(wrow) * nf + q] = 0.0 + jww_perf_bhp[k];
    a[size_t(q) * nf + q] = perf_has_wi[k] ? 1.0 : 0.0;
    for (int v = 0; v < 3; ++v) a[size_t(3 * cell + v) * nf + q] = 0.0 + jwr_perf[3 * k + v];
    b[q] = -res_tail[n_wells + k];
  }
}

// LU with partial pivoting, P A = L U, on one cluster of gridDim.x CTAs.  CTA `me` owns the
// columns j with j % cs == me, in local slot j / cs, column-major in dynamic shared memory.
// Writes the factors column-major to `lu`, the row permutation to `perm` and status[0] = 1 when
// every pivot was nonzero (0 otherwise).
__global__ void __launch_bounds__(kDirThreads) k_direct_lu(int n, const double* __restrict__ a_in,
                                                            double* __restrict__ lu, int* __restrict__ perm,
                                                            int* __restrict__ status) {
  extern __shared__ double dsm[];
  __shared__ int s_piv[2];
  __shared__ int s_perm[kDirectSolveRows];
  __shared__ double s_best[kDirThreads / 32];
  __shared__ int s_arg[kDirThreads / 32];
  const int cs = gridDim.x, t = threadIdx.x, nt = blockDim.x, lane = t & 31, warp = t >> 5;
  const int me = int(dir_cta_rank());
  const int ncl = (n + cs - 1) / cs;
  const int cnt = (n - me + cs - 1) / cs;  // local columns that exist
  double* A = dsm;                // [ncl][n]
  double* lbuf = dsm + size_t(ncl) * n;  // [2][n] multipliers of the current step
  for (int idx = t; idx < ncl * n; idx += nt) {
    const int s = idx / n, i = idx % n, j = s * cs + me;
    A[idx] = j < n ? a_in[size_t(j) * n + i] : 0.0;
  }
  if (me == 0)
    for (int i = t; i < n; i += nt) s_perm[i] = i;
  // every CTA of the cluster is running before any remote store
  dir_cluster_sync();
  for (int k = 0; k < n; ++k) {
    const int owner = k % cs, par = k & 1;
    if (me == owner) {
      const double* colk = A + size_t(k / cs) * n;
      // first largest |a_ik| over i >= k: strictly larger replaces, ties keep the smaller row
      double best = -1.0;
      int arg = -1;
      for (int i = k + t; i < n; i += nt) {
        const double v = fabs(colk[i]);
        if (arg < 0 || v > best) {
          best = v;
          arg = i;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oa = __shfl_down_sync(0xffffffffu, arg, o);
        if (oa >= 0 && (arg < 0 || ob > best || (ob == best && oa < arg))) {
          best = ob;
          arg = oa;
        }
      }
      if (lane == 0) {
        s_best[warp] = best;
        s_arg[warp] = arg;
      }
      __syncthreads();
      if (t == 0) {
        double bb = -1.0;
        int ba = -1;
        for (int q = 0; q < nt / 32; ++q) {
          const int oa = s_arg[q];
          const double ob = s_best[q];
          if (oa >= 0 && (ba < 0 || ob > bb || (ob == bb && oa < ba))) {
            bb = ob;
            ba = oa;
          }
        }
        // a NaN never compares larger, so an all-NaN or all-zero column fails here
        s_arg[0] = (ba >= 0 && fabs(colk[ba]) > 0.0) ? ba : -1;
      }
      __syncthreads();
      const int p = s_arg[0];
      if (p >= 0) {
        const double piv = colk[p];
        for (int i = k + 1 + t; i < n; i += nt) {
          const double v = (i == p) ? colk[k] : colk[i];
          const double l = v / piv;
          for (int r = 0; r < cs; ++r) dir_store_remote(dir_remote(lbuf + size_t(par) * n + i, r), l);
        }
      }
      if (t < cs) dir_store_remote(dir_remote(s_piv + par, t), p);
    }
    dir_cluster_sync();
    const int p = s_piv[par];
    if (p < 0) {
      if (me == 0 && t == 0) status[0] = 0;
      return;  // every CTA returns here, after the last remote store
    }
    if (p != k) {
      for (int s = t; s < cnt; s += nt) {
        double* c = A + size_t(s) * n;
        const double x = c[k];
        c[k] = c[p];
        c[p] = x;
      }
      if (me == 0 && t == 0) {
        const int q = s_perm[k];
        s_perm[k] = s_perm[p];
        s_perm[p] = q;
      }
    }
    __syncthreads();
    const double* l = lbuf + size_t(par) * n;
    if (me == owner) {
      double* colk = A + size_t(k / cs) * n;
      for (int i = k + 1 + t; i < n; i += nt) colk[i] = l[i];
    }
    // rank-1 update of the local columns j > k
    const int s0 = k >= me ? (k - me) / cs + 1 : 0;
    const int m = n - k - 1;
    if (m > 0 && s0 < cnt) {
      const int total = (cnt - s0) * m;
      for (int idx = t; idx < total; idx += nt) {
        const int s = s0 + idx / m, i = k + 1 + idx % m;
        double* c = A + size_t(s) * n;
        const double u = c[k];
        if (u == 0.0) continue;
        const double li = l[i];
        if (li != 0.0) c[i] = c[i] - li * u;
      }
    }
    __syncthreads();
  }
  for (int idx = t; idx < cnt * n; idx += nt) {
    const int s = idx / n, i = idx % n, j = s * cs + me;
    lu[size_t(j) * n + i] = A[idx];
  }
  if (me == 0) {
    for (int i = t; i < n; i += nt) perm[i] = s_perm[i];
    if (t == 0) status[0] = 1;
  }
}

// x = U^-1 L^-1 P b on one CTA of kDirThreads threads (thread i owns row i).  The factor column of
// the next eight steps is already in flight while a step runs.  flag[0] is set when x has a
// non-finite entry.
__global__ void __launch_bounds__(kDirThreads) k_direct_solve(int n, const double* __restrict__ lu,
                                                               const int* __restrict__ perm,
                                                               const double* __restrict__ b, double* __restrict__ x,
                                                               int* __restrict__ flag) {
  __shared__ double y[kDirectSolveRows];
  const int t = threadIdx.x;
  const bool row = t < n;
  if (row) y[t] = b[perm[t]];
  constexpr int D = 8;
  double ring[D];
#pragma unroll
  for (int d = 0; d < D; ++d) ring[d] = (row && d < n) ? lu[size_t(d) * n + t] : 0.0;
  __syncthreads();
  // forward: unit lower, columns in increasing order
  for (int k0 = 0; k0 < n; k0 += D) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const int k = k0 + d;
      if (k < n) {
        const double lk = ring[d];
        const int kn = k + D;
        ring[d] = (row && kn < n) ? lu[size_t(kn) * n + t] : 0.0;
        const double yk = y[k];
        if (yk != 0.0 && row && t > k) y[t] = y[t] - lk * yk;
      }
      __syncthreads();
    }
  }
  // backward: upper, columns in decreasing order
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int k = n - 1 - d;
    ring[d] = (row && k >= 0) ? lu[size_t(k) * n + t] : 0.0;
  }
  for (int k0 = n - 1; k0 >= 0; k0 -= D) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const int k = k0 - d;
      if (k >= 0) {
        const double uk = ring[d];
        const int kn = k - D;
        ring[d] = (row && kn >= 0) ? lu[size_t(kn) * n + t] : 0.0;
        // thread k holds the diagonal of column k
        if (t == k) y[k] = y[k] / uk;
        __syncthreads();
        const double xk = y[k];
        if (xk != 0.0 && row && t < k) y[t] = y[t] - uk * xk;
      }
      __syncthreads();
    }
  }
  if (row) {
    x[t] = y[t];
    if (!isfinite(y[t])) atomicOr(flag, 1);
  }
}

// r = b - A (x + c) when c != nullptr (the candidate is also written to `cand`), else r = b - A x;
// out[0] = |r| (squares summed left to right), out[1] = |b| likewise.
__global__ void __launch_bounds__(kDirThreads) k_direct_residual(int n, const double* __restrict__ a,
                                                                  const double* __restrict__ b,
                                                                  const double* __restrict__ x,
                                                                  const double* __restrict__ c,
                                                                  double* __restrict__ cand,
                                                                  double* __restrict__ r, double* __restrict__ out) {
  __shared__ double xs[kDirectSolveRows];
  __shared__ double rs[kDirectSolveRows];
  const int t = threadIdx.x;
  if (t < n) {
    const double v = c ? x[t] + c[t] : x[t];
    xs[t] = v;
    if (c) cand[t] = v;
  }
  __syncthreads();
  if (t < n) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) {
      const double aij = a[size_t(j) * n + t];
      if (aij != 0.0) s += aij * xs[j];
    }
    rs[t] = b[t] - s;
    r[t] = rs[t];
  }
  __syncthreads();
  if (t == 0) {
    double s = 0.0, sb = 0.0;
    for (int i = 0; i < n; ++i) {
      s += rs[i] * rs[i];
      sb += b[i] * b[i];
    }
    out[0] = sqrt(s);
    out[1] = sqrt(sb);
  }
}

}  // namespace

int direct_rows(const Ctx& c, bool with_wells) {
  return 3 * c.n + (with_wells ? c.topo.n_wells + c.topo.n_perfs : 0);
}

static void ensure_direct_workspace(Ctx& c, int nf) {
  if (c.dir_rows >= nf) return;
  const size_t n2 = size_t(nf) * nf;
  c.d_dir_a.free();
  c.d_dir_lu.free();
  c.d_dir_vec.free();
  c.d_dir_perm.free();
  c.d_dir_a.alloc(n2);
  c.d_dir_lu.alloc(n2);
  c.d_dir_vec.alloc(6 * size_t(nf) + 8);  // b, x, r, correction, candidate, candidate residual, scalars
  c.d_dir_perm.alloc(size_t(nf) + 4);
  c.dir_rows = nf;
  // cluster shape: the smallest power of two (<= 16) whose column slices fit shared memory
  int optin = 0;
  RF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
  cudaFuncAttributes fa;
  RF_CUDA(cudaFuncGetAttributes(&fa, (const void*)k_direct_lu));
  c.dir_cs = 0;
  for (int cs = 1; cs <= 16; cs *= 2) {
    const int ncl = (nf + cs - 1) / cs;
    const size_t bytes = sizeof(double) * (size_t(ncl) * nf + 2 * size_t(nf));
    if (bytes + fa.sharedSizeBytes > size_t(optin)) continue;
    if (bytes > 48 * 1024)
      RF_CUDA(cudaFuncSetAttribute((const void*)k_direct_lu, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(bytes)));
    if (cs > 8) RF_CUDA(cudaFuncSetAttribute((const void*)k_direct_lu, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kDirThreads);
    cfg.dynamicSmemBytes = bytes;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl_active = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl_active, (const void*)k_direct_lu, &cfg) == cudaSuccess && ncl_active >= 1) {
      c.dir_cs = cs;
      c.dir_smem = bytes;
      break;
    }
  }
  cudaGetLastError();
  if (c.dir_cs == 0) throw CudaError("no thread-block cluster shape fits the direct LU of " + std::to_string(nf) + " rows");
}

LinResult linear_solve_direct(Ctx& c, bool with_wells, std::vector<double>* h_dx_tail) {
  PhaseScope ps(c, kPhDirect);
  const int nf = direct_rows(c, with_wells);
  const int n = c.n, n3 = 3 * n;
  ensure_direct_workspace(c, nf);
  double* A = c.d_dir_a.p;
  double* LU = c.d_dir_lu.p;
  double* b = c.d_dir_vec.p;
  double* x = b + nf;
  double* r = x + nf;
  double* cor = r + nf;
  double* cand = cor + nf;
  double* rc = cand + nf;
  double* scal = rc + nf;  // [0] |r|, [1] |b|, [2] candidate |r|
  int* perm = c.d_dir_perm.p;
  int* status = perm + nf;  // [0] factorisation ok, [1] non-finite solve
  RF_CUDA(cudaMemsetAsync(A, 0, sizeof(double) * size_t(nf) * nf, c.stream));
  if (with_wells) {
    // rhs = -residual
    k_direct_build_cells<<<blocks_for(n), kBlock, 0, c.stream>>>(n, nf, c.d_row_ptr.p, c.d_col.p, c.d_val.p,
                                                                  c.d_res.p, -1.0, A, b);
    c.launches++;
    if (c.topo.n_wells > 0) {
      k_direct_build_wells<<<blocks_for(c.topo.n_wells), kBlock, 0, c.stream>>>(
          n, c.topo.n_wells, nf, c.d_well_ptr.p, c.d_well_perfs.p, c.d_perf_cell.p, c.d_perf_has_wi.p, c.d_jrw.p,
          c.d_jwr_perf.p, c.d_jwr_ctrl.p, c.d_jww_perf_bhp.p, c.d_jww_ctrl_q.p, c.d_jww_ctrl_bhp.p, c.d_res_tail.p, A,
          b);
      c.launches++;
    }
  } else {
    // tail-free seam: rhs already in d_rhs_red
    k_direct_build_cells<<<blocks_for(n), kBlock, 0, c.stream>>>(n, nf, c.d_row_ptr.p, c.d_col.p, c.d_val.p,
                                                                  c.d_rhs_red.p, 1.0, A, b);
    c.launches++;
  }
  RF_CUDA(cudaMemsetAsync(status, 0, 2 * sizeof(int), c.stream));
  {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c.dir_cs);
    cfg.blockDim = dim3(kDirThreads);
    cfg.dynamicSmemBytes = c.dir_smem;
    cfg.stream = c.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = c.dir_cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nn = nf;
    const double* ain = A;
    void* args[] = {&nn, &ain, &LU, &perm, &status};
    RF_CUDA(cudaLaunchKernelExC(&cfg, (const void*)k_direct_lu, args));
    c.launches++;
  }
  k_direct_solve<<<1, kDirThreads, 0, c.stream>>>(nf, LU, perm, b, x, status + 1);
  k_direct_residual<<<1, kDirThreads, 0, c.stream>>>(nf, A, b, x, nullptr, nullptr, r, scal);
  c.launches += 2;
  int st[2] = {0, 0};
  double sc[2] = {0.0, 0.0};
  d2h(c, st, status, sizeof(st));
  d2h(c, sc, scal, sizeof(sc));
  d2h_wait(c);
  LinResult out;
  out.backend = 1;
  out.rhs_norm = sc[1];
  if (!st[0]) {
    out.converged = false;
    out.final_residual_norm = sc[1];
    return out;
  }
  const double tol = 1e-12 + 5e-3 * std::fmax(sc[1], kF64Eps);
  double rn = sc[0];
  int solves = rn > 0.0 ? 1 : 0;
  for (int it = 0; it < 2; ++it) {
    if (!std::isfinite(rn) || rn <= tol) break;
    RF_CUDA(cudaMemsetAsync(status + 1, 0, sizeof(int), c.stream));
    k_direct_solve<<<1, kDirThreads, 0, c.stream>>>(nf, LU, perm, r, cor, status + 1);
    k_direct_residual<<<1, kDirThreads, 0, c.stream>>>(nf, A, b, x, cor, cand, rc, scal + 2);
    c.launches += 2;
    int bad = 0;
    double crn = 0.0;
    d2h(c, &bad, status + 1, sizeof(int));
    d2h(c, &crn, scal + 2, sizeof(double));
    d2h_wait(c);
    if (bad) break;
    if (!std::isfinite(crn) || crn >= rn * 0.95) break;
    // accept the candidate and its residual
    RF_CUDA(cudaMemcpyAsync(x, cand, sizeof(double) * nf, cudaMemcpyDeviceToDevice, c.stream));
    RF_CUDA(cudaMemcpyAsync(r, rc, sizeof(double) * nf, cudaMemcpyDeviceToDevice, c.stream));
    rn = crn;
    ++solves;
  }
  RF_CUDA(cudaMemcpyAsync(c.d_x.p, x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c.stream));
  if (nf > n3)
    RF_CUDA(cudaMemcpyAsync(c.d_dx_tail.p, x + n3, sizeof(double) * (nf - n3), cudaMemcpyDeviceToDevice, c.stream));
  std::vector<double> hx(nf);
  d2h(c, hx.data(), x, sizeof(double) * nf);
  d2h_wait(c);
  bool finite = true;
  for (double v : hx) finite = finite && std::isfinite(v);
  if (h_dx_tail) h_dx_tail->assign(hx.begin() + n3, hx.end());
  out.converged = rn <= tol;
  out.iterations = solves;
  out.final_residual_norm = rn;
  out.finite = finite;
  return out;
}

}  // namespace rf
