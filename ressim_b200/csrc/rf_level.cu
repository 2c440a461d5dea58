// rf_level.cu — the CPR's level-scheduled solves as ONE thread block working in level order:
// the pressure stage's BiCGStab (solve_pressure_with_bicgstab, gmres_block_jacobi.rs:622-729) and
// the block-ILU0 sweep (FimBlockIlu0Factors::apply, gmres_block_jacobi.rs:190-237).
//
// The ILU0 sweeps are chains of dependent levels (a natural-order 7-point grid has nx+ny+nz-2 of
// them), so a sweep costs levels x (one dependent step).  The cluster kernels of rf_linear.cu pay
// for each step a cross-SM signal plus a round of dependent global loads.  These kernels keep a
// whole solve on one SM:
//   - every vector of the solve is stored in position order (rows numbered level by level,
//     ascending within a level), so a level's rows are contiguous in every array;
//   - a row of level l reads its dependencies from a shared-memory window holding the values of
//     the level processed just before (l-1 forward, l+1 backward); the few rows a dependency
//     reaches from further away (the wells' fill) are kept in a shared-memory cache;
//   - the pressure solve copies the per-row data of the levels ahead (16-byte-aligned records of
//     factor values, pivot and the dependencies' shared-memory indices, plus the input vectors)
//     into shared memory with bulk copies that one thread issues per level, `stages - 1` levels
//     ahead of use, so a level step is an mbarrier wait, a block barrier, shared-memory reads and
//     the row arithmetic, with no branch per dependency;
//   - the BiCGStab updates are fused into the sweeps that read them (the search direction p into
//     the first forward sweep, s = r - alpha v and its norm into the second).
// Every row is computed with the same operations in the same order as the natural-order
// sequential sweep (entries in column order, pivot division as the reference does it), so the
// preconditioner equals the reference's; only the dot products are summed in another order (a
// fixed tree for a given thread count, hence deterministic).
#include <algorithm>
#include <cstring>
#include <mutex>

#include "rf_fiber.hpp"
#include "rf_level_layout.hpp"
#include "rf_ops.hpp"

namespace rf {

namespace {

constexpr double kEpsL = kF64Eps;
constexpr int kLvlMaxThreads = 512;
constexpr int kLvlMaxStages = 4;
constexpr unsigned kFarBit = 0x8000u;
constexpr unsigned kLongCnt = 7u;
constexpr int kSpK = 7;  // pressure-matrix entries per row held in the fixed-width layout

__device__ __forceinline__ unsigned smem_u32a(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
template <class T>
struct LvlArgs {
  int n, L, width, stages, nfar;
  int threads;  // threads that work on this solve (a batched launch may have more; they only
                // take part in the barriers, so the solve is the same as its own launch's)
  const int* lstart;   // [L + 1] first position of each level
  const int* pos_row;  // [n] natural row of each position
  // rows with more than three entries in a sweep direction (the wells' fill): entry ranges,
  // copied into shared memory with their indices and values at the start of a solve
  int n_flong_rows, n_blong_rows, n_flong, n_blong;  // rows and entries, forward and backward
  const int* flong_ptr;  // [n_flong_rows + 1]
  const int* blong_ptr;  // [n_blong_rows + 1]
  // pressure matrix in position space: rows of at most kSpK entries as [kSpK][n] column positions
  // (-1: no entry; -2 in slot 0: a longer row, listed separately) and values, in column order
  const int* sp_col;
  int n_splong;
  const int* splong_row;  // [n_splong] positions of the longer rows
  const int* splong_ptr;  // [n_splong + 1]
  const int* splong_col;
  const FRec<T>* frec;  // [n] forward records
  const BRec<T>* brec;  // [n] backward records
  const unsigned short* flong_abs;  // long rows' dependency indices into S
  const unsigned short* blong_abs;
  const T* flong_val;
  const T* blong_val;
  const T* spval;    // [kSpK][n]
  const T* splongval;
  const double* rhs;  // natural order
  double* x;          // natural order
  double* xq;         // the iterate in position order
  T* r;
  T* rh;
  T* p;
  T* v;
  T* s;
  T* t;
  T* y;
  T* ph;
  T* sh;
  int max_iters;
  long long* iter_counter;
  int* status;  // set to 3 when a wait for staged data gave up (may be null)
};

// Sums of two per-thread values over the block with a fixed tree; every thread gets both totals.
__device__ __forceinline__ void block_sum2(double& a, double& b, double* red) {
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    red[wid] = a;
    red[32 + wid] = b;
  }
  __syncthreads();
  if (t < 32) {
    double ra = t < nw ? red[t] : 0.0, rb = t < nw ? red[32 + t] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ra += __shfl_down_sync(0xffffffffu, ra, o);
      rb += __shfl_down_sync(0xffffffffu, rb, o);
    }
    if (t == 0) {
      red[64] = ra;
      red[65] = rb;
    }
  }
  __syncthreads();
  a = red[64];
  b = red[65];
}

// Staging of a level's records and inputs: one bulk copy per array (cp.async.bulk, global to
// shared memory, completion counted in bytes on the stage's mbarrier), issued by one thread.
// Both addresses must be 16-byte aligned and the size a multiple of 16 bytes: record arrays have
// 16-byte-multiple records, and input vectors are copied from their 16-byte boundary below the
// level's first position to the one above its last (the vectors are padded to that boundary).
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32a(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32a(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32a(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase of parity `parity` to complete; false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (int i = 0; i < (1 << 20); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32a(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32a(bar))
               : "memory");
}

// The long rows' entry ranges, dependency indices and values in shared memory.
template <class T>
struct LvlLongSm {
  const int* fptr;
  const int* bptr;
  const unsigned short* fidx;
  const unsigned short* bidx;
  const T* fval;
  const T* bval;
};

// One triangular sweep over all levels.  MODE 0: forward sweep of p = r + beta (p - omega v)
// (p = r on the first iteration), p stored; MODE 1: forward sweep of s = r - alpha v, s stored and
// its squares summed into acc; MODE 2: backward sweep of y.  The result goes to `out` (position
// order).  With D > 0 stages, thread 0 copies each level's records and inputs `D - 1` levels ahead
// into a ring of D slots (bulk copies completing on the slot's mbarrier), and every thread waits
// on the mbarrier before the level; a slot is refilled only after the block barrier that ends the
// level that read it.  `phase` holds each slot's mbarrier parity across sweeps.  S holds the window
// of level l at S[(l & 1) W ..], the far cache at S[2W ..] and the zero slot after it; sl is the
// level pointers.
template <class T, int MODE>
__device__ void lvl_sweep(const LvlArgs<T>& a, unsigned char* stage, unsigned long long* mbar, unsigned& phase,
                          T* S, const int* sl, const LvlLongSm<T>& lg, T* out, double& acc, double beta,
                          double omega, double alpha, bool first) {
  constexpr bool FWD = MODE != 2;
  constexpr size_t RB = FWD ? sizeof(FRec<T>) : sizeof(BRec<T>);
  constexpr int E = 16 / int(sizeof(T));  // values per 16 bytes
  const int NT = a.threads, L = a.L, W = a.width, D = a.stages;
  const int t = int(threadIdx.x) < NT ? int(threadIdx.x) : (1 << 30);  // idle threads: barriers only
  const unsigned char* recs = FWD ? reinterpret_cast<const unsigned char*>(a.frec)
                                  : reinterpret_cast<const unsigned char*>(a.brec);
  const int* lptr = FWD ? lg.fptr : lg.bptr;
  const unsigned short* lidx = FWD ? lg.fidx : lg.bidx;
  const T* lval = FWD ? lg.fval : lg.bval;
  const T* in0 = MODE == 2 ? a.y : a.r;
  const T* in1 = a.v;
  const T* in2 = a.p;
  const size_t slot_bytes = lvl_slot_bytes<T>(W);
  const size_t in_off = size_t(W) * sizeof(BRec<T>), in_bytes = lvl_in_bytes<T>(W);
  auto level_at = [&](int k) { return FWD ? k : L - 1 - k; };
  auto issue = [&](int k, int slot) {
    if (k >= L || threadIdx.x != 0) return;
    const int l = level_at(k), lst = sl[l], w = sl[l + 1] - lst;
    unsigned char* base = stage + size_t(slot) * slot_bytes;
    int a0, a1;
    lvl_input_span(lst, w, E, a0, a1);
    const unsigned rb = unsigned(size_t(w) * RB), ib = unsigned(size_t(a1 - a0) * sizeof(T));
    constexpr int nin = MODE == 0 ? 3 : MODE == 1 ? 2 : 1;
    // the slot was last read by the level before this one, finished at the block barrier
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(mbar + slot, rb + nin * ib);
    bulk_g2s(base, recs + size_t(lst) * RB, rb, mbar + slot);
    bulk_g2s(base + in_off, in0 + a0, ib, mbar + slot);
    if (MODE != 2) bulk_g2s(base + in_off + in_bytes, in1 + a0, ib, mbar + slot);
    if (MODE == 0) bulk_g2s(base + in_off + 2 * in_bytes, in2 + a0, ib, mbar + slot);
  };
  int s_iss = 0, s_cur = 0;
  if (D > 0) {
    for (int k = 0; k < D - 1; ++k) issue(k, k);
    s_iss = D - 1;
  }
  T* far = S + 2 * size_t(W);
  for (int k = 0; k < L; ++k) {
    const int l = level_at(k), lst = sl[l], w = sl[l + 1] - lst;
    const unsigned char* rbase;
    const T *inp0 = nullptr, *inp1 = nullptr, *inp2 = nullptr;
    if (D > 0) {
      issue(k + D - 1, s_iss);
      s_iss = s_iss + 1 == D ? 0 : s_iss + 1;
      if (!mbar_wait(mbar + s_cur, (phase >> s_cur) & 1u) && a.status) atomicExch(a.status, 3);
      phase ^= 1u << s_cur;
      rbase = stage + size_t(s_cur) * slot_bytes;
      const int sh = lst & (E - 1);
      inp0 = reinterpret_cast<const T*>(rbase + in_off) + sh;
      inp1 = reinterpret_cast<const T*>(rbase + in_off + in_bytes) + sh;
      inp2 = reinterpret_cast<const T*>(rbase + in_off + 2 * in_bytes) + sh;
      s_cur = s_cur + 1 == D ? 0 : s_cur + 1;
    } else {
      rbase = recs + size_t(lst) * RB;
    }
    const size_t rstride = RB;
    T* cur = S + size_t(l & 1) * W;
    // A thread's rows of one level read only earlier levels (the window of the previous level and
    // the far cache), never each other, so its rows are taken in pairs (offsets off and off + NT):
    // both rows' loads first, then both rows' arithmetic, then the stores, so the two dependency
    // chains overlap.  Per row the operations and their order are those of a single row, and the
    // rows keep their order in the thread's sum.
    struct Row {
      unsigned long long word;
      T v0, v1, v2, v3, pre, s;
      int q;
    };
    auto load_row = [&](int off, Row& R) {
      R.q = lst + off;
      const unsigned char* rp = rbase + size_t(off) * rstride;
      R.word = *reinterpret_cast<const unsigned long long*>(rp);
      const T* v = reinterpret_cast<const T*>(rp + 8);
      R.v0 = v[0];
      R.v1 = v[1];
      R.v2 = v[2];
      R.v3 = MODE == 2 ? v[3] : T(0);
      const T x0 = inp0 ? inp0[off] : in0[R.q];
      if (MODE == 0) {
        const T x1 = inp1 ? inp1[off] : in1[R.q];
        const T x2 = inp2 ? inp2[off] : in2[R.q];
        R.pre = first ? x0 : T(double(x0) + beta * (double(x2) - omega * double(x1)));
      } else if (MODE == 1) {
        const T x1 = inp1 ? inp1[off] : in1[R.q];
        R.pre = T(double(x0) - alpha * double(x1));
      } else {
        R.pre = x0;
      }
    };
    auto solve_row = [&](Row& R) {
      T s = R.pre;
      const unsigned meta = unsigned(R.word >> 48);
      if ((meta & 7u) != kLongCnt) {
        // absent entries point at the zero slot with a zero value: exact no-ops
        const T d0 = S[unsigned(R.word) & 0xffffu], d1 = S[unsigned(R.word >> 16) & 0xffffu],
                d2 = S[unsigned(R.word >> 32) & 0xffffu];
        s -= R.v0 * d0;
        s -= R.v1 * d1;
        s -= R.v2 * d2;
      } else {
        const int li = int(R.word & 0xffffu);
        for (int e = lptr[li]; e < lptr[li + 1]; ++e) s -= lval[e] * S[lidx[e]];
      }
      if (MODE == 2) s = fabs(double(R.v3)) > kEpsL ? s / R.v3 : s;
      R.s = s;
    };
    auto store_row = [&](int off, const Row& R) {
      if (MODE == 0) a.p[R.q] = R.pre;
      if (MODE == 1) {
        a.s[R.q] = R.pre;
        acc += double(R.pre) * double(R.pre);
      }
      cur[off] = R.s;
      out[R.q] = R.s;
      const unsigned fs = unsigned(R.word >> 48) >> 3;
      if (fs) far[fs - 1] = R.s;
    };
    for (int off = t; off < w; off += 2 * NT) {
      const int offb = off + NT;
      Row A, B;
      load_row(off, A);
      if (offb < w) {
        load_row(offb, B);
        solve_row(A);
        solve_row(B);
        store_row(off, A);
        store_row(offb, B);
      } else {
        solve_row(A);
        store_row(off, A);
      }
    }
    __syncthreads();
  }
}

// out = A in (pressure matrix, position space), with the dot products the solve needs next:
// MODE 0: acc0 += rh . out;  MODE 1: acc0 += out . out, acc1 += out . s.  A row's entries are
// loaded together (fixed-width layout, coalesced across the warp) and summed in column order.
template <class T, int MODE>
__device__ __forceinline__ void spmv_row_done(const LvlArgs<T>& a, int q, T s, T* out, double& acc0, double& acc1) {
  out[q] = s;
  if (MODE == 0) {
    acc0 += double(a.rh[q]) * double(s);
  } else {
    const double ti = double(s);
    acc0 += ti * ti;
    acc1 += ti * double(a.s[q]);
  }
}
template <class T, int MODE>
__device__ void lvl_spmv(const LvlArgs<T>& a, const T* in, T* out, double& acc0, double& acc1) {
  const int NT = a.threads, n = a.n;
  const int t0 = int(threadIdx.x) < NT ? int(threadIdx.x) : (1 << 30);
  // rows q and q + NT together: both rows' loads are issued before either's stores; each row's sum
  // and the thread's dot-product order are those of one row at a time
  for (int q = t0; q < n; q += 2 * NT) {
    const int nr = q + NT < n ? 2 : 1;
    int c[2][kSpK];
    T v[2][kSpK];
#pragma unroll
    for (int r = 0; r < 2; ++r)
      if (r < nr) {
#pragma unroll
        for (int j = 0; j < kSpK; ++j) {
          c[r][j] = a.sp_col[size_t(j) * n + q + r * NT];
          v[r][j] = a.spval[size_t(j) * n + q + r * NT];
        }
      }
    T s[2] = {T(0), T(0)};
#pragma unroll
    for (int r = 0; r < 2; ++r)
      if (r < nr && c[r][0] != -2) {  // -2: a longer row, below
        T x[kSpK];
#pragma unroll
        for (int j = 0; j < kSpK; ++j) x[j] = c[r][j] >= 0 ? in[c[r][j]] : T(0);
#pragma unroll
        for (int j = 0; j < kSpK; ++j)
          if (c[r][j] >= 0) s[r] += v[r][j] * x[j];
      }
#pragma unroll
    for (int r = 0; r < 2; ++r)
      if (r < nr && c[r][0] != -2) spmv_row_done<T, MODE>(a, q + r * NT, s[r], out, acc0, acc1);
  }
  for (int e = t0; e < a.n_splong; e += NT) {
    const int q = a.splong_row[e];
    T s = T(0);
    for (int k = a.splong_ptr[e]; k < a.splong_ptr[e + 1]; ++k) s += a.splongval[k] * in[a.splong_col[k]];
    spmv_row_done<T, MODE>(a, q, s, out, acc0, acc1);
  }
}

// The whole BiCGStab solve (at most max_iters iterations, tol = max(|rhs|, EPS) * 1e-6) in one
// thread block.  Dot products accumulate in double and the iterate is kept in double for either
// storage type T, as in the cluster kernels.
template <class T>
__device__ void bicgstab_level_body(const LvlArgs<T>& a, unsigned char* lvl_smem, double* red,
                                    unsigned long long* mbar) {
  const int W = a.width, n = a.n, NT = a.threads;
  const int t = int(threadIdx.x) < NT ? int(threadIdx.x) : (1 << 30);  // idle threads: barriers only
  unsigned char* stage = lvl_smem;
  T* S = reinterpret_cast<T*>(lvl_smem + size_t(a.stages) * lvl_slot_bytes<T>(W));
  int* sl = reinterpret_cast<int*>(S + 2 * size_t(W) + a.nfar + 1);
  for (int l = threadIdx.x; l <= a.L; l += blockDim.x) sl[l] = a.lstart[l];
  // the long rows, copied once per solve (their values change with every factorisation)
  const LvlLongLayout lo = lvl_long_layout<T>(LvlArgsLong{a.n_flong_rows, a.n_blong_rows, a.n_flong, a.n_blong});
  unsigned char* lbase = reinterpret_cast<unsigned char*>(S) + lvl_win_bytes<T>(W, a.nfar) +
                         lvl_up16(sizeof(int) * (size_t(a.L) + 1));
  LvlLongSm<T> lg;
  {
    T* fv = reinterpret_cast<T*>(lbase + lo.fval);
    T* bv = reinterpret_cast<T*>(lbase + lo.bval);
    int* fp = reinterpret_cast<int*>(lbase + lo.fptr);
    int* bp = reinterpret_cast<int*>(lbase + lo.bptr);
    unsigned short* fi = reinterpret_cast<unsigned short*>(lbase + lo.fidx);
    unsigned short* bi = reinterpret_cast<unsigned short*>(lbase + lo.bidx);
    for (int e = threadIdx.x; e < a.n_flong; e += blockDim.x) {
      fv[e] = a.flong_val[e];
      fi[e] = a.flong_abs[e];
    }
    for (int e = threadIdx.x; e < a.n_blong; e += blockDim.x) {
      bv[e] = a.blong_val[e];
      bi[e] = a.blong_abs[e];
    }
    for (int r = threadIdx.x; r <= a.n_flong_rows; r += blockDim.x) fp[r] = a.flong_ptr[r];
    for (int r = threadIdx.x; r <= a.n_blong_rows; r += blockDim.x) bp[r] = a.blong_ptr[r];
    lg = LvlLongSm<T>{fp, bp, fi, bi, fv, bv};
  }
  if (threadIdx.x == 0) {
    S[2 * size_t(W) + a.nfar] = T(0);  // the zero slot
    for (int k = 0; k < a.stages; ++k) mbar_init(mbar + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  unsigned phase = 0;  // parity of each staging slot's mbarrier
  double d0 = 0.0, d1 = 0.0;
  for (int q = t; q < n; q += NT) {
    const double ri = a.rhs[a.pos_row[q]] - 0.0;
    const T rt = T(ri);
    a.xq[q] = 0.0;
    a.r[q] = rt;
    a.rh[q] = rt;
    a.v[q] = T(0);
    a.p[q] = T(0);
    d0 += double(rt) * double(rt);
  }
  block_sum2(d0, d1, red);
  const double rnorm0 = sqrt(d0);
  const double tol = fmax(rnorm0, kEpsL) * 1e-6;
  const int max_iters = rnorm0 <= tol ? 0 : a.max_iters;
  double rho = d0, rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  int started = 0;
  for (int it = 0; it < max_iters; ++it) {
    started = it + 1;
    if (!isfinite(rho) || fabs(rho) < kEpsL) break;
    const double beta = it == 0 ? 0.0 : (rho / rho_prev) * (alpha / omega);
    d0 = 0.0;
    d1 = 0.0;
    lvl_sweep<T, 0>(a, stage, mbar, phase, S, sl, lg, a.y, d0, beta, omega, 0.0, it == 0);
    lvl_sweep<T, 2>(a, stage, mbar, phase, S, sl, lg, a.ph, d0, 0.0, 0.0, 0.0, false);
    lvl_spmv<T, 0>(a, a.ph, a.v, d0, d1);
    block_sum2(d0, d1, red);
    const double vd = d0;
    if (!isfinite(vd) || fabs(vd) < kEpsL) break;
    alpha = rho / vd;
    d0 = 0.0;
    d1 = 0.0;
    lvl_sweep<T, 1>(a, stage, mbar, phase, S, sl, lg, a.y, d0, 0.0, 0.0, alpha, false);
    block_sum2(d0, d1, red);
    if (sqrt(d0) <= tol) {
      for (int q = t; q < n; q += NT) a.xq[q] += alpha * double(a.ph[q]);
      break;
    }
    lvl_sweep<T, 2>(a, stage, mbar, phase, S, sl, lg, a.sh, d0, 0.0, 0.0, 0.0, false);
    d0 = 0.0;
    d1 = 0.0;
    lvl_spmv<T, 1>(a, a.sh, a.t, d0, d1);
    block_sum2(d0, d1, red);
    const double tt = d0;
    if (!isfinite(tt) || tt <= kEpsL) break;
    omega = d1 / tt;
    if (!isfinite(omega) || fabs(omega) < kEpsL) break;
    d0 = 0.0;
    d1 = 0.0;
    // positions q and q + NT together (all loads before the stores), sums in position order
    for (int q = t; q < n; q += 2 * NT) {
      const int nr = q + NT < n ? 2 : 1;
      double xv[2], pv[2], sv[2], s0[2], tv[2], hv[2];
#pragma unroll
      for (int r = 0; r < 2; ++r)
        if (r < nr) {
          const int k = q + r * NT;
          xv[r] = a.xq[k];
          pv[r] = double(a.ph[k]);
          sv[r] = double(a.sh[k]);
          s0[r] = double(a.s[k]);
          tv[r] = double(a.t[k]);
          hv[r] = double(a.rh[k]);
        }
#pragma unroll
      for (int r = 0; r < 2; ++r)
        if (r < nr) {
          const int k = q + r * NT;
          a.xq[k] = xv[r] + (alpha * pv[r] + omega * sv[r]);
          const T ri = T(s0[r] - omega * tv[r]);
          a.r[k] = ri;
          d0 += double(ri) * double(ri);
          d1 += hv[r] * double(ri);
        }
    }
    block_sum2(d0, d1, red);
    if (sqrt(d0) <= tol) break;
    rho_prev = rho;
    rho = d1;
  }
  __syncthreads();
  for (int q = t; q < n; q += NT) a.x[a.pos_row[q]] = a.xq[q];
  if (threadIdx.x == 0 && a.iter_counter) atomicAdd((unsigned long long*)a.iter_counter, (unsigned long long)started);
}

template <class T>
__global__ void __launch_bounds__(kLvlMaxThreads, 1) k_bicgstab_level(const __grid_constant__ LvlArgs<T> a) {
  extern __shared__ __align__(16) unsigned char lvl_smem[];
  __shared__ double red[72];
  __shared__ unsigned long long mbar[kLvlMaxStages];
  bicgstab_level_body(a, lvl_smem, red, mbar);
}

// Many independent pressure solves in one launch: thread block b solves item b (every item lays
// out its own shared memory inside the launch's allocation, the largest item's size).
template <class T>
struct LvlBatch {
  int count;
  LvlArgs<T> item[kBatchItems];
};
template <class T>
__global__ void __launch_bounds__(kLvlMaxThreads, 1) k_bicgstab_level_batch(const __grid_constant__ LvlBatch<T> b) {
  extern __shared__ __align__(16) unsigned char lvl_smem[];
  __shared__ double red[72];
  __shared__ unsigned long long mbar[kLvlMaxStages];
  if (blockIdx.x < unsigned(b.count)) bicgstab_level_body(b.item[blockIdx.x], lvl_smem, red, mbar);
}

// ============================================================================================
// Block ILU0 sweep in level order
// ============================================================================================
// x = U^-1 L^-1 cr for the 3x3 block factors, one thread block.  The structure is the pressure
// plan's (the same block pattern, levels, dependency codes and far rows); each row reads its factor
// blocks straight from the CSR-ordered factors (the row's lower or upper blocks are contiguous) and
// its dependencies, three values per row, from the shared-memory window of the neighbouring level
// or the far cache.  Row arithmetic as block_fwd_row / block_bwd_row: same products and sums in
// the same order.
template <class T>
struct BlkArgs {
  int n, L, width;
  int threads;  // working threads (see LvlArgs::threads)
  const int* lstart;
  const int* pos_row;
  const int* f0;  // [n] CSR index of each position's first lower block
  const int* b0;  // [n] CSR index of each position's first upper block
  const unsigned long long* fcode;
  const unsigned long long* bcode;
  const int* flong_ptr;
  const unsigned short* flong_code;
  const int* blong_ptr;
  const unsigned short* blong_code;
  const T* lu;    // nnzb x 9
  const T* dinv;  // n x 9
  const double* cr;  // natural order, 3 per row
  T* y;              // position order, 3 per row
  double* x;         // natural order, 3 per row
};

template <class T>
__device__ __forceinline__ const T* dep3(unsigned c, const T* nb, const T* far) {
  return (c & kFarBit) ? far + 3 * (c & 0x7fffu) : nb + 3 * c;
}

template <class T>
__device__ __forceinline__ void blk_sub(T& b0, T& b1, T& b2, const T* B, const T* v) {
  const T v0 = v[0], v1 = v[1], v2 = v[2];
  b0 -= B[0] * v0 + B[1] * v1 + B[2] * v2;
  b1 -= B[3] * v0 + B[4] * v1 + B[5] * v2;
  b2 -= B[6] * v0 + B[7] * v1 + B[8] * v2;
}

template <class T>
__device__ void block_sweep_level_body(const BlkArgs<T>& a, unsigned char* blk_smem) {
  const int W = a.width, L = a.L, NT = a.threads;
  const int t = int(threadIdx.x) < NT ? int(threadIdx.x) : (1 << 30);  // idle threads: barriers only
  T* win = reinterpret_cast<T*>(blk_smem);  // [2][3 W]
  T* far = win + 6 * size_t(W);
  // forward: y = L^-1 cr
  for (int l = 0; l < L; ++l) {
    const int lst = a.lstart[l], w = a.lstart[l + 1] - lst;
    const T* nb = win + 3 * size_t(W) * ((l + 1) & 1);
    T* cur = win + 3 * size_t(W) * (l & 1);
    for (int off = t; off < w; off += NT) {
      const int q = lst + off, i = a.pos_row[q], k0 = a.f0[q];
      const unsigned long long code = a.fcode[q];
      const unsigned meta = unsigned(code >> 48), cnt = meta & 7u;
      T b0 = T(a.cr[3 * size_t(i)]), b1 = T(a.cr[3 * size_t(i) + 1]), b2 = T(a.cr[3 * size_t(i) + 2]);
      if (cnt != kLongCnt) {
#pragma unroll
        for (unsigned j = 0; j < 3; ++j)
          if (j < cnt)
            blk_sub(b0, b1, b2, a.lu + size_t(k0 + int(j)) * 9, dep3(unsigned(code >> (16 * j)) & 0xffffu, nb, far));
      } else {
        const int li = int(code & 0xffffu), e0 = a.flong_ptr[li], e1 = a.flong_ptr[li + 1];
        for (int e = e0; e < e1; ++e)
          blk_sub(b0, b1, b2, a.lu + size_t(k0 + e - e0) * 9, dep3(unsigned(a.flong_code[e]), nb, far));
      }
      cur[3 * off] = b0;
      cur[3 * off + 1] = b1;
      cur[3 * off + 2] = b2;
      a.y[3 * size_t(q)] = b0;
      a.y[3 * size_t(q) + 1] = b1;
      a.y[3 * size_t(q) + 2] = b2;
      const unsigned fs = meta >> 3;
      if (fs) {
        far[3 * (fs - 1)] = b0;
        far[3 * (fs - 1) + 1] = b1;
        far[3 * (fs - 1) + 2] = b2;
      }
    }
    __syncthreads();
  }
  // backward: x = U^-1 y with the inverse diagonal blocks
  for (int k = 0; k < L; ++k) {
    const int l = L - 1 - k, lst = a.lstart[l], w = a.lstart[l + 1] - lst;
    const T* nb = win + 3 * size_t(W) * ((k + 1) & 1);
    T* cur = win + 3 * size_t(W) * (k & 1);
    for (int off = t; off < w; off += NT) {
      const int q = lst + off, i = a.pos_row[q], k0 = a.b0[q];
      const unsigned long long code = a.bcode[q];
      const unsigned meta = unsigned(code >> 48), cnt = meta & 7u;
      T b0 = a.y[3 * size_t(q)], b1 = a.y[3 * size_t(q) + 1], b2 = a.y[3 * size_t(q) + 2];
      if (cnt != kLongCnt) {
#pragma unroll
        for (unsigned j = 0; j < 3; ++j)
          if (j < cnt)
            blk_sub(b0, b1, b2, a.lu + size_t(k0 + int(j)) * 9, dep3(unsigned(code >> (16 * j)) & 0xffffu, nb, far));
      } else {
        const int li = int(code & 0xffffu), e0 = a.blong_ptr[li], e1 = a.blong_ptr[li + 1];
        for (int e = e0; e < e1; ++e)
          blk_sub(b0, b1, b2, a.lu + size_t(k0 + e - e0) * 9, dep3(unsigned(a.blong_code[e]), nb, far));
      }
      const T* D = a.dinv + 9 * size_t(i);
      const T o0 = D[0] * b0 + D[1] * b1 + D[2] * b2;
      const T o1 = D[3] * b0 + D[4] * b1 + D[5] * b2;
      const T o2 = D[6] * b0 + D[7] * b1 + D[8] * b2;
      cur[3 * off] = o0;
      cur[3 * off + 1] = o1;
      cur[3 * off + 2] = o2;
      a.x[3 * size_t(i)] = double(o0);
      a.x[3 * size_t(i) + 1] = double(o1);
      a.x[3 * size_t(i) + 2] = double(o2);
      const unsigned fs = meta >> 3;
      if (fs) {
        far[3 * (fs - 1)] = o0;
        far[3 * (fs - 1) + 1] = o1;
        far[3 * (fs - 1) + 2] = o2;
      }
    }
    __syncthreads();
  }
}

template <class T>
__global__ void __launch_bounds__(kLvlMaxThreads, 1) k_block_sweep_level(const __grid_constant__ BlkArgs<T> a) {
  extern __shared__ __align__(16) unsigned char blk_smem[];
  block_sweep_level_body(a, blk_smem);
}

template <class T>
struct BlkBatch {
  int count;
  BlkArgs<T> item[kBatchItems];
};
template <class T>
__global__ void __launch_bounds__(kLvlMaxThreads, 1) k_block_sweep_level_batch(const __grid_constant__ BlkBatch<T> b) {
  extern __shared__ __align__(16) unsigned char blk_smem[];
  if (blockIdx.x < unsigned(b.count)) block_sweep_level_body(b.item[blockIdx.x], blk_smem);
}

template <class T>
size_t blk_smem_bytes(int W, int nfar) {
  return (6 * size_t(W) + 3 * size_t(std::max(nfar, 1))) * sizeof(T);
}

// dst[i] = T(src[map[i]]), or 0 where map[i] < 0
template <class T>
__global__ void k_lvl_gather(long long m, const int* __restrict__ map, const double* __restrict__ src,
                             T* __restrict__ dst) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += stride) {
    const int k = map[i];
    dst[i] = k >= 0 ? T(src[k]) : T(0);
  }
}

// The sweep records from the gathered factor values (position order) and the static words.
template <class T>
__global__ void k_lvl_pack_rec(int n, const unsigned long long* __restrict__ fword,
                               const unsigned long long* __restrict__ bword, const T* __restrict__ fval,
                               const T* __restrict__ bval, const T* __restrict__ piv, FRec<T>* __restrict__ frec,
                               BRec<T>* __restrict__ brec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  FRec<T> f;
  BRec<T> b;
  f.word = fword[q];
  b.word = bword[q];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    f.v[j] = fval[size_t(j) * n + q];
    b.v[j] = bval[size_t(j) * n + q];
  }
  b.piv = piv[q];
  frec[q] = f;
  brec[q] = b;
}

template <class T>
size_t lvl_smem_bytes(int W, int stages, int nfar, int L, const LvlArgsLong& lg) {
  return size_t(stages) * lvl_slot_bytes<T>(W) + lvl_win_bytes<T>(W, nfar) + lvl_up16(sizeof(int) * (size_t(L) + 1)) +
         lvl_long_layout<T>(lg).total;
}

// offsets of the packed value segments (elements)
struct LvlSeg {
  size_t fval, bval, flong, blong, piv, sp, splong, total;
};
LvlSeg lvl_segments(const LevelPlan& P, int n) {
  LvlSeg s;
  s.fval = 0;
  s.bval = 3 * size_t(n);
  s.flong = 6 * size_t(n);
  s.blong = s.flong + size_t(P.n_flong);
  s.piv = s.blong + size_t(P.n_blong);
  s.sp = s.piv + size_t(n);
  s.splong = s.sp + size_t(kSpK) * n;
  s.total = s.splong + size_t(P.n_splong_entries);
  return s;
}

int auto_threads(const Ctx& c) {
  const int nt = c.level_threads > 0 ? c.level_threads
                                     : std::min(kLvlMaxThreads, std::max(64, (c.lvl.width + 31) / 32 * 32));
  return std::max(32, std::min(kLvlMaxThreads, nt / 32 * 32));
}

template <class T>
void choose_block_shape(Ctx& c, int f) {
  LevelPlan& P = c.lvl;
  int optin = 0;
  RF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
  const size_t bytes = blk_smem_bytes<T>(P.width, std::max(P.nfar_f, P.nfar_b));
  P.blk_fits[f] = 0;
  if (bytes + 1024 > size_t(optin)) return;
  P.blk_smem[f] = bytes;
  P.blk_threads[f] = auto_threads(c);
  raise_dynamic_smem((const void*)k_block_sweep_level<T>, bytes);
  raise_dynamic_smem((const void*)k_block_sweep_level_batch<T>, bytes);
  P.blk_fits[f] = 1;
}

template <class T>
void choose_shape(Ctx& c, int f) {
  LevelPlan& P = c.lvl;
  int optin = 0;
  RF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
  cudaFuncAttributes fa;
  RF_CUDA(cudaFuncGetAttributes(&fa, (const void*)k_bicgstab_level<T>));
  const size_t budget = size_t(optin) > fa.sharedSizeBytes + 1024 ? size_t(optin) - fa.sharedSizeBytes - 1024 : 0;
  const int nfar = std::max(P.nfar_f, P.nfar_b);
  P.fits[f] = 0;
  const LvlArgsLong lg{P.n_flong_rows, P.n_blong_rows, P.n_flong, P.n_blong};
  if (lvl_smem_bytes<T>(P.width, 0, nfar, P.n_levels, lg) > budget) return;
  int st = kLvlMaxStages;
  while (st > 0 && lvl_smem_bytes<T>(P.width, st, nfar, P.n_levels, lg) > budget) --st;
  if (st == 1) st = 0;  // one stage only re-reads what it just copied: direct loads do the same
  P.stages[f] = st;
  P.smem[f] = lvl_smem_bytes<T>(P.width, st, nfar, P.n_levels, lg);
  P.threads[f] = auto_threads(c);
  raise_dynamic_smem((const void*)k_bicgstab_level<T>, P.smem[f]);
  raise_dynamic_smem((const void*)k_bicgstab_level_batch<T>, P.smem[f]);
  P.fits[f] = 1;
}

}  // namespace

// Level-order structure of the current block pattern and level schedule (built once per topology).
void build_level_plan(Ctx& c) {
  LevelPlan& P = c.lvl;
  P.built = 0;
  const int n = c.n, L = c.levels.n_levels;
  if (n <= 0 || L <= 0) return;
  const std::vector<int>& lp = c.levels.h_ptr;
  const std::vector<int>& rows = c.levels.h_rows;
  std::vector<int> lvl(n), pos(n);
  int W = 1;
  for (int l = 0; l < L; ++l) {
    W = std::max(W, lp[l + 1] - lp[l]);
    for (int q = lp[l]; q < lp[l + 1]; ++q) {
      lvl[rows[q]] = l;
      pos[rows[q]] = q;
    }
  }
  if (W >= int(kFarBit)) return;
  // far-cache slots: rows a dependency reaches from further than the neighbouring level
  std::vector<int> ffar(n, -1), bfar(n, -1);
  int nff = 0, nfb = 0;
  for (int r = 0; r < n; ++r) {
    for (int k = c.h_row_ptr[r]; k < c.h_diag[r]; ++k) {
      const int col = c.h_col[k];
      if (lvl[col] != lvl[r] - 1 && ffar[col] < 0) ffar[col] = nff++;
    }
    for (int k = c.h_diag[r] + 1; k < c.h_row_ptr[r + 1]; ++k) {
      const int col = c.h_col[k];
      if (lvl[col] != lvl[r] + 1 && bfar[col] < 0) bfar[col] = nfb++;
    }
  }
  if (nff >= 8191 || nfb >= 8191) return;
  std::vector<unsigned long long> fcode(n), bcode(n);
  std::vector<int> fmap(6 * size_t(n), -1), flong_ptr{0}, blong_ptr{0}, flong_map, blong_map;
  std::vector<unsigned short> flong_code, blong_code;
  auto pack_row = [&](bool fwd, int q, int r) {
    const int l = lvl[r];
    const int k0 = fwd ? c.h_row_ptr[r] : c.h_diag[r] + 1;
    const int k1 = fwd ? c.h_diag[r] : c.h_row_ptr[r + 1];
    const int cnt = k1 - k0;
    auto code_of = [&](int col) -> unsigned {
      const int lc = lvl[col];
      if (lc == (fwd ? l - 1 : l + 1)) return unsigned(pos[col] - lp[lc]);
      return kFarBit | unsigned(fwd ? ffar[col] : bfar[col]);
    };
    unsigned long long word = 0;
    unsigned meta;
    const size_t seg = fwd ? 0 : 3 * size_t(n);
    if (cnt <= 3) {
      for (int j = 0; j < cnt; ++j) {
        word |= (unsigned long long)code_of(c.h_col[k0 + j]) << (16 * j);
        fmap[seg + size_t(j) * n + q] = k0 + j;
      }
      meta = unsigned(cnt);
    } else {
      std::vector<int>& ptr = fwd ? flong_ptr : blong_ptr;
      std::vector<int>& map = fwd ? flong_map : blong_map;
      std::vector<unsigned short>& code = fwd ? flong_code : blong_code;
      word = (unsigned long long)(ptr.size() - 1);
      for (int k = k0; k < k1; ++k) {
        code.push_back(static_cast<unsigned short>(code_of(c.h_col[k])));
        map.push_back(k);
      }
      ptr.push_back(int(map.size()));
      meta = kLongCnt;
    }
    meta |= unsigned((fwd ? ffar[r] : bfar[r]) + 1) << 3;
    word |= (unsigned long long)meta << 48;
    (fwd ? fcode : bcode)[q] = word;
  };
  for (int q = 0; q < n; ++q) {
    pack_row(true, q, rows[q]);
    pack_row(false, q, rows[q]);
  }
  if (flong_ptr.size() > 65536 || blong_ptr.size() > 65536) return;
  // the pressure sweeps' words: dependency indices into S (window of level lc at (lc & 1) W, far
  // cache at 2W, zero slot at 2W + nfar)
  const int nfar = std::max(nff, nfb);
  const unsigned zero_slot = unsigned(2 * W + nfar);
  if (zero_slot >= 65535u) return;
  std::vector<unsigned long long> fword(n), bword(n);
  std::vector<unsigned short> flong_abs, blong_abs;
  for (int q = 0; q < n; ++q) {
    const int r = rows[q], l = lvl[r];
    for (int dir = 0; dir < 2; ++dir) {
      const bool fwd = dir == 0;
      const int k0 = fwd ? c.h_row_ptr[r] : c.h_diag[r] + 1;
      const int k1 = fwd ? c.h_diag[r] : c.h_row_ptr[r + 1];
      auto abs_of = [&](int col) -> unsigned {
        const int lc = lvl[col];
        if (lc == (fwd ? l - 1 : l + 1)) return unsigned((lc & 1) * W + pos[col] - lp[lc]);
        return unsigned(2 * W + (fwd ? ffar[col] : bfar[col]));
      };
      const unsigned long long code = (fwd ? fcode : bcode)[q];
      const unsigned meta = unsigned(code >> 48);
      unsigned long long word;
      if ((meta & 7u) != kLongCnt) {
        word = 0;
        for (int j = 0; j < 3; ++j)
          word |= (unsigned long long)(j < k1 - k0 ? abs_of(c.h_col[k0 + j]) : zero_slot) << (16 * j);
      } else {
        word = code & 0xffffull;  // the long-row index
        std::vector<unsigned short>& out = fwd ? flong_abs : blong_abs;
        for (int k = k0; k < k1; ++k) out.push_back(static_cast<unsigned short>(abs_of(c.h_col[k])));
      }
      word |= (unsigned long long)meta << 48;
      (fwd ? fword : bword)[q] = word;
    }
  }
  P.n_levels = L;
  P.width = W;
  P.nfar_f = nff;
  P.nfar_b = nfb;
  P.n_flong = int(flong_map.size());
  P.n_blong = int(blong_map.size());
  P.n_flong_rows = int(flong_ptr.size()) - 1;
  P.n_blong_rows = int(blong_ptr.size()) - 1;
  P.nnz = c.h_row_ptr[n];
  fmap.insert(fmap.end(), flong_map.begin(), flong_map.end());
  fmap.insert(fmap.end(), blong_map.begin(), blong_map.end());
  // pressure matrix in position space: fixed-width rows, longer rows separately; smap gathers the
  // values: [kSpK][n] fixed-width slots, then the longer rows' entries
  std::vector<int> sp_col(size_t(kSpK) * n, -1), smap(size_t(kSpK) * n, -1), splong_row, splong_ptr{0},
      splong_col, splong_map, f0(n), b0(n);
  for (int q = 0; q < n; ++q) {
    const int r = rows[q];
    const int k0 = c.h_row_ptr[r], k1 = c.h_row_ptr[r + 1];
    if (k1 - k0 <= kSpK) {
      for (int k = k0; k < k1; ++k) {
        sp_col[size_t(k - k0) * n + q] = pos[c.h_col[k]];
        smap[size_t(k - k0) * n + q] = k;
      }
    } else {
      sp_col[q] = -2;
      splong_row.push_back(q);
      for (int k = k0; k < k1; ++k) {
        splong_col.push_back(pos[c.h_col[k]]);
        splong_map.push_back(k);
      }
      splong_ptr.push_back(int(splong_col.size()));
    }
    f0[q] = c.h_row_ptr[r];
    b0[q] = c.h_diag[r] + 1;
  }
  P.n_splong = int(splong_row.size());
  P.n_splong_entries = int(splong_col.size());
  smap.insert(smap.end(), splong_map.begin(), splong_map.end());
  auto up_i = [](DBuf<int>& b, const std::vector<int>& h) {
    b.free();
    b.alloc(h.size());
    if (!h.empty()) RF_CUDA(cudaMemcpy(b.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
  };
  auto up_u64 = [](DBuf<unsigned long long>& b, const std::vector<unsigned long long>& h) {
    b.free();
    b.alloc(h.size());
    RF_CUDA(cudaMemcpy(b.p, h.data(), sizeof(unsigned long long) * h.size(), cudaMemcpyHostToDevice));
  };
  auto up_u16 = [](DBuf<unsigned short>& b, const std::vector<unsigned short>& h) {
    b.free();
    b.alloc(h.size());
    if (!h.empty()) RF_CUDA(cudaMemcpy(b.p, h.data(), sizeof(unsigned short) * h.size(), cudaMemcpyHostToDevice));
  };
  up_i(P.d_lstart, lp);
  up_i(P.d_pos_row, rows);
  up_u64(P.d_fcode, fcode);
  up_u64(P.d_bcode, bcode);
  up_i(P.d_flong_ptr, flong_ptr);
  up_i(P.d_blong_ptr, blong_ptr);
  up_u16(P.d_flong_code, flong_code);
  up_u16(P.d_blong_code, blong_code);
  up_u64(P.d_fword, fword);
  up_u64(P.d_bword, bword);
  up_u16(P.d_flong_abs, flong_abs);
  up_u16(P.d_blong_abs, blong_abs);
  P.d_frec.free();
  P.d_brec.free();
  P.d_frec.alloc(size_t(n) * sizeof(FRec<double>));
  P.d_brec.alloc(size_t(n) * sizeof(BRec<double>));
  up_i(P.d_sp_col, sp_col);
  up_i(P.d_splong_row, splong_row);
  up_i(P.d_splong_ptr, splong_ptr);
  up_i(P.d_splong_col, splong_col);
  up_i(P.d_fmap, fmap);
  up_i(P.d_smap, smap);
  up_i(P.d_blk_f0, f0);
  up_i(P.d_blk_b0, b0);
  P.d_vals64.free();
  P.d_vals32.free();
  P.d_work.free();
  // ten position-order vectors (the iterate in double, nine of the solve's type), each padded to
  // a multiple of four values so every vector starts on a 16-byte boundary and the staging's bulk
  // copies, rounded out to 16-byte boundaries, stay inside the buffer
  P.work_bytes = lvl_work_pad(n) * (9 * sizeof(double) + sizeof(double)) + 64;
  P.d_work.alloc(P.work_bytes);
  P.d_blk_y.free();
  P.d_blk_y.alloc(3 * size_t(n) * sizeof(double));
  P.packed = -1;
  choose_shape<double>(c, 0);
  choose_shape<float>(c, 1);
  choose_block_shape<double>(c, 0);
  choose_block_shape<float>(c, 1);
  P.built = 1;
}

void free_level_plan(Ctx& c) {
  LevelPlan& P = c.lvl;
  for (auto* b : {&P.d_lstart, &P.d_pos_row, &P.d_flong_ptr, &P.d_blong_ptr, &P.d_sp_col, &P.d_splong_row,
                  &P.d_splong_ptr, &P.d_splong_col, &P.d_fmap, &P.d_smap, &P.d_blk_f0, &P.d_blk_b0})
    b->free();
  P.d_fcode.free();
  P.d_bcode.free();
  P.d_flong_code.free();
  P.d_blong_code.free();
  P.d_fword.free();
  P.d_bword.free();
  P.d_flong_abs.free();
  P.d_blong_abs.free();
  P.d_frec.free();
  P.d_brec.free();
  P.d_vals64.free();
  P.d_vals32.free();
  P.d_work.free();
  P.d_blk_y.free();
  P.built = 0;
}

// Re-derive the launch shapes (thread count changed).
void level_plan_reshape(Ctx& c) {
  if (!c.lvl.built) return;
  choose_shape<double>(c, 0);
  choose_shape<float>(c, 1);
  choose_block_shape<double>(c, 0);
  choose_block_shape<float>(c, 1);
}

// Automatic choice: the one-block level-order kernels for decks of up to kLevelAutoCells cells and
// for every variant of a batched ensemble (their launches join the group's batched launches); the
// cluster kernels for larger single decks, where a level holds more rows than one SM issues
// quickly (measured crossover between 19k and 40k cells).
constexpr int kLevelAutoCells = 32768;

static bool level_chosen(const Ctx& c) {
  if (c.pressure_solver == 2) return true;
  return c.pressure_solver == 0 && (c.batched || c.n <= kLevelAutoCells);
}

bool level_solver_active(const Ctx& c) {
  const int f = c.precision == 1 ? 1 : 0;
  return c.lvl.built && c.lvl.fits[f] && level_chosen(c);
}

bool level_block_sweep_active(const Ctx& c) {
  const int f = c.precision == 1 ? 1 : 0;
  return c.lvl.built && c.lvl.blk_fits[f] && level_chosen(c);
}

void level_pack(Ctx& c) {
  LevelPlan& P = c.lvl;
  const int n = c.n;
  const LvlSeg g = lvl_segments(P, n);
  const long long mf = (long long)g.piv;                    // factor entries: fval, bval, long rows
  const long long ms = (long long)(g.total - g.sp);           // matrix entries: fixed width, longer rows
  if (c.precision == 1) {
    if (!P.d_vals32.p) P.d_vals32.alloc(g.total);
    float* v = P.d_vals32.p;
    k_lvl_gather<float><<<blocks_for(mf), kBlock, 0, c.stream>>>(mf, P.d_fmap.p, c.d_plu.p, v);
    k_lvl_gather<float><<<blocks_for(n), kBlock, 0, c.stream>>>(n, P.d_pos_row.p, c.d_pdiag.p, v + g.piv);
    k_lvl_gather<float><<<blocks_for(ms), kBlock, 0, c.stream>>>(ms, P.d_smap.p, c.d_pval.p, v + g.sp);
    k_lvl_pack_rec<float><<<blocks_for(n), kBlock, 0, c.stream>>>(
        n, P.d_fword.p, P.d_bword.p, v + g.fval, v + g.bval, v + g.piv, reinterpret_cast<FRec<float>*>(P.d_frec.p),
        reinterpret_cast<BRec<float>*>(P.d_brec.p));
    P.packed = 1;
  } else {
    if (!P.d_vals64.p) P.d_vals64.alloc(g.total);
    double* v = P.d_vals64.p;
    k_lvl_gather<double><<<blocks_for(mf), kBlock, 0, c.stream>>>(mf, P.d_fmap.p, c.d_plu.p, v);
    k_lvl_gather<double><<<blocks_for(n), kBlock, 0, c.stream>>>(n, P.d_pos_row.p, c.d_pdiag.p, v + g.piv);
    k_lvl_gather<double><<<blocks_for(ms), kBlock, 0, c.stream>>>(ms, P.d_smap.p, c.d_pval.p, v + g.sp);
    k_lvl_pack_rec<double><<<blocks_for(n), kBlock, 0, c.stream>>>(
        n, P.d_fword.p, P.d_bword.p, v + g.fval, v + g.bval, v + g.piv, reinterpret_cast<FRec<double>*>(P.d_frec.p),
        reinterpret_cast<BRec<double>*>(P.d_brec.p));
    P.packed = 0;
  }
  c.launches += 4;
}

static_assert(sizeof(LvlArgs<double>) <= kBatchArgBytes && sizeof(BlkArgs<double>) <= kBatchArgBytes,
              "batched launch arguments must fit a batch item");

// File a launch with the calling fiber's group (batched stepping); false when not in a fiber.
static bool submit_item(int kind, int type, const void* args, size_t bytes, int threads, size_t smem) {
  return fiber_file(kind, type, args, bytes, threads, smem);
}

template <class A, class B>
static bool launch_batch(const BatchItem* const* items, int count, cudaStream_t stream, const void* fn) {
  B b;
  b.count = count;
  int threads = 32;
  size_t smem = 0;
  for (int i = 0; i < count; ++i) {
    std::memcpy(&b.item[i], items[i]->args, sizeof(A));
    threads = std::max(threads, items[i]->threads);
    smem = std::max(smem, items[i]->smem);
  }
  void* args[] = {&b};
  return cudaLaunchKernel(fn, dim3(count), dim3(threads), args, smem, stream) == cudaSuccess;
}

bool launch_batch_items(int kind, int type, const BatchItem* const* items, int count, cudaStream_t stream) {
  if (count <= 0) return true;
  if (kind == kBatchFactor) return launch_factor_batch(items, count, stream);
  if (kind == kBatchPressure) {
    if (type == 1)
      return launch_batch<LvlArgs<float>, LvlBatch<float>>(items, count, stream,
                                                           (const void*)k_bicgstab_level_batch<float>);
    return launch_batch<LvlArgs<double>, LvlBatch<double>>(items, count, stream,
                                                           (const void*)k_bicgstab_level_batch<double>);
  }
  if (type == 1)
    return launch_batch<BlkArgs<float>, BlkBatch<float>>(items, count, stream,
                                                         (const void*)k_block_sweep_level_batch<float>);
  return launch_batch<BlkArgs<double>, BlkBatch<double>>(items, count, stream,
                                                         (const void*)k_block_sweep_level_batch<double>);
}

template <class T>
static void launch_level(Ctx& c, const double* rhs, double* x) {
  LevelPlan& P = c.lvl;
  const int f = sizeof(T) == 4 ? 1 : 0;
  if (P.packed != f) throw CudaError("level-order pressure solve: factors not packed for this precision");
  const int n = c.n;
  const LvlSeg g = lvl_segments(P, n);
  const T* vals;
  if constexpr (sizeof(T) == 4)
    vals = P.d_vals32.p;
  else
    vals = P.d_vals64.p;
  LvlArgs<T> a;
  a.n = n;
  a.L = P.n_levels;
  a.width = P.width;
  a.stages = P.stages[f];
  a.lstart = P.d_lstart.p;
  a.pos_row = P.d_pos_row.p;
  a.n_flong_rows = P.n_flong_rows;
  a.n_blong_rows = P.n_blong_rows;
  a.n_flong = P.n_flong;
  a.n_blong = P.n_blong;
  a.flong_ptr = P.d_flong_ptr.p;
  a.blong_ptr = P.d_blong_ptr.p;
  a.sp_col = P.d_sp_col.p;
  a.n_splong = P.n_splong;
  a.splong_row = P.d_splong_row.p;
  a.splong_ptr = P.d_splong_ptr.p;
  a.splong_col = P.d_splong_col.p;
  a.frec = reinterpret_cast<const FRec<T>*>(P.d_frec.p);
  a.brec = reinterpret_cast<const BRec<T>*>(P.d_brec.p);
  a.flong_abs = P.d_flong_abs.p;
  a.blong_abs = P.d_blong_abs.p;
  a.nfar = std::max(P.nfar_f, P.nfar_b);
  a.flong_val = vals + g.flong;
  a.blong_val = vals + g.blong;
  a.spval = vals + g.sp;
  a.splongval = vals + g.splong;
  a.rhs = rhs;
  a.x = x;
  const size_t np = lvl_work_pad(n);
  double* xq = reinterpret_cast<double*>(P.d_work.p);
  T* vb = reinterpret_cast<T*>(P.d_work.p + sizeof(double) * np);
  a.xq = xq;
  a.r = vb;
  a.rh = vb + np;
  a.p = vb + 2 * np;
  a.v = vb + 3 * np;
  a.s = vb + 4 * np;
  a.t = vb + 5 * np;
  a.y = vb + 6 * np;
  a.ph = vb + 7 * np;
  a.sh = vb + 8 * np;
  a.max_iters = 50;
  a.iter_counter = c.d_bicg_iters;
  a.status = c.d_pipe_status.p;
  a.threads = P.threads[f];
  if (c.batched && submit_item(kBatchPressure, f, &a, sizeof(a), P.threads[f], P.smem[f])) return;
  c.launches++;
  k_bicgstab_level<T><<<1, P.threads[f], P.smem[f], c.stream>>>(a);
  RF_CUDA(cudaGetLastError());
}

void launch_bicgstab_level(Ctx& c, const double* rhs, double* x) {
  if (c.precision == 1)
    launch_level<float>(c, rhs, x);
  else
    launch_level<double>(c, rhs, x);
}

// x = BlockILU(cr) with the level-order sweep kernel and the factors of the current precision.
void launch_block_sweep_level(Ctx& c, const double* cr, double* x, const void* lu, const void* dinv) {
  LevelPlan& P = c.lvl;
  const int f = c.precision == 1 ? 1 : 0;
  auto fill = [&](auto& a) {
    a.n = c.n;
    a.L = P.n_levels;
    a.width = P.width;
    a.lstart = P.d_lstart.p;
    a.pos_row = P.d_pos_row.p;
    a.f0 = P.d_blk_f0.p;
    a.b0 = P.d_blk_b0.p;
    a.fcode = P.d_fcode.p;
    a.bcode = P.d_bcode.p;
    a.flong_ptr = P.d_flong_ptr.p;
    a.flong_code = P.d_flong_code.p;
    a.blong_ptr = P.d_blong_ptr.p;
    a.blong_code = P.d_blong_code.p;
    a.cr = cr;
    a.x = x;
    a.threads = P.blk_threads[f];
  };
  if (f == 1) {
    BlkArgs<float> a;
    fill(a);
    a.lu = static_cast<const float*>(lu);
    a.dinv = static_cast<const float*>(dinv);
    a.y = reinterpret_cast<float*>(P.d_blk_y.p);
    if (c.batched && submit_item(kBatchBlockSweep, 1, &a, sizeof(a), P.blk_threads[1], P.blk_smem[1])) return;
    c.launches++;
    k_block_sweep_level<float><<<1, P.blk_threads[1], P.blk_smem[1], c.stream>>>(a);
  } else {
    BlkArgs<double> a;
    fill(a);
    a.lu = static_cast<const double*>(lu);
    a.dinv = static_cast<const double*>(dinv);
    a.y = reinterpret_cast<double*>(P.d_blk_y.p);
    if (c.batched && submit_item(kBatchBlockSweep, 0, &a, sizeof(a), P.blk_threads[0], P.blk_smem[0])) return;
    c.launches++;
    k_block_sweep_level<double><<<1, P.blk_threads[0], P.blk_smem[0], c.stream>>>(a);
  }
  RF_CUDA(cudaGetLastError());
}

}  // namespace rf
