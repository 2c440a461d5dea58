// rf_context.hpp — host-side context of the device FIM path: deck copy, well topology, device
// buffers and the linear-solver workspace.  One context per simulator; one CUDA stream each.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <cstring>
#include <vector>

#include "../../include/ressim_fim.h"
#include "rf_device.cuh"
#include "rf_physics.cuh"

namespace rf {


struct Topology {
  int n_wells = 0, n_perfs = 0;
  std::vector<int> perf_cell, perf_well, perf_entry, perf_inj, perf_has_wi;
  std::vector<double> perf_wi;
  std::vector<int> well_rep, well_inj, well_ptr, well_perfs;  // perfs of well w: well_perfs[well_ptr[w]..]
  int max_perfs_per_well = 0;
};

// Level schedule of a lower-triangular block pattern: rows of level l are rows[ptr[l]..ptr[l+1]).
struct Levels {
  int n_levels = 0;
  std::vector<int> h_ptr;
  std::vector<int> h_rows;
  int* d_rows = nullptr;
  int* d_ptr = nullptr;
  // rows with more than kLongRowBlocks blocks (perforated rows with the well fill), per level;
  // the factorisation gives each of them a warp
  int* d_long_rows = nullptr;
  int* d_long_ptr = nullptr;
};
constexpr int kLongRowBlocks = 9;

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (count == 0) count = 1;
    RF_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// Level-order plan of the single-CTA pressure BiCGStab and block-ILU0 sweep (rf_level.cu).
// Positions number the rows level by level (rows ascending within a level); every vector of those
// solves is stored in position order.  A sweep row reads the rows of the neighbouring level through
// a shared-memory window of the previous level, and the rows a dependency reaches from further away
// ("far" rows: the well fill) through a small shared-memory cache.  Per position, a 64-bit code word
// holds up to three dependency codes (bit 15 set: far-cache slot, else offset in the neighbouring
// level) and a meta field (bits 0-2 entry count, 7 = long row listed separately; bits 3-15 own far
// slot + 1).
struct LevelPlan {
  int built = 0;          // structure present
  int n_levels = 0, width = 0, nfar_f = 0, nfar_b = 0, n_flong = 0, n_blong = 0, nnz = 0;
  int n_flong_rows = 0, n_blong_rows = 0;  // rows behind the n_flong / n_blong long entries
  DBuf<int> d_lstart, d_pos_row;
  DBuf<unsigned long long> d_fcode, d_bcode;
  DBuf<int> d_flong_ptr, d_blong_ptr;                  // long rows: entry ranges
  DBuf<unsigned short> d_flong_code, d_blong_code;     // long rows: dependency codes
  // the pressure sweeps: words with shared-memory dependency indices (static) and the per-position
  // records built from them and the factors after each factorisation; long rows' indices
  DBuf<unsigned long long> d_fword, d_bword;
  DBuf<unsigned short> d_flong_abs, d_blong_abs;
  DBuf<unsigned char> d_frec, d_brec;
  // pressure matrix in position space: [7][n] fixed-width columns, longer rows separately
  DBuf<int> d_sp_col, d_splong_row, d_splong_ptr, d_splong_col;
  int n_splong = 0, n_splong_entries = 0;
  // gather maps of the value packing: packed value i = T(src[map[i]]) (0 when map[i] < 0)
  //   factor map over plu: [fwd 3n | bwd 3n | fwd long | bwd long]; matrix map over pval:
  //   [fixed width 7n | longer rows]
  DBuf<int> d_fmap, d_smap;
  DBuf<double> d_vals64;  // [fwd 3n | bwd 3n | fwd long | bwd long | piv n | matrix 7n | longer rows]
  DBuf<float> d_vals32;
  DBuf<unsigned char> d_work;  // BiCGStab vectors in position order (9 x T) and x (double)
  size_t work_bytes = 0;
  // launch shape per value type (0 double, 1 float): threads, staging depth, dynamic shared memory
  int threads[2] = {0, 0}, stages[2] = {0, 0};
  size_t smem[2] = {0, 0};
  int fits[2] = {0, 0};
  int packed = -1;  // value type of the last packing (-1: none since the last factorisation)
  // the block-ILU0 sweep in the same level order: CSR index of each position's first lower and
  // first upper block, the forward result in position order, launch shape per value type
  DBuf<int> d_blk_f0, d_blk_b0;
  DBuf<unsigned char> d_blk_y;
  int blk_threads[2] = {0, 0}, blk_fits[2] = {0, 0};
  size_t blk_smem[2] = {0, 0};
};

// Cooperative scheduling of an ensemble's variants on shared host threads (rf_fiber.cu).  Inside a
// batch step each variant's controller runs as a fiber on its group's thread: a wait on the
// stream suspends the fiber instead of blocking the thread, and the level-scheduled kernels of the
// group's variants are collected into one launch per kind.
bool fiber_active();
void fiber_wait_event(cudaEvent_t ev);

struct Ctx {
  std::string err;
  cudaStream_t stream = nullptr;
  int stream_owned = 1;  // 0: the stream belongs to an ensemble group (rf_batch_create)
  int batched = 0;       // the context's level-scheduled kernels join its group's batched launches
  cudaEvent_t ev_wait = nullptr;  // stream waits of a fiber
  long long launches = 0;
  int device = 0, num_sms = 0;

  // deck
  int nx = 0, ny = 0, nz = 0, n = 0;
  double dx = 0, dy = 0;
  std::vector<double> dz, depth_layer, porosity, kx, ky, kz, pv;
  Fluid fluid{};   // kernels' copy (PVT table pointer in device memory)
  Fluid hfluid{};  // host controller's copy (PVT table pointer in host memory)
  std::vector<double> h_pvt;  // flat PVT table (three-phase mode)
  std::vector<RfWell> wells;
  std::vector<double> head_offset;
  int inj_rate_ctl = 0, prod_rate_ctl = 0, inj_enabled = 1;
  double tgt_inj = 0, tgt_prod = 0, tgt_inj_surf = NAN, tgt_prod_surf = NAN, bhp_min = -100, bhp_max = 2000;
  Topology topo;

  // simulator state on the host side (mirrors of what the device holds after each step)
  std::vector<double> h_p, h_sw, h_so, h_sg, h_rs;
  double time_days = 0;
  std::vector<RfTimePointRates> rate_history;
  double cum_inj = 0, cum_prod = 0, cum_mb = 0, cum_mb_oil = 0, cum_mb_gas = 0;
  std::string last_warning;

  // block pattern (reduced reservoir system): stencil + well fill
  int nnzb = 0;
  std::vector<int> h_row_ptr, h_col, h_diag, h_stencil;  // h_stencil: 7 positions per row, -1 absent
  DBuf<int> d_row_ptr, d_col, d_diag, d_stencil;
  Levels levels;
  // well fill positions: for each well, m*m block positions (row perf a, col perf b)
  std::vector<int> h_fill_off, h_fill_pos;
  DBuf<int> d_fill_off, d_fill_pos;

  // device state
  DBuf<double> d_pv, d_tx, d_ty, d_tz, d_depth;
  DBuf<double> d_p, d_sw, d_hc, d_pp, d_psw, d_phc, d_cp, d_csw, d_chc;
  DBuf<double> d_res, d_val;
  // three-phase mode: regimes (frozen per Newton attempt), the simulator's So, Sg, Rs, PVT table
  DBuf<int> d_reg;
  DBuf<double> d_so, d_sg, d_rs, d_pvt;
  // wells on the device
  DBuf<int> d_perf_cell, d_perf_well, d_perf_inj, d_perf_has_wi, d_well_ptr, d_well_perfs;
  DBuf<double> d_perf_wi, d_perf_head;
  DBuf<WellControlH> d_ctrl;
  DBuf<double> d_bhp, d_q;
  DBuf<double> d_res_tail;                       // W + P
  DBuf<double> d_jrw;                            // P*3: cell rows x own q column
  DBuf<double> d_jwr_perf, d_jwr_ctrl;           // P*3 each
  DBuf<double> d_jww_perf_bhp, d_jww_ctrl_q;     // P each
  DBuf<double> d_jww_ctrl_bhp;                   // W
  DBuf<double> d_tinv;                           // per well (1+m)^2 dense inverse
  std::vector<int> h_tinv_off;
  DBuf<int> d_tinv_off;
  DBuf<double> d_rhs_red, d_rhs_full, d_dx_tail, d_jrr_perf;  // d_jrr_perf: original perforated-row blocks
  std::vector<int> h_perf_row_blocks_off;  // per perforation: offset into d_jrr_perf (row block copy)
  DBuf<int> d_perf_row_off;

  // linear solver workspace (reduced system, 3N unknowns)
  static constexpr int kRestart = 30;
  DBuf<double> d_V, d_Z, d_w, d_x, d_tmp, d_tmp2, d_cand;
  DBuf<double> d_cpr_w;       // 3N restriction weights
  DBuf<double> d_pval;        // nnzb pressure matrix values (block pattern)
  DBuf<double> d_plu, d_pdiag;  // pressure ILU factors on the same pattern, diagonal
  DBuf<double> d_lu, d_dinv;  // block ILU factors (nnzb*9), inverse diagonal blocks (N*9)
  DBuf<unsigned char> d_bmask;  // block present in the reduced matrix (any |v| > EPS, or diagonal)
  DBuf<double> d_cres, d_full;  // last FGMRES true residual, full-system residual rows
  DBuf<double> d_dense;       // N*N dense pressure inverse when N <= 299
  DBuf<int> d_dense_perm;     // its row permutation
  int dense_ok = 0;
  // direct route of small systems: dense matrix and factors (column-major), vectors, permutation
  DBuf<double> d_dir_a, d_dir_lu, d_dir_vec;
  DBuf<int> d_dir_perm;
  int dir_rows = 0, dir_cs = 0;
  size_t dir_smem = 0;
  DBuf<double> d_pvec;        // BiCGStab workspace: 10 x N
  DBuf<double> d_partials, d_scal;
  // pinned staging for the step path's small device-to-host readbacks (d2h / d2h_wait below):
  // pageable copies stage through the driver and serialise when many contexts step at once
  unsigned char* h_pin = nullptr;
  size_t h_pin_bytes = 0, h_pin_used = 0;
  struct PinCopy {
    void* dst;
    size_t off, bytes;
  };
  std::vector<PinCopy> pin_pending;
  // controller options (rf_set_controller_options): one substep per report step, and CNV / MB
  // tolerances replacing the reference's tiers when > 0
  int ctl_one_substep = 0;
  // 1 while the adjoint solves a transposed system in d_val: the CPR build and apply use the
  // transpose of the forward coarse correction (rf_linear.cu, k_cpr_weights_t)
  int cpr_transposed = 0;
  double ctl_cnv = 0.0, ctl_mb = 0.0;
  // refinement of each CPR-FGMRES solve of the Newton systems (rf_set_linear_refinement):
  // x += solve(b - A x) until |b - A x| <= lin_refine_rtol |b|, at most lin_refine_passes solves;
  // 0 keeps the reference's single solve.  d_ref_b / d_ref_x hold b and x meanwhile.
  double lin_refine_rtol = 0.0;
  int lin_refine_passes = 0;
  DBuf<double> d_ref_b, d_ref_x;
  // discrete adjoint tape (rf_adjoint.cu); null until recording starts
  struct AdjointTape* tape = nullptr;
  int cluster_size = 0;  // CTAs in the one cluster that runs the level-scheduled kernels
  // slice ownership schedule of the distributed-shared-memory BiCGStab (built for cluster_size)
  int own_slice = 0;
  size_t dsm_bytes[2] = {0, 0};  // dynamic shared memory per CTA for double / float; 0: does not fit
  DBuf<int> d_own_rows, d_own_ptr;
  DBuf<int> d_fcnt, d_bcnt, d_fdep, d_bdep;  // packed sweep structure (ownership order)
  DBuf<unsigned short> d_reqf, d_reqb;       // per-CTA, per-position progress needed from each CTA
  DBuf<unsigned> d_cons;                     // [2][cs] consumer masks of the forward / backward sweeps
  DBuf<int> d_pipe_status;                   // nonzero: a pipelined sweep's bounded wait gave up
  DBuf<double> d_fval, d_bval, d_dval;       // packed factor values, FP64
  DBuf<float> d_fval32, d_bval32, d_dval32;  // packed factor values, mixed form
  // linear-solver precision: 0 FP64; 1 mixed (FP32 block-ILU0 and pressure stage under FP64 FGMRES)
  int precision = 0;
  DBuf<float> d_lu32, d_dinv32, d_plu32, d_pval32, d_pdiag32, d_pvec32, d_sweep32;
  DBuf<int> d_flag_dense;
  // update lists of the factorisation (rf_linear.cu, FacRecipes)
  DBuf<int> d_tri_ptr, d_tri_up, d_tri_ip, d_pt_ptr, d_pt_lp, d_pt_ue;
  DBuf<unsigned char> d_fac_simple;  // [n] rows of the simple shape (rf_linear.cu, ilu_row_simple)
  // pressure-stage solver: 0 automatic, 1 the cluster kernels, 2 the single-CTA level-order kernels
  int pressure_solver = 0;
  int level_threads = 0;  // threads of the level-order kernels (0: automatic)
  LevelPlan lvl;

  // timing
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // opt-in phase profiler: pairs of events per phase, resolved at the end of each step
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
  double phase_ms[9] = {};        // per Phase (kPhCount entries)
  long long phase_count[9] = {};
  long long* d_bicg_iters = nullptr;  // device counter of BiCGStab iterations
};

// Queue a device-to-host copy through the context's pinned staging buffer; the bytes reach `dst`
// at the next d2h_wait.  A copy larger than the buffer goes directly (and synchronously).
inline void d2h_wait(Ctx& c);
inline void d2h(Ctx& c, void* dst, const void* src, size_t bytes) {
  if (c.h_pin == nullptr || bytes > c.h_pin_bytes) {
    RF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
    return;
  }
  size_t off = (c.h_pin_used + 15) & ~size_t(15);
  if (off + bytes > c.h_pin_bytes) {
    d2h_wait(c);
    off = 0;
  }
  RF_CUDA(cudaMemcpyAsync(c.h_pin + off, src, bytes, cudaMemcpyDeviceToHost, c.stream));
  c.pin_pending.push_back({dst, off, bytes});
  c.h_pin_used = off + bytes;
}
// Wait until the context's stream has finished its queued work: a host block, or inside an
// ensemble fiber a suspension of the fiber until an event recorded now has completed.
inline void stream_wait(Ctx& c) {
  if (fiber_active() && c.ev_wait) {
    RF_CUDA(cudaEventRecord(c.ev_wait, c.stream));
    fiber_wait_event(c.ev_wait);
    RF_CUDA(cudaEventSynchronize(c.ev_wait));  // complete by now; reports a device error, if any
  } else {
    RF_CUDA(cudaStreamSynchronize(c.stream));
  }
}
// Synchronise the context's stream and deliver the queued readbacks.
inline void d2h_wait(Ctx& c) {
  stream_wait(c);
  for (const auto& q : c.pin_pending) std::memcpy(q.dst, c.h_pin + q.off, q.bytes);
  c.pin_pending.clear();
  c.h_pin_used = 0;
}

// Phases of one Newton iteration reported by rf_profile.
enum Phase {
  kPhAssembly = 0,  // residual/Jacobian assembly and norms
  kPhSchur = 1,     // well elimination and recovery
  kPhCprBuild = 2,  // weights, pressure matrix, ILU0 factorisations
  kPhCoarse = 3,    // pressure stage (BiCGStab or dense)
  kPhSmoother = 4,  // r - A x_p and the block-ILU0 sweep
  kPhKrylov = 5,    // FGMRES SpMV, Gram-Schmidt, candidate and true residual
  kPhUpdate = 6,    // chop/update, wells, substep reductions
  kPhBicgKernel = 7,  // the BiCGStab kernel alone (inside kPhCoarse)
  kPhDirect = 8,      // direct LU route of small systems
  kPhCount = 9
};
static_assert(sizeof(Ctx::phase_ms) / sizeof(double) == kPhCount, "one timing slot per phase");

inline cudaEvent_t prof_event(Ctx& c) {
  if (c.ev_used == c.ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c.ev_pool.push_back(e);
  }
  return c.ev_pool[c.ev_used++];
}
struct PhaseScope {
  Ctx& c;
  int phase;
  cudaEvent_t a = nullptr;
  PhaseScope(Ctx& c_, int ph) : c(c_), phase(ph) {
    if (c.profiling) {
      a = prof_event(c);
      cudaEventRecord(a, c.stream);
    }
  }
  ~PhaseScope() {
    if (c.profiling) {
      cudaEvent_t b = prof_event(c);
      cudaEventRecord(b, c.stream);
      c.ev_pending.push_back({phase, {a, b}});
    }
  }
};
inline void prof_resolve(Ctx& c) {
  if (!c.profiling) return;
  stream_wait(c);
  for (auto& pe : c.ev_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess) {
      c.phase_ms[pe.first] += ms;
      c.phase_count[pe.first]++;
    }
  }
  c.ev_pending.clear();
  c.ev_used = 0;
}

}  // namespace rf
