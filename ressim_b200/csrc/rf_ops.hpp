// rf_ops.hpp — host launchers of the device kernels (assembly, norms, linear solve).
#pragma once

#include <vector>

#include "rf_context.hpp"

namespace rf {

constexpr int kNormQuantities = 13;  // see k_norms_cells

void launch_assembly(Ctx& c, double dt);
// h_out receives kNormQuantities + 1 doubles (family maxima, FVF sums, CNV maxima, residual
// sums, pore-volume sum, violating pore volume).
void launch_norms(Ctx& c, double dt, double* h_out);
// Three-phase assembly and the first pass of the norms (rf_blackoil.cu).
void launch_assembly3(Ctx& c, double dt);
void launch_norm_partials3(Ctx& c, double dt, int nb);

struct LinResult {
  bool converged = false;
  int iterations = 0;
  double rhs_norm = 0, final_residual_norm = 0;
  bool finite = true;
  int backend = 0;             // 0: CPR-FGMRES, 1: direct LU
  bool used_fallback = false;  // the direct LU did not converge and CPR-FGMRES ran instead
};

// Well Schur elimination + CPR-FGMRES on the reduced system + recovery.  Reads d_res/d_res_tail
// (rhs = -residual) and the assembled Jacobian; writes the reduced solution into d_x and the
// tail solution into h_dx_tail (n_wells + n_perfs).
LinResult linear_solve_full(Ctx& c, std::vector<double>& h_dx_tail);
// Well Schur elimination of the assembled system: d_val becomes the reduced matrix
// S = A - B D^-1 C (fill added into the well cliques), d_tinv the per-well dense D^-1 and d_rhs_red
// the reduced right-hand side of rhs = -residual.
void schur_eliminate(Ctx& c);
// CPR-FGMRES on an already assembled tail-free system: rhs in d_rhs_red, solution in d_x.
// rebuild = false reuses the CPR factors of the previous call on the same matrix.
LinResult linear_solve_reduced(Ctx& c, bool rebuild = true);

// Accurate solve of the tail-free system in d_val: x = A^-1 b to |b - A x| <= rtol |b| by
// iterative refinement over the inner solve (at most max_passes inner solves; the direct LU for
// systems of at most 512 rows when allow_direct, else CPR-FGMRES).  b and x are device vectors of
// 3N (not d_rhs_red / d_x, which the inner solves use).
LinResult solve_reduced_accurate(Ctx& c, const double* b, double* x, double rtol, int max_passes,
                                 bool allow_direct = true);

// Discrete adjoint kernels (rf_adjoint.cu)
void adj_transpose(Ctx& c, const int* d_tpos);
void adj_accum(Ctx& c, const double* lam_next, double* out);
void adj_grad(Ctx& c, double dt, const double* kx, const double* ky, const double* kz, const double* dz,
              const double* lam, double* grad);
void adj_add_at(Ctx& c, const std::vector<int>& idx, const std::vector<double>& v, double* out, int* d_idx);
void adj_gather_at(Ctx& c, const std::vector<int>& idx, const double* v, std::vector<double>& out, int* d_idx);

// Direct route for systems of at most kDirectSolveRows rows (fim/linear/mod.rs:15, 262-300).
// Rows of the system the route would factor: the full Newton system (with_wells) or the
// tail-free cell system.
int direct_rows(const Ctx& c, bool with_wells);
// Dense LU with partial pivoting on one thread-block cluster, then one solve and at most two
// refinement solves (sparse_lu_debug.rs:148-232).  with_wells: the full system from the assembled
// Jacobian, rhs = -residual, tail solution into *h_dx_tail; otherwise the tail-free system in
// d_val / d_rhs_red.  The cell solution goes to d_x.  Not converged when a pivot is zero or the
// residual stays above 1e-12 + 5e-3 |b|.
LinResult linear_solve_direct(Ctx& c, bool with_wells, std::vector<double>* h_dx_tail);

// Discrete adjoint tape hooks of the outer controller (rf_adjoint.cu); no-ops unless recording.
void adjoint_on_step_begin(Ctx& c);
void adjoint_on_substep_accepted(Ctx& c, double dt);
void adjoint_free(Ctx& c);

// Build-once helpers
void build_levels(Ctx& c);
void setup_linear_workspace(Ctx& c);
// 0: FP64 throughout; 1: FP32 block-ILU0 factors, FP32 pressure stage, FP64 FGMRES.
void set_linear_precision(Ctx& c, int mode);
// CTAs of the cluster that runs the level-scheduled kernels: the largest launchable power of two
// <= want (1..16); returns it.
int set_cluster_size(Ctx& c, int want);
int auto_cluster_size(const Ctx& c);
// Raise a kernel's dynamic shared-memory limit (never lowers it: the limit is shared by every
// context in the process).
void raise_dynamic_smem(const void* fn, size_t bytes);

// Single-CTA level-order kernels (rf_level.cu): structure of the current pattern (once per
// topology), launch shapes after a thread-count change, whether they serve the pressure stage and
// the block-ILU0 sweep at the current precision, packing of the pressure factors after each
// factorisation, and the solves.
void build_level_plan(Ctx& c);
void free_level_plan(Ctx& c);
void level_plan_reshape(Ctx& c);
bool level_solver_active(const Ctx& c);
bool level_block_sweep_active(const Ctx& c);
void level_pack(Ctx& c);
void launch_bicgstab_level(Ctx& c, const double* rhs, double* x);
void launch_block_sweep_level(Ctx& c, const double* cr, double* x, const void* lu, const void* dinv);

}  // namespace rf
