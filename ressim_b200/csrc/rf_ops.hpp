// rf_ops.hpp — host launchers of the device kernels (assembly, norms, linear solve).
#pragma once

#include "rf_context.hpp"

namespace rf {

constexpr int kNormQuantities = 13;  // see k_norms_cells

void launch_assembly(Ctx& c, double dt);
// h_out receives kNormQuantities + 1 doubles (family maxima, FVF sums, CNV maxima, residual
// sums, pore-volume sum, violating pore volume).
void launch_norms(Ctx& c, double dt, double* h_out);

struct LinResult {
  bool converged = false;
  int iterations = 0;
  double rhs_norm = 0, final_residual_norm = 0;
  bool finite = true;
};

// Well Schur elimination + CPR-FGMRES on the reduced system + recovery.  Reads d_res/d_res_tail
// (rhs = -residual) and the assembled Jacobian; writes the reduced solution into d_x and the
// tail solution into h_dx_tail (n_wells + n_perfs).
LinResult linear_solve_full(Ctx& c, std::vector<double>& h_dx_tail);
// CPR-FGMRES on an already assembled tail-free system: rhs in d_rhs_red, solution in d_x.
LinResult linear_solve_reduced(Ctx& c);

// Build-once helpers
void build_levels(Ctx& c);
void setup_linear_workspace(Ctx& c);
// 0: FP64 throughout; 1: FP32 block-ILU0 factors, FP32 pressure stage, FP64 FGMRES.
void set_linear_precision(Ctx& c, int mode);
// CTAs of the cluster that runs the level-scheduled kernels: the largest launchable power of two
// <= want (1..16); returns it.
int set_cluster_size(Ctx& c, int want);
int auto_cluster_size(const Ctx& c);

}  // namespace rf
