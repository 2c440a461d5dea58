/*
 * ressim_fim.h — C ABI of the B200-native fully implicit (FIM) Newton step.
 *
 * This is the drop-in boundary under the simulator's step API.  Every entry point takes plain
 * pointers and sizes and returns an int32_t status (0 ok, >0 recoverable solver status, <0 usage
 * or device error).  rf_create and rf_batch_create allocate the context's device buffers (freed
 * by rf_destroy / rf_batch_destroy); the other entry points work in those buffers and in the
 * caller's memory.  A context owns one CUDA stream and its device buffers; calls on one context
 * must be serialised by the caller (the reference simulator object is `&mut self`, single
 * threaded).
 *
 * Units follow the reference (bar, m, day, mD, cP).  Cell order is natural:
 * idx = k*nx*ny + j*nx + i (src/lib/ressim/src/grid.rs:25-27).
 */
#ifndef RESSIM_FIM_H
#define RESSIM_FIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RF_ABI_VERSION 4

/* status codes */
#define RF_OK 0
#define RF_STEP_WARNING 1        /* step finished with a solver warning (dt collapse, retry budget) */
#define RF_ERR_INVALID (-1)      /* invalid argument or deck */
#define RF_ERR_UNSUPPORTED (-2)  /* deck uses a feature the device path does not implement */
#define RF_ERR_CUDA (-3)         /* CUDA runtime error */
#define RF_ERR_DEVICE_STATUS (-4)/* a device-side check reported failure (reserved) */

/* linear-solver precision modes (rf_set_linear_precision) */
#define RF_PRECISION_FP64 0
#define RF_PRECISION_MIXED 1

/* One completion entry (src/lib/ressim/src/well.rs:64-90).  Entries that share a physical well
 * id (or, when none is given, the legacy fingerprint injector/i/j/bhp/radius/skin) form one
 * physical well (src/lib/ressim/src/fim/wells.rs:544-594). */
typedef struct RfWell {
  int32_t i, j, k;
  int32_t injector;          /* 1 injector, 0 producer */
  int32_t physical_well_id;  /* >= 0 explicit id; -1 legacy fingerprint grouping */
  int32_t has_schedule;      /* 1: explicit per-well schedule below (WellSchedule) */
  int32_t schedule_enabled;
  int32_t schedule_control;  /* 0 none, 1 pressure, 2 rate */
  double bhp;                /* BHP target / last accepted BHP [bar] */
  double well_radius;        /* [m] */
  double skin;
  double schedule_target_rate;         /* NaN: none */
  double schedule_target_surface_rate; /* NaN: none */
  double schedule_bhp_limit;           /* NaN: none */
  double datum_depth_m;                /* NaN: shallowest completion */
  double wellbore_density_kg_m3;       /* NaN: derived from completions */
} RfWell;

/* Static deck: grid, rock, fluid, SCAL, wells and controls.  Mirrors the fields of
 * ReservoirSimulator (src/lib/ressim/src/lib.rs:93-217) that the FIM path reads. */
typedef struct RfDeck {
  int32_t abi_version;
  int32_t nx, ny, nz;
  double dx, dy;
  const double* dz;        /* [nz] */
  const double* porosity;  /* [N] */
  const double* perm_x;    /* [N] mD */
  const double* perm_y;    /* [N] mD */
  const double* perm_z;    /* [N] mD */
  /* fluid (FluidProperties + rock properties) */
  double mu_o, mu_w, c_o, c_w, rho_o, rho_w;
  double b_o, b_w;
  double water_pvt_reference_pressure_bar;
  double rock_compressibility;
  double rock_reference_pressure_bar;
  double depth_reference_m;
  int32_t gravity_enabled;
  /* two-phase Corey SCAL (RockFluidProps) and the FIM relperm table knot count */
  double s_wc, s_or, n_w, n_o, k_rw_max, k_ro_max;
  int32_t corey_table_points;
  /* oil-water capillary pressure (Brooks-Corey, capped at 20x entry) */
  double pc_entry, pc_lambda;
  /* wells and family controls (src/lib/ressim/src/fim/wells.rs:691-798) */
  int32_t n_wells;
  const RfWell* wells;
  int32_t injector_rate_controlled;
  int32_t producer_rate_controlled;
  int32_t injector_enabled;
  double target_injector_rate_m3_day;
  double target_producer_rate_m3_day;
  double target_injector_surface_rate_m3_day; /* NaN: none */
  double target_producer_surface_rate_m3_day; /* NaN: none */
  double well_bhp_min, well_bhp_max;
  /* three-phase black-oil mode (setThreePhaseModeEnabled, frontend.rs:1088-1241) */
  int32_t three_phase_mode;
  int32_t injected_fluid; /* 0 water, 1 gas (the reference's default); water in two-phase mode */
  /* PVT table (setPvtTable, pvt.rs:36-104): n_pvt_rows rows of six doubles in input order,
   * p [bar], Rs [Sm3/Sm3], Bo, mu_o [cP], Bg, mu_g [cP]; the table's undersaturated oil
   * compressibility is pvt_c_o (the fluid c_o when the table was set) */
  int32_t n_pvt_rows;
  const double* pvt_rows;
  double pvt_c_o;
  /* three-phase Corey SCAL (setThreePhaseRelPermProps, relperm.rs:199-228); has_scal_3p = 0
   * keeps the two-phase curves and an immobile gas phase */
  int32_t has_scal_3p;
  double s_wc_3p, s_or_3p, n_w_3p, n_o_3p, k_rw_max_3p, k_ro_max_3p;
  double s_gc, s_gr, s_org, n_g, k_rg_max;
  /* gas-oil capillary pressure (setGasOilCapillaryParams, capillary.rs:100-172) */
  int32_t has_pc_og;
  double pc_og_entry, pc_og_lambda;
  /* gas properties (setGasFluidProperties) and redissolution (setGasRedissolutionEnabled) */
  double mu_g, c_g, rho_g;
  int32_t gas_redissolution_enabled;
  /* SWOF / SGOF tables (setThreePhaseScalTables, relperm.rs:43-122): rows of three doubles,
   * (sw, krw, krow) and (sg, krg, krog), at least two each with strictly increasing saturations;
   * when present they replace the three-phase Corey curves (relperm.rs:391-429) and need
   * has_scal_3p.  The tables' capillary-pressure columns are not read by the FIM path. */
  int32_t n_swof_rows;
  const double* swof_rows;
  int32_t n_sgof_rows;
  const double* sgof_rows;
} RfDeck;

/* Per-report-step outcome (FimStepStats subset, src/lib/ressim/src/reporting.rs:191-243). */
typedef struct RfStepReport {
  int32_t substeps;             /* accepted substeps */
  int32_t retries;              /* failed Newton attempts */
  int32_t newton_iterations;    /* summed over accepted and failed attempts */
  int32_t linear_iterations;    /* summed FGMRES iterations */
  int32_t linear_solves;
  int32_t warning;              /* 0 none, 1 dt collapse, 2 retry budget, 3 max substeps */
  double time_days;             /* simulator time after the step */
  double advanced_days;
  double last_dt_days;
  double device_ms;             /* device time of the step measured with CUDA events */
} RfStepReport;

/* One accepted-substep rate record (TimePointRates subset, reporting.rs:246-291). */
typedef struct RfTimePointRates {
  double time;
  double total_production_oil;
  double total_production_liquid;
  double total_production_liquid_reservoir;
  double total_injection;
  double total_injection_reservoir;
  double material_balance_error_m3;
  double material_balance_error_oil_m3;
  double avg_reservoir_pressure;
  double avg_water_saturation;
  double producer_bhp_limited_fraction;
  double injector_bhp_limited_fraction;
  /* three-phase mode (zero otherwise): surface gas produced per day (free plus dissolved), the
   * mean gas saturation, the cumulative gas material-balance error [Sm3] and the producing GOR */
  double total_production_gas;
  double avg_gas_saturation;
  double material_balance_error_gas_m3;
  double producing_gor;
} RfTimePointRates;

/* Linear-solve report (FimLinearSolveReport, src/lib/ressim/src/fim/linear/mod.rs:213-230).
 * backend: RF_BACKEND_FGMRES_CPR or RF_BACKEND_SPARSE_LU (`backend_used`); used_fallback: the
 * direct LU of a system of at most 512 rows did not converge and CPR-FGMRES ran instead. */
#define RF_BACKEND_FGMRES_CPR 0
#define RF_BACKEND_SPARSE_LU 1
typedef struct RfLinearReport {
  int32_t converged;
  int32_t iterations;
  double rhs_norm;
  double final_residual_norm;
  int32_t used_fallback;
  int32_t backend;
} RfLinearReport;

typedef struct RfCtx RfCtx;

/* Replaces ReservoirSimulator::new + setters (src/lib/ressim/src/frontend.rs:36-123): copies
 * the deck to the device on the current CUDA device. */
int32_t rf_create(const RfDeck* deck, RfCtx** out);
int32_t rf_destroy(RfCtx* ctx);

/* Message of the last error on this context (or the last rf_create failure when ctx is NULL). */
int32_t rf_last_error(const RfCtx* ctx, char* buf, size_t len);

/* Replaces loadState's grid/well payload (frontend.rs:931-1008).  sg and rs may be NULL in
 * two-phase mode. */
int32_t rf_set_state(RfCtx* ctx, const double* pressure, const double* sat_water,
                     const double* sat_gas, const double* rs, double time_days);
/* Replaces getPressures/getSatWater/getSatOil/getSatGas/getRs (frontend.rs:523-605); any
 * output pointer may be NULL. */
int32_t rf_get_state(const RfCtx* ctx, double* pressure, double* sat_water, double* sat_oil,
                     double* sat_gas, double* rs, double* time_days);
/* Current BHP of every completion entry (getWellState's `bhp`). */
int32_t rf_get_well_bhp(const RfCtx* ctx, double* bhp, int32_t n);

/* Replaces ReservoirSimulator::step (frontend.rs:345-349 -> fim/timestep.rs:989-1848): one
 * report step of the OPM-aligned FIM controller, Newton iterations on the device. */
int32_t rf_step(RfCtx* ctx, double target_dt_days, RfStepReport* out);

/* getRateHistory (frontend.rs:562-565): number of records and one record. */
int32_t rf_rate_history_len(const RfCtx* ctx);
int32_t rf_rate_history_get(const RfCtx* ctx, int32_t index, RfTimePointRates* out);

/* Linear-solver seam replacing solve_linearized_system for a tail-free system
 * (src/lib/ressim/src/fim/linear/mod.rs:252-300): CPR-FGMRES with block-ILU0 on a 3x3 block
 * CSR matrix given on the host (block row pointers, block columns, row-major 3x3 values).  A
 * system of at most 512 rows goes to the dense direct LU first, as the reference's routing does. */
int32_t rf_linear_solve_bsr(RfCtx* ctx, int32_t n_block_rows, const int32_t* block_row_ptr,
                            const int32_t* block_cols, const double* block_vals,
                            const double* rhs, double* x, RfLinearReport* out);

/* Linear-solver seam replacing solve_linearized_system for the full Newton system with its well
 * tail (src/lib/ressim/src/fim/linear/mod.rs:252-300, tail elimination well_schur.rs:70-471):
 * a scalar CSR matrix (the reference's CsMat) of n_rows = 3 cells + wells + perforations rows in
 * FimLinearBlockLayout order (cells, then one BHP per physical well, then one rate per
 * perforation, in this context's well and perforation order).  Entries are accumulated into the
 * device's Newton-system storage: a cell block outside the stencil-plus-well pattern, a tail entry
 * that is not one of a well's couplings (a perforation row to its own cell, BHP and rate; a
 * control row to its well's BHP, perforation rates and perforated cells; a cell row to the rates
 * of its own perforations), or a perforation diagonal other than 1 (0 without a well index) is
 * rejected with RF_ERR_INVALID, explicit zeros excepted.  Systems of at most 512 rows go to the
 * dense direct LU first; otherwise the wells are eliminated, the reduced system is solved by
 * CPR-FGMRES and the tail recovered, exactly as inside rf_step.  x receives n_rows values. */
int32_t rf_linear_solve_csr(RfCtx* ctx, int32_t n_rows, const int32_t* row_ptr, const int32_t* cols,
                            const double* vals, const double* rhs, double* x, RfLinearReport* out);

/* Precision of the CPR-FGMRES linear solver.  RF_PRECISION_FP64 (default) computes everything in
 * FP64, as the reference does.  RF_PRECISION_MIXED keeps the block-ILU0 factors, the pressure
 * matrix, its ILU0 factors and the pressure BiCGStab vectors in FP32 (dot products accumulate in
 * FP64), under the FP64 FGMRES; residuals, the well Schur complement, Gram-Schmidt and the Newton
 * update stay FP64.  No counterpart in the reference (an extension of the device path); takes
 * effect at the next linear solve. */
int32_t rf_set_linear_precision(RfCtx* ctx, int32_t mode);

/* Tuning: CTAs (1..16, rounded down to a launchable power of two) in the thread-block cluster that
 * runs the level-scheduled ILU factorisation, ILU sweeps and pressure BiCGStab; 0 restores the
 * automatic choice (enough 1024-thread CTAs for the widest level).  Returns the size in use (> 0)
 * or an error.  The size fixes the reduction order, so results are deterministic for a given size
 * and differ between sizes only by rounding.  No counterpart in the reference. */
int32_t rf_set_cluster_size(RfCtx* ctx, int32_t ctas);

/* Tuning: the kernels of the CPR's level-scheduled solves (the pressure BiCGStab with pressure
 * ILU0, and the block-ILU0 sweep).  RF_PRESSURE_SOLVER_CLUSTER runs them on the thread-block
 * cluster of rf_set_cluster_size; RF_PRESSURE_SOLVER_LEVEL runs each as one thread block with its
 * vectors in level order and the sweeps' dependencies in shared memory (`threads` threads,
 * 32..512 in steps of 32, 0 automatic); RF_PRESSURE_SOLVER_AUTO (default) takes the level-order
 * kernels, where their level window fits shared memory, for decks of up to 32,768 cells and for
 * every variant of an ensemble stepped in RF_BATCH_GROUPS mode, and the cluster kernels otherwise.  Both compute the same preconditioner;
 * the solves differ only in the summation order of their dot products.  Takes effect at the next
 * linear solve; RF_ERR_UNSUPPORTED when the level-order kernels cannot run this deck.  No
 * counterpart in the reference. */
#define RF_PRESSURE_SOLVER_AUTO 0
#define RF_PRESSURE_SOLVER_CLUSTER 1
#define RF_PRESSURE_SOLVER_LEVEL 2
int32_t rf_set_pressure_solver(RfCtx* ctx, int32_t kind, int32_t threads);

/* Number of kernel launches this context has issued since creation (device work counter). */
int64_t rf_kernel_launches(const RfCtx* ctx);

/* Phase timing (FimStepStats' assembly / preconditioner / linear-solve / update split,
 * src/lib/ressim/src/reporting.rs:191-243) measured with CUDA events on the context's stream.
 * out (may be NULL) receives up to n values, read before the enable/reset below take effect:
 * ms for assembly, well elimination, CPR build, pressure stage, block-ILU0 smoother, Krylov,
 * update, the BiCGStab kernel alone, the direct LU route; then the BiCGStab iteration total, the number of BiCGStab
 * launches timed, the block count of the reduced matrix, and 1 when the level-order kernels serve
 * the pressure stage (0: the cluster kernels).
 * enable > 0 switches the profiler on, 0 off, < 0 leaves it as is; reset != 0 zeroes the totals. */
int32_t rf_profile(RfCtx* ctx, int32_t enable, int32_t reset, double* out, int32_t n);

/* Controller options; no counterpart in the reference (whose controller picks substeps by its
 * PID rule and accepts by its CNV/MB tiers).  one_substep_per_report_step != 0 takes every report
 * step as exactly one substep of the full dt, without retries (a Newton failure ends the step with
 * a warning); cnv_tol > 0 replaces the CNV tiers with this one tolerance (and mb_tol > 0 the MB
 * ones), without the pore-volume relaxation.  Both make the converged states smooth functions of
 * the inputs, which finite-difference checks of the adjoint need.  Defaults: 0, 0, 0. */
int32_t rf_set_controller_options(RfCtx* ctx, int32_t one_substep_per_report_step, double cnv_tol, double mb_tol);

/* Linear refinement; no counterpart in the reference (whose Newton systems get one CPR-FGMRES
 * solve to 1e-12 + 5e-3 |b|, fim/linear/mod.rs:252-372).  rtol > 0 refines every CPR-FGMRES solve
 * of the well-eliminated system: x += solve(b - A x), the CPR factors of the first pass reused,
 * until |b - A x| <= rtol |b| or max_passes solves (0: 12).  With a tight rtol the Newton iterates
 * no longer depend on the preconditioner's rounding, so two implementations take the same Newton
 * path; with tight CNV / MB tolerances (rf_set_controller_options) this is the matched profile
 * used to compare against other implementations at 1e-6.  The direct route for systems of at most
 * 512 rows is unchanged.  rtol = 0 (default) restores the reference's single solve.  The first
 * call with rtol > 0 allocates two vectors of 3 x cells doubles. */
int32_t rf_set_linear_refinement(RfCtx* ctx, double rtol, int32_t max_passes);

/* ---- Discrete adjoint (no counterpart in the reference, which has no adjoint).
 * rf_adjoint_record(ctx, 1) clears the tape and starts recording: every later rf_step checkpoints
 * the simulator state at its start (p, Sw; So, Sg, Rs in three-phase mode; device copies) and
 * keeps the dt of each accepted substep.  rf_adjoint_record(ctx, 0) stops recording.
 * rf_backward runs the backward pass over the recorded report steps: each report step is replayed
 * from its checkpoint (same substeps, same converged states), then the transposed Newton systems
 * are solved in reverse time (well Schur complement transposed, CPR-FGMRES with iterative
 * refinement to 1e-11 relative).  It returns the objective value, its gradient with respect to
 * the log of each cell's permeability multiplier (kx, ky, kz scaled together; n_cells values) and
 * with respect to each physical well's active control (its target rate when rate controlled, its
 * BHP target otherwise; physical wells in order of first appearance, rf_well_count of them).  The
 * substep sizes are held fixed.  The simulator state is left as it was. */
#define RF_OBJECTIVE_CUMULATIVE_OIL 0 /* surface oil produced by the producers' connections [Sm3] */
typedef struct RfObjective {
  int32_t kind;
} RfObjective;
int32_t rf_adjoint_record(RfCtx* ctx, int32_t enable);
int32_t rf_backward(RfCtx* ctx, const RfObjective* objective, double* value, double* dJ_dlnk, double* dJ_dcontrols,
                    int32_t n_controls);
int32_t rf_well_count(const RfCtx* ctx);

/* ---- Dense pressure solve that allocates nothing.  No counterpart in the reference.  It is the
 * dense coarse solve of the CPR pressure stage, offered alone for callers that may not call
 * cudaMalloc (a host that reserves its device memory up front for its own pool, an embedding
 * framework that owns the allocator, a loop that must not block on an allocation).
 * x = A^{-1} b, A dense row-major n x n; a, b and x are device memory owned by the caller; the
 * call runs on `stream` (a cudaStream_t, NULL for the default stream) and synchronises it before
 * returning, so it may not be called while that stream is being captured into a CUDA graph.
 * n must lie in 1..RF_NOALLOC_MAX_ROWS, otherwise RF_ERR_INVALID.  An exactly zero pivot returns
 * RF_ERR_INVALID ("singular") and leaves x unchanged.  Its scratch is one fixed device array of
 * about 1.4 MB that every GPU loading the library keeps until exit; the first call on a device
 * looks up that array's address.  Calls share the array: calls that overlap on the GPU race.  On
 * failure a message is written to err (may be NULL, err_len bytes). */
#define RF_NOALLOC_MAX_ROWS 299
int32_t rf_dense_solve_noalloc(int32_t n, const double* a, const double* b, double* x, void* stream,
                               char* err, size_t err_len);

/* ---- Ensemble batch (sensitivity variants of uneven sizes); no counterpart in the reference, whose
 * simulator object steps one deck.  Each variant gets its own context (the rf_* calls above work on
 * rf_batch_context(b, i)); rf_batch_step advances every variant by one report step, driving the
 * variants from `host_threads` host threads (<= 0: max(32, hardware threads), at most n) so their
 * kernels run concurrently on the device (see rf_batch_set_mode).  Set the environment variable
 * CUDA_DEVICE_MAX_CONNECTIONS=32 before CUDA initialises in the process: with the default of 8
 * hardware queues the variants' streams alias and short kernels wait behind long pressure solves
 * (the Python package sets it on import).  Returns the first negative
 * status of any variant, else the largest positive one; per-variant reports go to reports[n]. */
typedef struct RfBatch RfBatch;
int32_t rf_batch_create(const RfDeck* const* decks, int32_t n, int32_t host_threads, RfBatch** out);
int32_t rf_batch_destroy(RfBatch* batch);
int32_t rf_batch_size(const RfBatch* batch);
RfCtx* rf_batch_context(RfBatch* batch, int32_t index);
int32_t rf_batch_step(RfBatch* batch, double target_dt_days, RfStepReport* reports);

/* How rf_batch_step drives the variants.  RF_BATCH_GROUPS (the default after rf_batch_create): the
 * variants are split into `host_threads` groups with one host thread and one CUDA stream each;
 * every variant's report step runs as a fiber on its group's thread, suspended instead of blocked
 * while its stream works, and the group's ILU0 factorisations, pressure BiCGStab solves and
 * block-ILU0 sweeps are issued as one batched launch per kind (thread block b runs variant b's solve), so far more solves run at
 * once than there are hardware queues.  RF_BATCH_THREADS: one stream per variant and a pool of
 * host threads stepping one variant at a time.  A variant's results do not depend on the mode.
 * No counterpart in the reference. */
#define RF_BATCH_GROUPS 0
#define RF_BATCH_THREADS 1
int32_t rf_batch_set_mode(RfBatch* batch, int32_t mode);
/* Batched-launch statistics of RF_BATCH_GROUPS (CUDA events on the groups' streams while enabled):
 * out (may be NULL) receives up to n values, read before enable/reset take effect: the group
 * count, then per kind (pressure BiCGStab, block-ILU0 sweep, ILU0 factorisation) the launches,
 * the solves they carried and their device ms.  enable > 0 switches the timing on, 0 off, < 0 leaves it; reset
 * != 0 zeroes the totals. */
int32_t rf_batch_profile(RfBatch* batch, int32_t enable, int32_t reset, double* out, int32_t n);

#ifdef __cplusplus
}
#endif

#endif /* RESSIM_FIM_H */
