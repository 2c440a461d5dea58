// rf_state.hpp — host launchers for the per-cell update and substep reductions.
#pragma once

#include <vector>

#include "rf_context.hpp"

namespace rf {

// Chop, relax and apply the reduced solution in d_x to (d_p, d_sw, d_hc) -> (d_cp, d_csw, d_chc).
void apply_cell_update(Ctx& c, double relax, double& pmax, bool& finite);
// Sums over cells of (a = previous, b = current): [rel-change delta, rel-change denom, water
// inventory, oil inventory, sum p*pv, sum pv, sum sw].
void state_sums(Ctx& c, const double* ap, const double* asw, const double* ahc, const double* bp, const double* bsw,
                const double* bhc, double out[7]);
// (p, sw, hc) of every perforated cell, 3 values per perforation.
void gather_perf_cells(Ctx& c, const double* p, const double* sw, const double* hc, std::vector<double>& out);
// Final pass of a per-block (max p, non-finite flag) reduction left in d_partials by an update
// kernel of nb blocks.
void max2_final(Ctx& c, int nb, double& pmax, bool& finite);

// ---- three-phase black-oil mode (rf_blackoil.cu) ----
constexpr int kStateQ3 = 9;
// Chop and apply the update with the regimes' implied saturation changes.
void apply_cell_update3(Ctx& c, double relax, double& pmax, bool& finite);
// Substep start: regimes and the hc primary (d_reg, d_phc) from d_pp and the simulator's Sg, Rs.
void from_simulator3(Ctx& c);
// Write-back: the simulator's So, Sg, Rs (d_so, d_sg, d_rs) from (d_p, d_sw, d_hc, d_reg).
void derive3(Ctx& c);
// Relative change between cell states a and b (sharing d_reg), then inventories and reporting
// sums over the simulator arrays (sp, ssw with d_so, d_sg, d_rs): [delta, denom, water, oil,
// gas, sum p*pv, sum pv, sum sw, sum sg].
void state_sums3(Ctx& c, const double* ap, const double* asw, const double* ahc, const double* bp, const double* bsw,
                 const double* bhc, const double* sp, const double* ssw, double out[kStateQ3]);
// (a, b, c, regime) of every perforated cell, 4 values per perforation (reg may be null: 0).
void gather_perf_cells3(Ctx& c, const double* a, const double* b, const double* cc, const int* reg,
                        std::vector<double>& out);

}  // namespace rf
