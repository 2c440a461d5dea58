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

}  // namespace rf
