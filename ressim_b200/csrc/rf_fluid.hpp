// rf_fluid.hpp — the kernels' fluid, rock and SCAL parameters (`Fluid`) from the C ABI deck,
// including the flat PVT table of the three-phase mode.  Shared by the context set-up and the
// host build of the row functions that the CPU tests check against the oracle.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/ressim_fim.h"
#include "rf_blackoil.cuh"

namespace rf {

// Fills f from the deck; h_pvt receives the flat PVT table and f.pvt points at it (host memory).
inline int fluid_from_deck(const RfDeck* d, Fluid& f, std::vector<double>& h_pvt, std::string& err) {
  f = Fluid{};
  f.mu_o = d->mu_o;
  f.mu_w = d->mu_w;
  f.c_o = d->c_o;
  f.c_w = d->c_w;
  f.rho_o = d->rho_o;
  f.rho_w = d->rho_w;
  f.rho_g = 10.0;
  f.b_o = d->b_o;
  f.b_w = d->b_w;
  f.p_wref = d->water_pvt_reference_pressure_bar;
  f.c_r = d->rock_compressibility;
  f.p_rref = d->rock_reference_pressure_bar;
  f.gravity = d->gravity_enabled;
  f.s_wc = d->s_wc;
  f.s_or = d->s_or;
  f.n_w = d->n_w;
  f.n_o = d->n_o;
  f.krw_max = d->k_rw_max;
  f.kro_max = d->k_ro_max;
  f.table_points = d->corey_table_points;
  if (f.table_points > kMaxKnots) {
    err = "corey_table_points above 64 is not supported";
    return RF_ERR_UNSUPPORTED;
  }
  f.pc_entry = d->pc_entry;
  f.pc_lambda = d->pc_lambda;
  fill_knots(f);
  if (d->three_phase_mode) {
    f.three_phase = 1;
    f.drsdt0 = d->gas_redissolution_enabled ? 0 : 1;
    f.rho_g = d->rho_g;
    f.mu_g = d->mu_g;
    f.inject_gas = d->injected_fluid == 1;
    f.has_scal3 = d->has_scal_3p != 0;
    f.s3_wc = d->s_wc_3p;
    f.s3_or = d->s_or_3p;
    f.s3_nw = d->n_w_3p;
    f.s3_no = d->n_o_3p;
    f.s3_krw = d->k_rw_max_3p;
    f.s3_kro = d->k_ro_max_3p;
    f.s3_gc = d->s_gc;
    f.s3_gr = d->s_gr;
    f.s3_org = d->s_org;
    f.s3_ng = d->n_g;
    f.s3_krg = d->k_rg_max;
    f.has_pc_og = d->has_pc_og != 0;
    f.pcog_entry = d->pc_og_entry;
    f.pcog_lambda = d->pc_og_lambda;
    // PvtTable::new + build_oil_branches (pvt.rs:86-135): consecutive rows of one Rs with
    // non-decreasing p form an undersaturated branch; branches sorted by Rs, rows by p (stable);
    // the saturated curve is each branch's first row, sorted by p
    struct Branch {
      double rs;
      std::vector<std::array<double, 6>> rows;
    };
    std::vector<Branch> br;
    for (int r = 0; r < d->n_pvt_rows; ++r) {
      std::array<double, 6> row;
      for (int e = 0; e < 6; ++e) row[e] = d->pvt_rows[6 * size_t(r) + e];
      if (!br.empty()) {
        Branch& b = br.back();
        const bool same_rs = std::fabs(row[1] - b.rs) <= kPvtoRsTol;
        const bool higher = b.rows.empty() ? true : row[0] >= b.rows.back()[0] - 1e-9;
        if (same_rs && higher) {
          b.rows.push_back(row);
          continue;
        }
      }
      br.push_back(Branch{row[1], {row}});
    }
    for (Branch& b : br)
      std::stable_sort(b.rows.begin(), b.rows.end(), [](const auto& a, const auto& z) { return a[0] < z[0]; });
    std::stable_sort(br.begin(), br.end(), [](const Branch& a, const Branch& z) { return a.rs < z.rs; });
    std::vector<std::array<double, 6>> sat;
    for (const Branch& b : br)
      if (!b.rows.empty()) sat.push_back(b.rows.front());
    std::stable_sort(sat.begin(), sat.end(), [](const auto& a, const auto& z) { return a[0] < z[0]; });
    h_pvt.clear();
    for (const auto& r : sat) h_pvt.insert(h_pvt.end(), r.begin(), r.end());
    f.pvt_n_sat = int(sat.size());
    f.pvt_n_br = int(br.size());
    f.pvt_hdr = int(h_pvt.size());
    int first = 0;
    for (const Branch& b : br) {
      h_pvt.push_back(b.rs);
      h_pvt.push_back(double(first));
      h_pvt.push_back(double(b.rows.size()));
      first += int(b.rows.size());
    }
    f.pvt_rows = int(h_pvt.size());
    for (const Branch& b : br)
      for (const auto& r : b.rows) h_pvt.insert(h_pvt.end(), r.begin(), r.end());
    f.pvt_c_o = d->pvt_c_o;
    // SWOF / SGOF tables (relperm.rs:43-122), appended to the same flat array
    if (d->n_swof_rows > 0 || d->n_sgof_rows > 0) {
      if (!f.has_scal3 || d->n_swof_rows < 2 || d->n_sgof_rows < 2 || !d->swof_rows || !d->sgof_rows) {
        err = "SWOF/SGOF tables need the three-phase relperm props and at least two rows each";
        return RF_ERR_INVALID;
      }
      const double* tabs[2] = {d->swof_rows, d->sgof_rows};
      const int counts[2] = {d->n_swof_rows, d->n_sgof_rows};
      const char* names[2] = {"SWOF", "SGOF"};
      int offs[2];
      for (int t = 0; t < 2; ++t) {
        double prev = -INFINITY;
        for (int r = 0; r < counts[t]; ++r) {
          const double* v = tabs[t] + 3 * size_t(r);
          if (!(std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2])) || v[0] < 0.0 || v[0] > 1.0 ||
              v[1] < 0.0 || v[1] > 1.0 || v[2] < 0.0 || v[2] > 1.0 || v[0] <= prev) {
            err = std::string(names[t]) + " row " + std::to_string(r) +
                  " must hold finite values within [0, 1] with strictly increasing saturation";
            return RF_ERR_INVALID;
          }
          prev = v[0];
        }
        offs[t] = int(h_pvt.size());
        h_pvt.insert(h_pvt.end(), tabs[t], tabs[t] + 3 * size_t(counts[t]));
      }
      f.swof_off = offs[0];
      f.n_swof = counts[0];
      f.sgof_off = offs[1];
      f.n_sgof = counts[1];
    }
    f.pvt = h_pvt.data();
  }
  return RF_OK;
}

}  // namespace rf
