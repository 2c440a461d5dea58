// Host build of the device path's three-phase row functions (ressim_b200/csrc/rf_blackoil_rows.cuh)
// for the CPU tests: the same source the kernels k_cells3 / k_perfs3 / k_wells3 run per thread,
// compiled by g++ with -ffp-contract=off (the oracle's flag), so that the tests compare the
// device path's residual and Jacobian rows with the oracle's assembly without a GPU.
#include <cstdint>
#include <string>
#include <vector>

#include "../../ressim_b200/csrc/rf_blackoil_rows.cuh"
#include "../../ressim_b200/csrc/rf_fluid.hpp"

extern "C" {

// Cells in natural order with a 7-slot block row each (blocks[(7 i + slot) * 9 + 3 e + v], slot
// order z-, y-, x-, diag, x+, y+, z+); prev / cur hold (p, sw, hc) per cell; ctrl holds 8 doubles
// per well (enabled, rate_controlled, uses_surface_target, has_target, injector, target_rate,
// bhp_limit, bhp_target).  res receives 3n + n_wells + n_perfs values (cells, then the well
// control rows, then the perforation rows).
int32_t rfh_assemble3(const RfDeck* deck, double dt, const double* tx, const double* ty, const double* tz,
                      const double* pv, const double* depth_layer, const int32_t* reg, const double* prev,
                      const double* cur, int32_t n_wells, int32_t n_perfs, const int32_t* perf_cell,
                      const int32_t* perf_inj, const int32_t* perf_well, const int32_t* perf_has_wi,
                      const double* perf_wi, const double* perf_head, const int32_t* well_ptr,
                      const int32_t* well_perfs, const double* ctrl, const double* bhp, const double* q, double* res,
                      double* blocks, double* jrw, double* jwr_perf, double* jww_perf_bhp, double* jwr_ctrl,
                      double* jww_ctrl_q, double* jww_ctrl_bhp, const double* base_rs) {
  rf::Fluid f;
  std::vector<double> pvt;
  std::string err;
  if (rf::fluid_from_deck(deck, f, pvt, err) != RF_OK) return RF_ERR_UNSUPPORTED;
  const int nx = deck->nx, ny = deck->ny, nz = deck->nz, n = nx * ny * nz, nxy = nx * ny;
  std::vector<double> p(n), sw(n), hc(n), pp(n), psw(n), phc(n);
  for (int i = 0; i < n; ++i) {
    p[i] = cur[3 * i];
    sw[i] = cur[3 * i + 1];
    hc[i] = cur[3 * i + 2];
    pp[i] = prev[3 * i];
    psw[i] = prev[3 * i + 1];
    phc[i] = prev[3 * i + 2];
  }
  std::vector<int> row_ptr(n + 1), stencil(7 * size_t(n), -1), diag(n);
  for (int i = 0; i < n; ++i) {
    row_ptr[i] = 7 * i;
    const int ci = i % nx, cj = (i / nx) % ny, ck = i / nxy;
    const bool has[7] = {ck > 0, cj > 0, ci > 0, true, ci + 1 < nx, cj + 1 < ny, ck + 1 < nz};
    for (int s = 0; s < 7; ++s)
      if (has[s]) stencil[7 * i + s] = 7 * i + s;
    diag[i] = 7 * i + rf::kDiag;
  }
  row_ptr[n] = 7 * n;
  for (size_t k = 0; k < 63 * size_t(n); ++k) blocks[k] = 0.0;
  for (int i = 0; i < n; ++i)
    rf::cell_row3(f, nx, ny, nz, i, dt, pv, tx, ty, tz, depth_layer, reg, p.data(), sw.data(), hc.data(), pp.data(),
                  psw.data(), phc.data(), row_ptr.data(), stencil.data(), res, blocks, base_rs);
  double* res_tail = res + 3 * size_t(n);
  for (int k = 0; k < n_perfs; ++k)
    rf::perf_row3(f, n_wells, k, dt, perf_cell, perf_inj, perf_well, perf_has_wi, perf_wi, perf_head, reg, p.data(),
                  sw.data(), hc.data(), bhp, q, diag.data(), res, blocks, res_tail, jrw, jwr_perf, jww_perf_bhp,
                  base_rs);
  for (int w = 0; w < n_wells; ++w) {
    const double* c = ctrl + 8 * w;
    const rf::WellControlH k{int(c[0]), int(c[1]), int(c[2]), int(c[3]), int(c[4]), c[5], c[6], c[7]};
    rf::well_row3(f, w, k, well_ptr, well_perfs, perf_cell, reg, p.data(), sw.data(), hc.data(), bhp, q, res_tail,
                  jwr_ctrl, jww_ctrl_q, jww_ctrl_bhp, base_rs);
  }
  return RF_OK;
}

// The cell flash and write-back of the device path (derive_cell3): out = (regime, so, sg, rs, bo, bg)
// per cell; and the substep-start classification (classify_regime) of (p, sg, rs).
int32_t rfh_derive3(const RfDeck* deck, int32_t n, const double* p, const double* sw, const double* hc,
                    const int32_t* reg, const double* base_rs, double* out) {
  rf::Fluid f;
  std::vector<double> pvt;
  std::string err;
  if (rf::fluid_from_deck(deck, f, pvt, err) != RF_OK) return RF_ERR_UNSUPPORTED;
  for (int i = 0; i < n; ++i) {
    const rf::Derived3 d = rf::derive_cell3(f, p[i], sw[i], hc[i], reg[i], base_rs[i]);
    const double o[6] = {double(d.regime), d.so, d.sg, d.rs, d.bo, d.bg};
    for (int e = 0; e < 6; ++e) out[6 * i + e] = o[e];
  }
  return RF_OK;
}
int32_t rfh_classify3(const RfDeck* deck, int32_t n, const double* p, const double* sg, const double* rs,
                      const double* base_rs, int32_t* reg) {
  rf::Fluid f;
  std::vector<double> pvt;
  std::string err;
  if (rf::fluid_from_deck(deck, f, pvt, err) != RF_OK) return RF_ERR_UNSUPPORTED;
  for (int i = 0; i < n; ++i) reg[i] = rf::classify_regime(f, p[i], sg[i], rs[i], base_rs[i]);
  return RF_OK;
}

}  // extern "C"
