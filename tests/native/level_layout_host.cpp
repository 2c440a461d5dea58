// Host build of the level-order pressure solve's layout (ressim_b200/csrc/rf_level_layout.hpp) for
// the CPU tests: every bulk copy the staging issues must start and end on 16-byte boundaries, stay
// inside its source array and fit its shared-memory slot.  The checks replay, for both value types,
// the copies of every level placement (first position lst, width w <= W) of position arrays of n
// values, as the kernel's issue step forms them.
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "../../ressim_b200/csrc/rf_level_layout.hpp"

namespace {

template <class T>
bool check_type(int n, int W, char* err, size_t len) {
  using rf::BRec;
  using rf::FRec;
  constexpr int E = 16 / int(sizeof(T));
  const size_t np = rf::lvl_work_pad(n);
  const size_t in_bytes = rf::lvl_in_bytes<T>(W), slot = rf::lvl_slot_bytes<T>(W);
  const size_t in_off = size_t(W) * sizeof(BRec<T>);
  auto fail = [&](const char* what, int lst, int w) {
    std::snprintf(err, len, "T=%zuB n=%d W=%d lst=%d w=%d: %s", sizeof(T), n, W, lst, w, what);
    return false;
  };
  if (sizeof(FRec<T>) % 16 || sizeof(BRec<T>) % 16) return fail("record size not a multiple of 16", 0, 0);
  if (slot % 16 || in_off % 16 || in_bytes % 16) return fail("slot offsets not 16-byte aligned", 0, 0);
  // the scratch vectors: the iterate (double) first, then nine of type T, each np values
  if ((sizeof(double) * np) % 16 || (sizeof(T) * np) % 16) return fail("scratch vector base unaligned", 0, 0);
  for (int w = 1; w <= W; ++w)
    for (int lst = 0; lst + w <= n; ++lst) {
      const size_t rb[2] = {size_t(w) * sizeof(FRec<T>), size_t(w) * sizeof(BRec<T>)};
      const size_t rs[2] = {size_t(lst) * sizeof(FRec<T>), size_t(lst) * sizeof(BRec<T>)};
      for (int d = 0; d < 2; ++d) {
        if (rs[d] % 16 || rb[d] % 16) return fail("record copy unaligned", lst, w);
        if (rb[d] > in_off) return fail("records overflow the slot", lst, w);
        if (rs[d] + rb[d] > size_t(n) * (d ? sizeof(BRec<T>) : sizeof(FRec<T>)))
          return fail("record copy past the array", lst, w);
      }
      int a0, a1;
      rf::lvl_input_span(lst, w, E, a0, a1);
      const size_t ib = size_t(a1 - a0) * sizeof(T);
      if (a0 < 0 || a0 > lst || a1 < lst + w) return fail("input span misses the level", lst, w);
      if ((size_t(a0) * sizeof(T)) % 16 || ib % 16 || ib == 0) return fail("input copy unaligned", lst, w);
      if (size_t(a1) > np) return fail("input copy past the padded vector", lst, w);
      if (ib > in_bytes) return fail("input copy overflows its slot region", lst, w);
      // the last staged value read: shift + (w - 1), inside the copied span
      if (size_t(lst - a0 + w) * sizeof(T) > ib) return fail("staged index outside the copy", lst, w);
    }
  // the long rows' shared-memory copy
  const int cases[4][4] = {{0, 0, 0, 0}, {1, 2, 3, 5}, {17, 13, 211, 97}, {64, 64, 1000, 1000}};
  for (const auto& c : cases) {
    const rf::LvlLongLayout o = rf::lvl_long_layout<T>(rf::LvlArgsLong{c[0], c[1], c[2], c[3]});
    const size_t offs[6] = {o.fval, o.bval, o.fptr, o.bptr, o.fidx, o.bidx};
    for (size_t x : offs)
      if (x % 16) return fail("long-row layout offset unaligned", c[0], c[2]);
    if (o.bval < o.fval + size_t(c[2]) * sizeof(T) || o.fptr < o.bval + size_t(c[3]) * sizeof(T) ||
        o.bptr < o.fptr + (size_t(c[0]) + 1) * 4 || o.fidx < o.bptr + (size_t(c[1]) + 1) * 4 ||
        o.bidx < o.fidx + size_t(c[2]) * 2 || o.total < o.bidx + size_t(c[3]) * 2 || o.total % 16)
      return fail("long-row layout regions overlap", c[0], c[2]);
  }
  return true;
}

}  // namespace

extern "C" {

// Checks every level placement with widths up to W in arrays of n positions, for FP64 and FP32;
// returns 1 when all hold, else 0 with the first failure in err.
int32_t rfh_level_layout_check(int32_t n, int32_t W, char* err, size_t len) {
  if (len) err[0] = 0;
  return check_type<double>(n, W, err, len) && check_type<float>(n, W, err, len) ? 1 : 0;
}

}  // extern "C"
