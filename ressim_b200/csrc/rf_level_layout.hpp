// rf_level_layout.hpp — memory layout of the level-order pressure solve (rf_level.cu): the
// per-position records, the shared-memory staging ring and the long rows' shared-memory copy, and
// the span of an input vector that one level's bulk copy covers.  Host and device code share these
// definitions; the CPU tests compile them with g++ to check the bulk copies' alignment and bounds.
#pragma once

#include <cstddef>

#ifdef __CUDACC__
#define RF_LVL_HD __host__ __device__
#else
#define RF_LVL_HD
#endif

namespace rf {

// Per-position records of the pressure sweeps (rebuilt after each factorisation), copied into
// shared memory a level at a time: a 64-bit word with three dependency indices into the
// shared-memory array S (the two level windows, the far cache and a zero slot that absent entries
// point at, their factor value being 0) and a meta field (bits 0-2 entry count, 7 = long row whose
// index is the word's low 16 bits; bits 3-15 own far slot + 1), then the factor values in column
// order (and the pivot for the backward sweep).
template <class T>
struct alignas(16) FRec {
  unsigned long long word;
  T v[3];
};
template <class T>
struct alignas(16) BRec {
  unsigned long long word;
  T v[3];
  T piv;
};

RF_LVL_HD constexpr size_t lvl_up16(size_t x) { return (x + 15) / 16 * 16; }

// Bytes of one staged input vector: a level's W values plus the alignment slack at both ends
// (the copy runs from the 16-byte boundary below the level to the one above it), rounded to 16.
template <class T>
RF_LVL_HD constexpr size_t lvl_in_bytes(int W) {
  return lvl_up16((size_t(W) + 2 * (16 / sizeof(T))) * sizeof(T));
}
// Bytes of one staging slot: the level's records (room for the larger record type) and up to three
// input vectors.
template <class T>
RF_LVL_HD constexpr size_t lvl_slot_bytes(int W) {
  return size_t(W) * sizeof(BRec<T>) + 3 * lvl_in_bytes<T>(W);
}
// Bytes of the two level windows, the far cache and the zero slot.
template <class T>
RF_LVL_HD constexpr size_t lvl_win_bytes(int W, int nfar) {
  return lvl_up16((2 * size_t(W) + size_t(nfar) + 1) * sizeof(T));
}

// The values [a0, a1) of an input vector that the bulk copy of the level [lst, lst + w) covers:
// from the 16-byte boundary at or below lst to the one at or above lst + w (E values per 16 bytes).
RF_LVL_HD inline void lvl_input_span(int lst, int w, int E, int& a0, int& a1) {
  a0 = lst & ~(E - 1);
  a1 = (lst + w + E - 1) & ~(E - 1);
}

// Values per position-order vector of the solve's scratch: n rounded up to a multiple of 4, so every
// vector starts on a 16-byte boundary and a level's copy, rounded out, stays inside its vector.
inline size_t lvl_work_pad(int n) { return (size_t(n) + 3) / 4 * 4; }

// Counts of the long rows (rows and entries, forward and backward) and the byte offsets of their
// shared-memory copy: values, entry ranges, dependency indices.
struct LvlArgsLong {
  int fr, br, fe, be;
};
struct LvlLongLayout {
  size_t fval, bval, fptr, bptr, fidx, bidx, total;
};
template <class T>
RF_LVL_HD inline LvlLongLayout lvl_long_layout(const LvlArgsLong& g) {
  LvlLongLayout o;
  size_t p = 0;
  o.fval = p;
  p += lvl_up16(size_t(g.fe) * sizeof(T));
  o.bval = p;
  p += lvl_up16(size_t(g.be) * sizeof(T));
  o.fptr = p;
  p += lvl_up16((size_t(g.fr) + 1) * sizeof(int));
  o.bptr = p;
  p += lvl_up16((size_t(g.br) + 1) * sizeof(int));
  o.fidx = p;
  p += lvl_up16(size_t(g.fe) * sizeof(unsigned short));
  o.bidx = p;
  p += lvl_up16(size_t(g.be) * sizeof(unsigned short));
  o.total = p;
  return o;
}

}  // namespace rf
