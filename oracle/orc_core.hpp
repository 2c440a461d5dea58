// ORACLE — test infrastructure only.  A single-threaded CPU restatement of the reference's
// (sergeyfarin/ressim) fully implicit Newton step, used by tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg as the parity checker.  Nothing in the product links or loads it.
//
// Core numerics shared by the oracle: forward-mode dual numbers (src/lib/ressim/src/fim/ad.rs),
// small dense inverses (the nalgebra 0.35.0 `try_inverse` contract), and triplet -> CSR
// assembly with duplicate summation (the sprs 0.11.5 `TriMatI::to_csr` contract).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

namespace orc {

constexpr double F64_EPS = 2.220446049250313080847263336181640625e-16;  // f64::EPSILON

// Rust f64::max / f64::min ignore a NaN operand; fmax/fmin have the same contract.
inline double rmax(double a, double b) { return std::fmax(a, b); }
inline double rmin(double a, double b) { return std::fmin(a, b); }
// Rust f64::clamp(lo, hi).
inline double rclamp(double x, double lo, double hi) {
  if (x < lo) return lo;
  if (x > hi) return hi;
  return x;
}
inline double rsignum(double x) {
  if (std::isnan(x)) return x;
  return std::signbit(x) ? -1.0 : 1.0;
}

// ---------------------------------------------------------------------------------------------
// Ad<N>: value + N partials (src/lib/ressim/src/fim/ad.rs:21-152).  Operator semantics follow
// the reference exactly, including division by a constant as multiplication by its reciprocal.
// ---------------------------------------------------------------------------------------------
template <int N>
struct Ad {
  double v;
  double d[N];
};

template <int N>
inline Ad<N> ad_const(double v) {
  Ad<N> r;
  r.v = v;
  for (int i = 0; i < N; ++i) r.d[i] = 0.0;
  return r;
}
template <int N>
inline Ad<N> ad_var(double v, int slot) {
  Ad<N> r = ad_const<N>(v);
  r.d[slot] = 1.0;
  return r;
}

template <int N>
inline Ad<N> operator+(const Ad<N>& a, const Ad<N>& b) {
  Ad<N> r;
  r.v = a.v + b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
inline Ad<N> operator-(const Ad<N>& a, const Ad<N>& b) {
  Ad<N> r;
  r.v = a.v - b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
inline Ad<N> operator*(const Ad<N>& a, const Ad<N>& b) {
  Ad<N> r;
  r.v = a.v * b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
inline Ad<N> operator/(const Ad<N>& a, const Ad<N>& b) {
  const double inv = 1.0 / b.v;
  const double inv2 = inv * inv;
  Ad<N> r;
  r.v = a.v * inv;
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) * inv2;
  return r;
}
template <int N>
inline Ad<N> operator-(const Ad<N>& a) {
  Ad<N> r;
  r.v = -a.v;
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
inline Ad<N> operator+(const Ad<N>& a, double b) {
  Ad<N> r = a;
  r.v = a.v + b;
  return r;
}
template <int N>
inline Ad<N> operator+(double a, const Ad<N>& b) {
  return b + a;
}
template <int N>
inline Ad<N> operator-(const Ad<N>& a, double b) {
  Ad<N> r = a;
  r.v = a.v - b;
  return r;
}
template <int N>
inline Ad<N> operator-(double a, const Ad<N>& b) {
  Ad<N> r;
  r.v = a - b.v;
  for (int i = 0; i < N; ++i) r.d[i] = -b.d[i];
  return r;
}
template <int N>
inline Ad<N> operator*(const Ad<N>& a, double b) {
  Ad<N> r;
  r.v = a.v * b;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
inline Ad<N> operator*(double a, const Ad<N>& b) {
  return b * a;
}
template <int N>
inline Ad<N> operator/(const Ad<N>& a, double b) {
  const double inv = 1.0 / b;
  Ad<N> r;
  r.v = a.v * inv;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * inv;
  return r;
}
template <int N>
inline Ad<N> operator/(double a, const Ad<N>& b) {
  return ad_const<N>(a) / b;
}

// Scalar trait (ad.rs:325-417) as overloads over double and Ad<N>.
template <class S>
struct ScalarT;
template <>
struct ScalarT<double> {
  static double from(double v) { return v; }
  static double value(double x) { return x; }
};
template <int N>
struct ScalarT<Ad<N>> {
  static Ad<N> from(double v) { return ad_const<N>(v); }
  static double value(const Ad<N>& x) { return x.v; }
};
template <class S>
inline S sc(double v) {
  return ScalarT<S>::from(v);
}
inline double val(double x) { return x; }
template <int N>
inline double val(const Ad<N>& x) {
  return x.v;
}

inline double s_exp(double x) { return std::exp(x); }
inline double s_powf(double x, double p) { return std::pow(x, p); }
inline double s_sqrt(double x) { return std::sqrt(x); }
inline double s_recip(double x) { return 1.0 / x; }
inline double max_floor(double x, double f) { return rmax(x, f); }
inline double min_ceil(double x, double c) { return rmin(x, c); }
inline double max_of(double a, double b) { return rmax(a, b); }
inline double min_of(double a, double b) { return rmin(a, b); }

template <int N>
inline Ad<N> s_exp(const Ad<N>& a) {
  Ad<N> r;
  r.v = std::exp(a.v);
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * r.v;
  return r;
}
template <int N>
inline Ad<N> s_powf(const Ad<N>& a, double p) {
  Ad<N> r;
  r.v = std::pow(a.v, p);
  const double coef = p * std::pow(a.v, p - 1.0);
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * coef;
  return r;
}
template <int N>
inline Ad<N> s_sqrt(const Ad<N>& a) {
  Ad<N> r;
  r.v = std::sqrt(a.v);
  const double coef = 0.5 / r.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * coef;
  return r;
}
template <int N>
inline Ad<N> s_recip(const Ad<N>& a) {
  Ad<N> r;
  r.v = 1.0 / a.v;
  const double coef = -r.v * r.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * coef;
  return r;
}
template <int N>
inline Ad<N> max_floor(const Ad<N>& a, double f) {
  return a.v >= f ? a : ad_const<N>(f);
}
template <int N>
inline Ad<N> min_ceil(const Ad<N>& a, double c) {
  return a.v <= c ? a : ad_const<N>(c);
}
template <int N>
inline Ad<N> max_of(const Ad<N>& a, const Ad<N>& b) {
  return a.v >= b.v ? a : b;
}
template <int N>
inline Ad<N> min_of(const Ad<N>& a, const Ad<N>& b) {
  return a.v <= b.v ? a : b;
}

// ---------------------------------------------------------------------------------------------
// Dense matrices (row-major) and the nalgebra try_inverse contract: closed-form cofactor
// inverses for 1x1..3x3 that fail only on an exactly zero determinant, LU with partial pivoting
// above that (fails only on an exactly zero pivot).  The fallback used by the reference
// (`invert_tail_block`, gmres_block_jacobi.rs:888-901) is a diagonal reciprocal with 1.0 for
// |d| <= EPS.
// ---------------------------------------------------------------------------------------------
struct Dense {
  int n = 0;
  std::vector<double> a;  // n*n row-major
  Dense() = default;
  explicit Dense(int n_) : n(n_), a(size_t(n_) * n_, 0.0) {}
  double& operator()(int r, int c) { return a[size_t(r) * n + c]; }
  double operator()(int r, int c) const { return a[size_t(r) * n + c]; }
};

inline bool try_inverse(const Dense& m, Dense& out) {
  const int n = m.n;
  out = Dense(n);
  if (n == 0) return true;
  if (n == 1) {
    if (m(0, 0) == 0.0) return false;
    out(0, 0) = 1.0 / m(0, 0);
    return true;
  }
  if (n == 2) {
    const double det = m(0, 0) * m(1, 1) - m(1, 0) * m(0, 1);
    if (det == 0.0) return false;
    out(0, 0) = m(1, 1) / det;
    out(0, 1) = -m(0, 1) / det;
    out(1, 0) = -m(1, 0) / det;
    out(1, 1) = m(0, 0) / det;
    return true;
  }
  if (n == 3) {
    const double m11 = m(0, 0), m12 = m(0, 1), m13 = m(0, 2);
    const double m21 = m(1, 0), m22 = m(1, 1), m23 = m(1, 2);
    const double m31 = m(2, 0), m32 = m(2, 1), m33 = m(2, 2);
    const double c11 = m22 * m33 - m32 * m23;
    const double c21 = m21 * m33 - m31 * m23;
    const double c31 = m21 * m32 - m31 * m22;
    const double det = m11 * c11 - m12 * c21 + m13 * c31;
    if (det == 0.0) return false;
    out(0, 0) = c11 / det;
    out(0, 1) = (m13 * m32 - m33 * m12) / det;
    out(0, 2) = (m12 * m23 - m22 * m13) / det;
    out(1, 0) = -c21 / det;
    out(1, 1) = (m11 * m33 - m31 * m13) / det;
    out(1, 2) = (m13 * m21 - m23 * m11) / det;
    out(2, 0) = c31 / det;
    out(2, 1) = (m12 * m31 - m32 * m11) / det;
    out(2, 2) = (m11 * m22 - m21 * m12) / det;
    return true;
  }
  // LU with partial pivoting, in nalgebra's operation order (linalg/lu.rs `try_invert_to`,
  // `gauss_step`; linalg/solve.rs triangular solves): the first largest |pivot| wins, the
  // multipliers are scaled by the pivot's reciprocal, each update is y = (-p) * c + y, and the
  // back substitution applies the columns from the last one down.
  Dense lu = m;
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  for (int c = 0; c < n; ++c) {
    int piv = c;
    double best = std::fabs(lu(c, c));
    for (int r = c + 1; r < n; ++r) {
      if (std::fabs(lu(r, c)) > best) {
        best = std::fabs(lu(r, c));
        piv = r;
      }
    }
    if (lu(piv, c) == 0.0) return false;
    if (piv != c) {
      for (int k = 0; k < n; ++k) std::swap(lu(c, k), lu(piv, k));
      std::swap(perm[c], perm[piv]);
    }
    const double inv_pivot = 1.0 / lu(c, c);
    for (int r = c + 1; r < n; ++r) lu(r, c) = lu(r, c) * inv_pivot;
    for (int k = c + 1; k < n; ++k) {
      const double p = -lu(c, k);
      for (int r = c + 1; r < n; ++r) lu(r, k) = p * lu(r, c) + lu(r, k);
    }
  }
  std::vector<double> col(n);
  for (int j = 0; j < n; ++j) {
    for (int r = 0; r < n; ++r) col[r] = (perm[r] == j) ? 1.0 : 0.0;
    for (int i = 0; i + 1 < n; ++i) {
      const double coeff = -col[i];
      for (int r = i + 1; r < n; ++r) col[r] = coeff * lu(r, i) + col[r];
    }
    for (int i = n - 1; i >= 0; --i) {
      const double d = lu(i, i);
      if (d == 0.0) return false;
      const double coeff = col[i] / d;
      col[i] = coeff;
      for (int r = 0; r < i; ++r) col[r] = (-coeff) * lu(r, i) + col[r];
    }
    for (int r = 0; r < n; ++r) out(r, j) = col[r];
  }
  return true;
}

// invert_tail_block (gmres_block_jacobi.rs:888-901)
inline Dense invert_or_diag(const Dense& m) {
  Dense out;
  if (try_inverse(m, out)) return out;
  out = Dense(m.n);
  for (int i = 0; i < m.n; ++i) {
    const double d = m(i, i);
    out(i, i) = std::fabs(d) > F64_EPS ? 1.0 / d : 1.0;
  }
  return out;
}

inline void dense_matmul(const Dense& a, const Dense& b, Dense& c) {
  const int n = a.n;
  c = Dense(n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += a(i, k) * b(k, j);
      c(i, j) = s;
    }
}

// ---------------------------------------------------------------------------------------------
// Scalar CSR with sorted columns; triplets summed in insertion order per (row, col).
// ---------------------------------------------------------------------------------------------
struct Trip {
  int r, c;
  double v;
};
struct Csr {
  int n = 0;
  std::vector<int> ptr, col;
  std::vector<double> val;
  double at(int r, int c) const {
    for (int k = ptr[r]; k < ptr[r + 1]; ++k)
      if (col[k] == c) return val[k];
    return 0.0;
  }
};

inline Csr to_csr(int n, std::vector<Trip>& t) {
  std::stable_sort(t.begin(), t.end(), [](const Trip& a, const Trip& b) {
    return a.r != b.r ? a.r < b.r : a.c < b.c;
  });
  Csr m;
  m.n = n;
  m.ptr.assign(n + 1, 0);
  for (size_t k = 0; k < t.size();) {
    size_t e = k;
    double s = 0.0;
    while (e < t.size() && t[e].r == t[k].r && t[e].c == t[k].c) {
      s += t[e].v;
      ++e;
    }
    m.col.push_back(t[k].c);
    m.val.push_back(s);
    m.ptr[t[k].r + 1]++;
    k = e;
  }
  for (int r = 0; r < n; ++r) m.ptr[r + 1] += m.ptr[r];
  return m;
}

inline void csr_matvec(const Csr& m, const std::vector<double>& x, std::vector<double>& y) {
  y.assign(m.n, 0.0);
  for (int r = 0; r < m.n; ++r) {
    double s = 0.0;
    for (int k = m.ptr[r]; k < m.ptr[r + 1]; ++k) s += m.val[k] * x[m.col[k]];
    y[r] = s;
  }
}

// Summation order of the vector dots and norms: 0 is the reference's left-to-right order.  A
// test hook sets w >= 2 (w interleaved partial sums, then added in order), which changes only the
// rounding, to measure how far rounding alone moves a run.
inline int g_sum_order = 0;
inline double vdot_n(size_t n, const double* a, const double* b) {
  if (g_sum_order < 2) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
  }
  const size_t w = size_t(g_sum_order);
  std::vector<double> part(w, 0.0);
  for (size_t i = 0; i < n; ++i) part[i % w] += a[i] * b[i];
  double s = 0.0;
  for (size_t k = 0; k < w; ++k) s += part[k];
  return s;
}
inline double vnorm(const std::vector<double>& x) { return std::sqrt(vdot_n(x.size(), x.data(), x.data())); }
inline double vdot(const std::vector<double>& a, const std::vector<double>& b) {
  return vdot_n(a.size(), a.data(), b.data());
}

}  // namespace orc
