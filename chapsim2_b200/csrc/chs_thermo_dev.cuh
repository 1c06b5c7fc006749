// Device-side property lookups of the variable-property path (table interpolation of
// src/input_thermo.f90:345-446), shared by the property-update and MLP kernels.
#pragma once
#include "chs_kernels.cuh"

namespace chs {

// bisection with the reference's sign test ((col[i1]-x)*(col[im]-x) > MINP moves i1) from the
// state (a, b); at most log2(b - a) iterations
__device__ __forceinline__ void tab_bracket_from(const double* __restrict__ col, int a, int b, double x, int& i1,
                                                 int& i2, double& w1) {
  while (b - a > 1) {
    const int m = a + (b - a) / 2;
    const double d1 = __ldg(col + a) - x, dm = __ldg(col + m) - x;
    if (d1 * dm > 1.0e-20) a = m;
    else b = m;
  }
  const double ca = __ldg(col + a), cb = __ldg(col + b);
  i1 = a;
  i2 = b;
  w1 = (cb - x) / (cb - ca);
}
__device__ __forceinline__ void tab_bracket(const double* __restrict__ col, int n, double x, int& i1, int& i2,
                                            double& w1) {
  tab_bracket_from(col, 0, n - 1, x, i1, i2, w1);
}
// the same search, started from the bracket index of column c (0: rho*h, 1: h) when x lies in
// the indexed range
__device__ __forceinline__ void tab_bracket_ix(const ThermoTab& tb, int c, const double* __restrict__ col, double x,
                                               int& i1, int& i2, double& w1) {
  int a = 0, b = tb.n - 1;
  if (tb.ix[c] && x >= tb.ix_lo[c] && x <= tb.ix_hi[c]) {
    int bi = (int)((x - tb.ix_lo[c]) * tb.ix_iw[c]);
    bi = bi < tb.ix_nb - 1 ? bi : tb.ix_nb - 1;
    const int2 s = __ldg(tb.ix[c] + bi);
    a = s.x;
    b = s.y;
  }
  tab_bracket_from(col, a, b, x, i1, i2, w1);
}

// Search of a strictly increasing column started near row r: bisection from (r - w, r + w + 1)
// when that range holds x.  Where x lies more than kBracketMargin from both ends of the bracket
// found, every node of the column is that far from x, so each sign test of the full search
// ((col[a]-x)*(col[m]-x) > 1e-20) takes the ordinary bisection branch and the full search ends in
// the same bracket: the result is then exactly the full search's.  false: not verified (the
// caller runs the full search).
constexpr double kBracketMargin = 2.0e-10;
__device__ __forceinline__ bool tab_bracket_near(const double* __restrict__ col, int n, int r, int w, double x,
                                                 int& i1, int& i2, double& w1) {
  int a = r - w, b = r + w + 1;
  if (a < 0) a = 0;
  if (b > n - 1) b = n - 1;
  if (a >= b || !(__ldg(col + a) < x && x < __ldg(col + b))) return false;
  tab_bracket_from(col, a, b, x, i1, i2, w1);
  return (x - __ldg(col + i1)) > kBracketMargin && (__ldg(col + i2) - x) > kBracketMargin;
}

struct CellProps {
  double h, t, k, d, m;
};

// Property lookup from rho*h (ftp_refresh_thermal_properties_from_DH): rho*h -> h0 on the rho*h
// column, h0 -> rho0 on the h column, h = rho*h/rho0, h -> properties on the h column.  hint >= 0:
// a predicted row of the rho*h bracket (e.g. from the surrogate network's T), tried within
// +-win rows; *hit tells whether it was verified
// (the h-column searches start from the bracket index).  Every path returns the full search's
// result.
__device__ __forceinline__ CellProps props_from_dh(const ThermoTab& tb, double rhoh, int hint = -1, int win = 0,
                                                   bool* hit = nullptr) {
  if (rhoh < tb.dhmin) rhoh = tb.dhmin;
  else if (rhoh > tb.dhmax) rhoh = tb.dhmax;
  int i1, i2;
  double w1;
  const bool near = hint >= 0 && tab_bracket_near(tb.rhoh, tb.n, hint, win, rhoh, i1, i2, w1);
  if (hit) *hit = near;
  if (!near) tab_bracket_ix(tb, 0, tb.rhoh, rhoh, i1, i2, w1);
  double w2 = 1.0 - w1;
  const double h0 = w1 * __ldg(tb.h + i1) + w2 * __ldg(tb.h + i2);
  tab_bracket_ix(tb, 1, tb.h, h0, i1, i2, w1);
  w2 = 1.0 - w1;
  const double d0 = w1 * __ldg(tb.d + i1) + w2 * __ldg(tb.d + i2);
  CellProps p;
  p.h = rhoh / d0;
  tab_bracket_ix(tb, 1, tb.h, p.h, i1, i2, w1);
  w2 = 1.0 - w1;
  p.d = w1 * __ldg(tb.d + i1) + w2 * __ldg(tb.d + i2);
  p.m = w1 * __ldg(tb.m + i1) + w2 * __ldg(tb.m + i2);
  p.k = w1 * __ldg(tb.k + i1) + w2 * __ldg(tb.k + i2);
  p.t = w1 * __ldg(tb.t + i1) + w2 * __ldg(tb.t + i2);
  return p;
}


}  // namespace chs
