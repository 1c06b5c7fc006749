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

struct CellProps {
  double h, t, k, d, m;
};

__device__ __forceinline__ CellProps props_from_dh(const ThermoTab& tb, double rhoh) {
  if (rhoh < tb.dhmin) rhoh = tb.dhmin;
  else if (rhoh > tb.dhmax) rhoh = tb.dhmax;
  int i1, i2;
  double w1;
  tab_bracket_ix(tb, 0, tb.rhoh, rhoh, i1, i2, w1);
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
