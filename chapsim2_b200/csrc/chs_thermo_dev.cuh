// Device-side property lookups of the variable-property path (table interpolation of
// src/input_thermo.f90:345-446), shared by the property-update and MLP kernels.
#pragma once
#include "chs_kernels.cuh"

namespace chs {

// bisection with the reference's sign test ((col[i1]-x)*(col[im]-x) > MINP moves i1); at most
// log2(n) iterations
__device__ __forceinline__ void tab_bracket(const double* __restrict__ col, int n, double x, int& i1, int& i2,
                                            double& w1) {
  int a = 0, b = n - 1;
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

struct CellProps {
  double h, t, k, d, m;
};

__device__ __forceinline__ CellProps props_from_dh(const ThermoTab& tb, double rhoh) {
  if (rhoh < tb.dhmin) rhoh = tb.dhmin;
  else if (rhoh > tb.dhmax) rhoh = tb.dhmax;
  int i1, i2;
  double w1;
  tab_bracket(tb.rhoh, tb.n, rhoh, i1, i2, w1);
  double w2 = 1.0 - w1;
  const double h0 = w1 * __ldg(tb.h + i1) + w2 * __ldg(tb.h + i2);
  tab_bracket(tb.h, tb.n, h0, i1, i2, w1);
  w2 = 1.0 - w1;
  const double d0 = w1 * __ldg(tb.d + i1) + w2 * __ldg(tb.d + i2);
  CellProps p;
  p.h = rhoh / d0;
  tab_bracket(tb.h, tb.n, p.h, i1, i2, w1);
  w2 = 1.0 - w1;
  p.d = w1 * __ldg(tb.d + i1) + w2 * __ldg(tb.d + i2);
  p.m = w1 * __ldg(tb.m + i1) + w2 * __ldg(tb.m + i2);
  p.k = w1 * __ldg(tb.k + i1) + w2 * __ldg(tb.k + i2);
  p.t = w1 * __ldg(tb.t + i1) + w2 * __ldg(tb.t + i2);
  return p;
}


}  // namespace chs
