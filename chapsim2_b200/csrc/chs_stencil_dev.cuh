// Device helpers shared by the line-operator translation units: output store modes, the bulk
// stencil of each family, the runtime-mode input expression, and the entry of the specialised
// explicit-operator kernels (compiled in chs_stencil_f64.cu / chs_stencil_f32.cu).
#pragma once
#include <cuda_runtime.h>

#include "chs_kernels.cuh"

namespace chs {

// The operands a store mode reads at the output position (the output itself when accumulating or
// for O_FRAC, the previous right-hand side and q for O_FRAC, the factor of O_DIV / O_MUL), loaded
// by load_out before any store of the thread: a load behind a store through another pointer of the
// same struct waits for that store, a full memory round trip per element.
template <typename T>
struct OutPre {
  T x;     // the factor of O_DIV / O_MUL, else the output's current value
  T last;  // O_FRAC: the previous right-hand side
  T q;     // O_FRAC: q
};
template <typename T>
__device__ __forceinline__ OutPre<T> load_out(const LineIOT<T>& io, int64_t a) {
  OutPre<T> o{T(0), T(0), T(0)};
  if (io.omode == O_DIV || io.omode == O_MUL) {
    o.x = io.onum[a];
  } else if (io.omode == O_FRAC) {
    o.x = io.out[a];
    o.last = io.rhs0[a];
    if (io.qupd) o.q = io.qupd[a];
  } else if (io.accumulate) {
    o.x = io.out[a];
  }
  return o;
}
template <typename T>
__device__ __forceinline__ void store_out(const LineIOT<T>& io, int64_t a, T g, T v, const OutPre<T>& o) {
  if (io.omode == O_DIV) {
    io.out[a] = o.x / (g * v);
  } else if (io.omode == O_MUL) {
    io.out[a] = o.x * (g * v);
  } else if (io.omode == O_FRAC) {
    // the arithmetic of fractional_step_kernel with pfc = g*v, then update_q_kernel's q += r
    const T tdt = T(io.dt), tg = T(io.gam), tz = T(io.zeta), ta = T(io.alpha);
    const T pfc = g * v;
    const T cur = o.x, last = o.last;
    T tot = tg * cur + tz * last;
    io.rhs0[a] = cur;
    tot = tot + ta * pfc;
    const T r = tdt * tot;
    io.out[a] = r;
    if (io.qupd) io.qupd[a] = o.q + (r - T(0));
  } else {
    io.out[a] = io.accumulate ? o.x + g * v : g * v;
  }
}
template <typename T>
__device__ __forceinline__ void store_out(const LineIOT<T>& io, int64_t a, T g, T v) {
  store_out(io, a, g, v, load_out(io, a));
}

template <int FAM, typename T, typename F>
__device__ __forceinline__ T bulk_fn(const F& f, int i, T r1, T r2) {
  T v;
  if (FAM == M1P2C) v = r1 * (f(i) + f(i + 1));
  else if (FAM == M1C2P) v = r1 * (f(i) + f(i - 1));
  else if (FAM == D1C2C || FAM == D1P2P) v = r1 * (f(i + 1) - f(i - 1));
  else if (FAM == D1C2P) v = r1 * (f(i) - f(i - 1));
  else v = r1 * (f(i + 1) - f(i));  // D1P2C
  if (r2 != T(0)) {
    if (FAM == M1P2C) v += r2 * (f(i - 1) + f(i + 2));
    else if (FAM == M1C2P) v += r2 * (f(i + 1) + f(i - 2));
    else if (FAM == D1C2C || FAM == D1P2P) v += r2 * (f(i + 2) - f(i - 2));
    else if (FAM == D1C2P) v += r2 * (f(i + 1) - f(i - 2));
    else v += r2 * (f(i + 2) - f(i - 1));
  }
  return v;
}

// int32-offset evaluation of the input expression (arrays below 2^31 values)
template <typename T>
__device__ __forceinline__ T eval_term32(const TermT<T>& t, int a) {
  switch (t.mode) {
    case T_X: return T(t.s) * t.X[a];
    case T_XY: return T(t.s) * (t.X[a] * t.Y[a]);
    case T_XpY: return T(t.s) * (t.X[a] + T(t.c) * t.Y[a]);
    case T_XpYZ: return T(t.s) * (t.X[a] + T(t.c) * t.Y[a]) * t.Z[a];
    default: return T(0);
  }
}
template <typename T>
__device__ __forceinline__ T eval_expr32(const LineIOT<T>& io, int a) {
  T v = eval_term32(io.t[0], a);
  if (io.t[1].mode != T_NONE) v += eval_term32(io.t[1], a);
  return v;
}

// specialised explicit operators for the expression signatures the substep forms; false: the
// caller runs the generic stencil_op_kernel
template <typename T, int DIR>
bool try_launch_win(const OpPlan& P, const LineIOT<T>& io, const double* table, cudaStream_t st, int nlines);

}  // namespace chs
