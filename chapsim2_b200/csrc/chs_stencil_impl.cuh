// Specialised explicit line operators (see chs_stencil_dev.cuh); included once per field type by
// chs_stencil_f64.cu and chs_stencil_f32.cu with CHS_STENCIL_T defined.
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>

#include "chs_stencil_dev.cuh"

namespace chs {

// ---------------------------------------------------------------------------
// Explicit operators, specialised: the input expression's term modes are template parameters
// (read-only loads, no per-value mode switch) and no integer division maps threads to positions.
//  * y and z lines: each thread forms kWin consecutive outputs of one line from a register window
//    of the input expression (each input value loaded once per thread instead of once per stencil
//    point);
//  * x lines (contiguous): the expression of a whole line is staged in shared memory, then every
//    output row (bulk, wrapped bulk or boundary row) reads it from there.
// Rows outside the bulk range evaluate the plan's boundary rows exactly as stencil_op_kernel does.
// ---------------------------------------------------------------------------
constexpr int kWin = 4;

// the value of one input term from its array values (the one formula every path uses, so the
// window, segment and vector paths give the same bits)
template <int M, typename T>
__device__ __forceinline__ T term_val(const TermT<T>& t, T x, T y, T z) {
  if (M == T_X) return T(t.s) * x;
  if (M == T_XY) return T(t.s) * (x * y);
  if (M == T_XpY) return T(t.s) * (x + T(t.c) * y);
  if (M == T_XpYZ) return T(t.s) * (x + T(t.c) * y) * z;
  return T(0);
}
template <int M, typename T>
__device__ __forceinline__ T term_ro(const TermT<T>& t, int a) {
  const T x = __ldg(t.X + a);
  const T y = (M == T_XY || M == T_XpY || M == T_XpYZ) ? __ldg(t.Y + a) : T(0);
  const T z = M == T_XpYZ ? __ldg(t.Z + a) : T(0);
  return term_val<M>(t, x, y, z);
}
template <int M0, int M1, typename T>
__device__ __forceinline__ T expr_ro(const LineIOT<T>& io, int a) {
  T v = term_ro<M0>(io.t[0], a);
  if (M1 != T_NONE) v += term_ro<M1>(io.t[1], a);
  return v;
}

// stencil reach of a family: offsets [lo4, hi4] of the 4-point (r2 != 0) bulk formula and
// [lo2, hi2] of its 2-point part
template <int FAM>
struct Reach {
  static constexpr int lo4 = (FAM == M1P2C || FAM == D1P2C) ? -1 : -2;
  static constexpr int hi4 = (FAM == M1C2P || FAM == D1C2P) ? 1 : 2;
  static constexpr int lo2 = (FAM == M1P2C || FAM == D1P2C) ? 0 : -1;
  static constexpr int hi2 = (FAM == M1C2P || FAM == D1C2P) ? 0 : 1;
};

// bulk_fn on a register window: w[b + o] holds the expression at offset o of the output row
template <int FAM, typename T>
__device__ __forceinline__ T bulk_win(const T* w, int b, T r1, T r2) {
  T v;
  if (FAM == M1P2C) v = r1 * (w[b] + w[b + 1]);
  else if (FAM == M1C2P) v = r1 * (w[b] + w[b - 1]);
  else if (FAM == D1C2C || FAM == D1P2P) v = r1 * (w[b + 1] - w[b - 1]);
  else if (FAM == D1C2P) v = r1 * (w[b] - w[b - 1]);
  else v = r1 * (w[b + 1] - w[b]);  // D1P2C
  if (r2 != T(0)) {
    if (FAM == M1P2C) v += r2 * (w[b - 1] + w[b + 2]);
    else if (FAM == M1C2P) v += r2 * (w[b + 1] + w[b - 2]);
    else if (FAM == D1C2C || FAM == D1P2P) v += r2 * (w[b + 2] - w[b - 2]);
    else if (FAM == D1C2P) v += r2 * (w[b + 1] - w[b - 2]);
    else v += r2 * (w[b + 2] - w[b - 1]);
  }
  return v;
}

// one boundary row of the plan (as stencil_op_kernel), input expression at ibase + q * istride
// (a call out of line measured slower than the registers it saves)
template <typename T, int M0, int M1>
__device__ __forceinline__ T boundary_row(const OpPlan& P, const LineIOT<T>& io, int ibase, int istride, int p, int L,
                                       int nlines) {
  T v = T(0);
  for (int s = 0; s < P.nspec; ++s) {
    if (P.sp[s].row != p) continue;
    const SpecialRow& R = P.sp[s];
    T acc = T(0);
    for (int t = 0; t < R.nt; ++t) acc += T(R.w[t]) * expr_ro<M0, M1>(io, ibase + R.idx[t] * istride);
    for (int u = 0; u < 4; ++u)
      if (R.wb[u] != 0.0) acc += T(R.wb[u]) * io.fbc[u * nlines + L];
    v = acc * T(P.dd);
  }
  return v;
}

// y metric, Neumann overrides and the store mode (as stencil_op_kernel)
template <typename T>
__device__ __forceinline__ void finish_row(const OpPlan& P, const LineIOT<T>& io, const double* __restrict__ table,
                                           int p, int L, int nlines, int64_t a, T v) {
  if (P.lmap >= 0) v *= T(table[P.lmap + p]);
  if (P.neu1 && p == 0) v = io.fbc[L];
  if (P.neu2 && p == P.nout - 1) v = io.fbc[nlines + L];
  store_out(io, a, T(io.g), v);
}

// 16-byte vectors of the field type: the main part of a segment is loaded with one vector load
// per array and lane where the line start is 16-byte aligned
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int n = 2;
};
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int n = 4;
};

// the V array values of a term at a (a multiple of V, arrays 16-byte aligned)
template <int M, typename T, int V>
__device__ __forceinline__ void term_load_vec(const TermT<T>& t, int a, T (&x)[V], T (&y)[V], T (&z)[V]) {
  using VT = typename Vec16<T>::type;
  *reinterpret_cast<VT*>(x) = __ldg(reinterpret_cast<const VT*>(t.X + a));
  if (M == T_XY || M == T_XpY || M == T_XpYZ) *reinterpret_cast<VT*>(y) = __ldg(reinterpret_cast<const VT*>(t.Y + a));
  else
#pragma unroll
    for (int u = 0; u < V; ++u) y[u] = T(0);
  if (M == T_XpYZ) *reinterpret_cast<VT*>(z) = __ldg(reinterpret_cast<const VT*>(t.Z + a));
  else
#pragma unroll
    for (int u = 0; u < V; ++u) z[u] = T(0);
}
// expr_ro at V consecutive positions from a, element by element the same formula
template <int M0, int M1, typename T, int V>
__device__ __forceinline__ void expr_vec(const LineIOT<T>& io, int a, T (&v)[V]) {
  T x0[V], y0[V], z0[V], x1[V], y1[V], z1[V];
  term_load_vec<M0>(io.t[0], a, x0, y0, z0);
  if (M1 != T_NONE) term_load_vec<M1>(io.t[1], a, x1, y1, z1);
#pragma unroll
  for (int u = 0; u < V; ++u) {
    v[u] = term_val<M0>(io.t[0], x0[u], y0[u], z0[u]);
    if (M1 != T_NONE) v[u] += term_val<M1>(io.t[1], x1[u], y1[u], z1[u]);
  }
}

// y (DIR 1) or z (DIR 2) lines: each thread owns V = 16 / sizeof(T) adjacent x positions (one
// 16-byte vector per load and store) and kWin consecutive rows of their lines; a register window
// of the input expression along the line serves all kWin rows (each input value loaded once per
// thread).  Needs n1 % V == 0 and 16-byte aligned arrays (checked by the launcher).
template <typename T, int DIR, int FAM, int M0, int M1>
__device__ __forceinline__ void stencil_win_body(const OpPlan& P, const LineIOT<T>& io,
                                                 const double* __restrict__ table, int nlines) {
  using RC = Reach<FAM>;
  using VT = typename Vec16<T>::type;
  constexpr int V = Vec16<T>::n;
  constexpr int W = kWin + RC::hi4 - RC::lo4;
  const int nin = P.nin, nout = P.nout, n1 = io.n1;
  int L, ibase, istride, p0;
  int64_t obase, ostride;
  if (DIR == 1) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    p0 = (blockIdx.y * blockDim.y + threadIdx.y) * kWin;
    const int k = blockIdx.z;
    if (i >= n1 || p0 >= nout) return;
    L = i + n1 * k;
    ibase = k * nin * n1 + i;
    istride = n1;
    obase = (int64_t)k * nout * n1 + i;
    ostride = n1;
  } else {
    const int plane = n1 * io.n2;
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    p0 = blockIdx.y * kWin;
    if (q >= plane) return;
    L = q;
    ibase = q;
    istride = plane;
    obase = q;
    ostride = plane;
  }
  const T r1 = T(P.r1), r2 = T(P.r2), dd = T(P.dd);
  const bool r2on = P.r2 != 0.0, wrap = P.wrap != 0;
  T w[W][V];
#pragma unroll
  for (int s = 0; s < W; ++s) {
    // the 2-point formula never reads the outermost slots
    const bool need = r2on || (s >= RC::lo2 - RC::lo4 && s <= kWin - 1 + RC::hi2 - RC::lo4);
    int q = p0 + RC::lo4 + s;
    // wrapped (periodic) or clamped; clamped slots are read only by boundary rows, which do not
    // use the window
    if (wrap) q = q < 0 ? q + nin : (q >= nin ? q - nin : q);
    else q = q < 0 ? 0 : (q >= nin ? nin - 1 : q);
    if (need) {
      expr_vec<M0, M1>(io, ibase + q * istride, w[s]);
    } else {
#pragma unroll
      for (int e = 0; e < V; ++e) w[s][e] = T(0);
    }
  }
  const bool plain = io.omode == O_STORE && !io.accumulate;
  const bool frac = io.omode == O_FRAC;
  const T g = T(io.g);
  const T tdt = T(io.dt), tg = T(io.gam), tz = T(io.zeta), ta = T(io.alpha);
#pragma unroll
  for (int u = 0; u < kWin; ++u) {
    const int p = p0 + u;
    if (p >= nout) break;
    T v[V];
    if (wrap || (p >= P.b_lo && p <= P.b_hi)) {
#pragma unroll
      for (int e = 0; e < V; ++e) {
        T col[W];
#pragma unroll
        for (int s = 0; s < W; ++s) col[s] = w[s][e];
        v[e] = bulk_win<FAM>(col, u - RC::lo4, r1, r2) * dd;
      }
    } else {
#pragma unroll
      for (int e = 0; e < V; ++e) v[e] = boundary_row<T, M0, M1>(P, io, ibase + e, istride, p, L + e, nlines);
    }
    if (P.lmap >= 0) {
      const T mp = T(table[P.lmap + p]);
#pragma unroll
      for (int e = 0; e < V; ++e) v[e] *= mp;
    }
    if ((P.neu1 && p == 0) || (P.neu2 && p == nout - 1)) {
      const int off = p == 0 ? 0 : nlines;
#pragma unroll
      for (int e = 0; e < V; ++e) v[e] = io.fbc[off + L + e];
    }
    const int64_t a = obase + (int64_t)p * ostride;
    if (plain) {
      T o[V];
#pragma unroll
      for (int e = 0; e < V; ++e) o[e] = g * v[e];
      *reinterpret_cast<VT*>(io.out + a) = *reinterpret_cast<const VT*>(o);
    } else if (frac) {
      // store_out's O_FRAC arithmetic on vectors of the output, the previous right-hand side and q
      T cur[V], last[V], r[V], q[V];
      *reinterpret_cast<VT*>(cur) = *reinterpret_cast<const VT*>(io.out + a);
      *reinterpret_cast<VT*>(last) = *reinterpret_cast<const VT*>(io.rhs0 + a);
      if (io.qupd) *reinterpret_cast<VT*>(q) = *reinterpret_cast<const VT*>(io.qupd + a);
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const T pfc = g * v[e];
        T tot = tg * cur[e] + tz * last[e];
        tot = tot + ta * pfc;
        r[e] = tdt * tot;
      }
      *reinterpret_cast<VT*>(io.rhs0 + a) = *reinterpret_cast<const VT*>(cur);
      *reinterpret_cast<VT*>(io.out + a) = *reinterpret_cast<const VT*>(r);
      if (io.qupd) {
#pragma unroll
        for (int e = 0; e < V; ++e) q[e] = q[e] + (r[e] - T(0));
        *reinterpret_cast<VT*>(io.qupd + a) = *reinterpret_cast<const VT*>(q);
      }
    } else {
      OutPre<T> o[V];
#pragma unroll
      for (int e = 0; e < V; ++e) o[e] = load_out(io, a + e);
#pragma unroll
      for (int e = 0; e < V; ++e) store_out(io, a + e, g, v[e], o[e]);
    }
  }
}

template <typename T, int FAM, int M0, int M1>
__global__ void __launch_bounds__(256) stencil_winy_kernel(const __grid_constant__ OpPlan P,
                                                              const __grid_constant__ LineIOT<T> io,
                                                              const double* __restrict__ table, int nlines) {
  stencil_win_body<T, 1, FAM, M0, M1>(P, io, table, nlines);
}
template <typename T, int FAM, int M0, int M1>
__global__ void __launch_bounds__(256) stencil_winz_kernel(const __grid_constant__ OpPlan P,
                                                           const __grid_constant__ LineIOT<T> io,
                                                           const double* __restrict__ table, int nlines) {
  stencil_win_body<T, 2, FAM, M0, M1>(P, io, table, nlines);
}

// x lines (DIR 0): each warp forms a segment of kSeg consecutive outputs of one line from a
// warp-private shared-memory copy of the input expression over the segment and two values either
// side (wrapped for periodic lines); boundary rows of non-periodic lines read the input directly
constexpr int kSeg = 128, kSegHalo = 2;

template <typename T, int FAM, int M0, int M1>
__global__ void __launch_bounds__(256) stencil_xseg_kernel(const __grid_constant__ OpPlan P,
                                                           const __grid_constant__ LineIOT<T> io,
                                                           const double* __restrict__ table, int nlines, int nseg) {
  constexpr int V = Vec16<T>::n;
  constexpr int kO = V;  // slot of the segment's first value (16-byte aligned); halo at kO-2, kO-1
  __shared__ __align__(16) T tile[8][kSeg + 2 * V];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * 8 + warp;  // global warp = line * nseg + segment
  if (gw >= nlines * nseg) return;
  const int L = gw / nseg, i0 = (gw - L * nseg) * kSeg;
  const int nin = P.nin, nout = P.nout;
  const int ibase = L * nin;
  const bool wrap = P.wrap != 0;
  T* s = tile[warp];
  // the segment: no wrap or clamp unless it runs past the end of the line
  const bool full = i0 + kSeg <= nin;
  const uintptr_t al = reinterpret_cast<uintptr_t>(io.t[0].X) | reinterpret_cast<uintptr_t>(io.t[0].Y) |
                       reinterpret_cast<uintptr_t>(io.t[0].Z) | reinterpret_cast<uintptr_t>(io.t[1].X) |
                       reinterpret_cast<uintptr_t>(io.t[1].Y) | reinterpret_cast<uintptr_t>(io.t[1].Z);
  if (full && (al & 15) == 0 && nin % V == 0) {
#pragma unroll
    for (int m = 0; m < kSeg / (32 * V); ++m) {
      const int c = lane + 32 * m;
      T v[V];
      expr_vec<M0, M1>(io, ibase + i0 + c * V, v);
      *reinterpret_cast<typename Vec16<T>::type*>(s + kO + c * V) = *reinterpret_cast<const typename Vec16<T>::type*>(v);
    }
  } else {
#pragma unroll
    for (int m = 0; m < kSeg / 32; ++m) {
      int q = i0 + lane + 32 * m;
      if (!full) {
        if (wrap) {
          while (q >= nin) q -= nin;  // lines shorter than a segment wrap more than once
        } else {
          q = q >= nin ? nin - 1 : q;  // clamped slots are read by boundary rows only
        }
      }
      s[kO + lane + 32 * m] = expr_ro<M0, M1>(io, ibase + q);
    }
  }
  // two values either side (lanes 0-1 left, 2-3 right)
  if (lane < 2 * kSegHalo) {
    int q = lane < kSegHalo ? i0 - kSegHalo + lane : i0 + kSeg + (lane - kSegHalo);
    if (wrap) {
      while (q < 0) q += nin;
      while (q >= nin) q -= nin;
    } else {
      q = q < 0 ? 0 : (q >= nin ? nin - 1 : q);
    }
    s[lane < kSegHalo ? kO - kSegHalo + lane : kO + kSeg + (lane - kSegHalo)] = expr_ro<M0, M1>(io, ibase + q);
  }
  __syncwarp();
  const T r1 = T(P.r1), r2 = T(P.r2), dd = T(P.dd);
  const int64_t obase = (int64_t)L * nout;
  // periodic full segments with a plain store: each lane forms V adjacent outputs from three
  // 16-byte tile reads and stores them as one vector
  const bool vout = wrap && i0 + kSeg <= nout && nout % V == 0 && io.omode == O_STORE && !io.accumulate &&
                    (reinterpret_cast<uintptr_t>(io.out) & 15) == 0;
  if (vout) {
    using VT = typename Vec16<T>::type;
    const T g = T(io.g);
#pragma unroll
    for (int m = 0; m < kSeg / (32 * V); ++m) {
      const int c = lane + 32 * m;  // outputs i0 + c*V .. i0 + c*V + V-1
      T win[3 * V];                 // input positions -V .. 2V-1 relative to the chunk
      *reinterpret_cast<VT*>(win) = *reinterpret_cast<const VT*>(s + kO + (c - 1) * V);
      *reinterpret_cast<VT*>(win + V) = *reinterpret_cast<const VT*>(s + kO + c * V);
      *reinterpret_cast<VT*>(win + 2 * V) = *reinterpret_cast<const VT*>(s + kO + (c + 1) * V);
      T o[V];
#pragma unroll
      for (int e = 0; e < V; ++e) o[e] = g * (bulk_win<FAM>(win, V + e, r1, r2) * dd);
      *reinterpret_cast<VT*>(io.out + obase + i0 + c * V) = *reinterpret_cast<const VT*>(o);
    }
    return;
  }
  auto fs = [&](int qq) -> T { return s[qq - i0 + kO]; };
#pragma unroll
  for (int m = 0; m < kSeg / 32; ++m) {
    const int p = i0 + lane + 32 * m;
    if (p >= nout) break;
    T v;
    if (wrap || (p >= P.b_lo && p <= P.b_hi)) v = bulk_fn<FAM>(fs, p, r1, r2) * dd;
    else v = boundary_row<T, M0, M1>(P, io, ibase, 1, p, L, nlines);
    finish_row(P, io, table, p, L, nlines, obase + p, v);
  }
}

template <typename T, int DIR, int FAM, int M0, int M1>
void launch_win(const OpPlan& P, const LineIOT<T>& io, const double* table, cudaStream_t st, int nlines) {
  if (DIR == 0) {
    const int nseg = (P.nout + kSeg - 1) / kSeg;
    const int64_t warps = (int64_t)nlines * nseg;
    if (warps >= 0x7fffffff) throw std::runtime_error("explicit operator: too many line segments");
    stencil_xseg_kernel<T, FAM, M0, M1><<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(P, io, table, nlines, nseg);
  } else if (DIR == 1) {
    // wide rows of x per warp group (contiguous DRAM segments), the rest of the CTA along y
    constexpr int V = Vec16<T>::n;
    const int nv = io.n1 / V;
    const int bx = nv >= 64 ? 64 : 32, by = 256 / bx;
    const int chunks = (P.nout + kWin - 1) / kWin;
    dim3 grid((unsigned)((nv + bx - 1) / bx), (unsigned)((chunks + by - 1) / by), (unsigned)io.n3);
    stencil_winy_kernel<T, FAM, M0, M1><<<grid, dim3(bx, by), 0, st>>>(P, io, table, nlines);
  } else {
    constexpr int V = Vec16<T>::n;
    const int nv = io.n1 * io.n2 / V;
    dim3 grid((unsigned)((nv + 255) / 256), (unsigned)((P.nout + kWin - 1) / kWin));
    stencil_winz_kernel<T, FAM, M0, M1><<<grid, 256, 0, st>>>(P, io, table, nlines);
  }
}

// the specialised kernels cover the interpolations of single arrays and the derivative inputs the
// substep forms (products, linear combinations, their sums); false: use stencil_op_kernel
template <typename T, int DIR>
bool try_launch_win(const OpPlan& P, const LineIOT<T>& io, const double* table, cudaStream_t st,
                           int nlines) {
  const int m0 = io.t[0].mode, m1 = io.t[1].mode;
  const int sig = m0 * 8 + m1;
  if (DIR != 0) {
    // y and z kernels: V adjacent x positions per thread, 16-byte vectors
    constexpr int V = Vec16<T>::n;
    uintptr_t al = reinterpret_cast<uintptr_t>(io.out) | reinterpret_cast<uintptr_t>(io.onum) |
                   reinterpret_cast<uintptr_t>(io.rhs0) | reinterpret_cast<uintptr_t>(io.qupd);
    for (int q = 0; q < 2; ++q)
      al |= reinterpret_cast<uintptr_t>(io.t[q].X) | reinterpret_cast<uintptr_t>(io.t[q].Y) |
            reinterpret_cast<uintptr_t>(io.t[q].Z);
    if (io.n1 % V != 0 || (al & 15) != 0) return false;
  }
#define CHS_WIN(F, A, B)                                        \
  if (P.fam == F && sig == A * 8 + B) {                         \
    launch_win<T, DIR, F, A, B>(P, io, table, st, nlines);      \
    return true;                                                \
  }
  CHS_WIN(M1P2C, T_X, T_NONE)
  CHS_WIN(M1C2P, T_X, T_NONE)
#define CHS_WIN_D(F)                 \
  CHS_WIN(F, T_X, T_NONE)            \
  CHS_WIN(F, T_XY, T_NONE)           \
  CHS_WIN(F, T_XpY, T_NONE)          \
  CHS_WIN(F, T_XpYZ, T_NONE)         \
  CHS_WIN(F, T_XY, T_XpY)            \
  CHS_WIN(F, T_XY, T_XpYZ)           \
  CHS_WIN(F, T_XY, T_XY)
  CHS_WIN_D(D1C2P)
  CHS_WIN_D(D1P2C)
#undef CHS_WIN_D
#undef CHS_WIN
  return false;
}


template bool try_launch_win<CHS_STENCIL_T, 0>(const OpPlan&, const LineIOT<CHS_STENCIL_T>&, const double*, cudaStream_t,
                                               int);
template bool try_launch_win<CHS_STENCIL_T, 1>(const OpPlan&, const LineIOT<CHS_STENCIL_T>&, const double*, cudaStream_t,
                                               int);
template bool try_launch_win<CHS_STENCIL_T, 2>(const OpPlan&, const LineIOT<CHS_STENCIL_T>&, const double*, cudaStream_t,
                                               int);

}  // namespace chs
