// sm_100a kernels of the CHAPSim2 hot path: batched compact line operators,
// Stockham FFTs, the FISHPACK y-tridiagonal solve, spectral division and the
// elementwise/reduction kernels of the RK3 substep.
#include <cuda_runtime.h>

#include <cstdio>
#include <stdexcept>

#include "chs_kernels.cuh"
#include "chs_stencil_dev.cuh"
#include "chs_thermo_dev.cuh"

namespace chs {

// ===========================================================================
// Compact line operator
//
// One CTA owns LT consecutive lines.  The tile is staged into shared memory
// with coalesced loads (rows for x, LT consecutive i for y and z), the input
// expression is evaluated on the fly, then one thread per line builds the RHS
// with a sliding 5-point register window and runs the Thomas forward sweep
// in place, followed by the backward sweep and the cyclic closure.  The store
// phase applies the cyclic correction, the y metric, the Neumann overrides and
// the output accumulation, again coalesced.
// ===========================================================================
// exact input reads of the bulk stencil of each family, rows i (0-based), column stride ld
template <int FAM, typename T>
__device__ __forceinline__ T bulk_at(const T* col, int ld, int i, T r1, T r2) {
  if (FAM == M1P2C) return r1 * (col[i * ld] + col[(i + 1) * ld]) + r2 * (col[(i - 1) * ld] + col[(i + 2) * ld]);
  if (FAM == M1C2P) return r1 * (col[i * ld] + col[(i - 1) * ld]) + r2 * (col[(i + 1) * ld] + col[(i - 2) * ld]);
  if (FAM == D1C2C || FAM == D1P2P)
    return r1 * (col[(i + 1) * ld] - col[(i - 1) * ld]) + r2 * (col[(i + 2) * ld] - col[(i - 2) * ld]);
  if (FAM == D1C2P) return r1 * (col[i * ld] - col[(i - 1) * ld]) + r2 * (col[(i + 1) * ld] - col[(i - 2) * ld]);
  return r1 * (col[(i + 1) * ld] - col[i * ld]) + r2 * (col[(i + 2) * ld] - col[(i - 1) * ld]);  // D1P2C
}

// boundary row of the plan evaluated from the staged column
template <typename T>
__device__ __forceinline__ T special_at(const SpecialRow& R, const T* col, int ld, const T* fbc, int nlines, int L) {
  T v = T(0);
  for (int t = 0; t < R.nt; ++t) v += T(R.w[t]) * col[R.idx[t] * ld];
  for (int u = 0; u < 4; ++u)
    if (R.wb[u] != 0.0) v += T(R.wb[u]) * fbc[u * nlines + L];
  return v;
}

template <typename T>
__device__ __forceinline__ T eval_term(const TermT<T>& t, int64_t a) {
  switch (t.mode) {
    case T_X: return T(t.s) * t.X[a];
    case T_XY: return T(t.s) * (t.X[a] * t.Y[a]);
    case T_XpY: return T(t.s) * (t.X[a] + T(t.c) * t.Y[a]);
    case T_XpYZ: return T(t.s) * (t.X[a] + T(t.c) * t.Y[a]) * t.Z[a];
    default: return T(0);
  }
}

// store one operator output: out = g*v, out += g*v, out = num / (g*v) or out = num * (g*v)

template <typename T>
__device__ __forceinline__ T eval_expr(const LineIOT<T>& io, int64_t a) {
  T v = eval_term(io.t[0], a);
  if (io.t[1].mode != T_NONE) v += eval_term(io.t[1], a);
  return v;
}

// address of (line L, position 0) of an array whose direction-DIR extent is n
template <int DIR>
__device__ __forceinline__ int64_t line_base(int L, int n, int n1) {
  if (DIR == 0) return (int64_t)L * n;
  if (DIR == 1) {
    const int k = L / n1, i = L - k * n1;
    return (int64_t)k * n * n1 + i;
  }
  return (int64_t)L;  // DIR == 2: L = i + n1*j
}
template <int DIR>
__device__ __forceinline__ int64_t pos_stride(int n1, int n2) {
  return DIR == 0 ? 1 : (DIR == 1 ? (int64_t)n1 : (int64_t)n1 * n2);
}

constexpr int kStageBatch = 8;

template <typename T, int DIR, int FAM>
__global__ void __launch_bounds__(256) line_op_kernel(const __grid_constant__ OpPlan P,
                                                      const __grid_constant__ LineIOT<T> io,
                                                      const double* __restrict__ table, int nlines, int LT) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s = reinterpret_cast<T*>(smem_raw);
  const int nin = P.nin, nout = P.nout;
  const int nmax = nin > nout ? nin : nout;
  const int ld = LT + 1;
  T* sa = s + (size_t)nmax * ld;  // LHS a
  T* sc = sa + nmax;              // LHS c'
  T* sd = sc + nmax;              // LHS 1/pivot
  T* sx = sd + nmax;              // cyclic correction x1
  T* sm = sx + nmax;              // y metric
  const int L0 = blockIdx.x * LT;
  const int nt = blockDim.x;
  const int tid = threadIdx.x;
  const int64_t ps = pos_stride<DIR>(io.n1, io.n2);

  // ---- stage the tile; loads are issued in batches of kStageBatch per thread so that enough
  // of them are in flight to cover HBM latency
  if (DIR == 0) {
    // LT consecutive rows are one contiguous run of LT*nin values
    const int tot = LT * nin;
    const int64_t g0 = (int64_t)L0 * nin;
    const int64_t gmax = (int64_t)nlines * nin;
    for (int e0 = tid; e0 < tot; e0 += kStageBatch * nt) {
      T v[kStageBatch];
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * nt;
        v[u] = (e < tot && g0 + e < gmax) ? eval_expr(io, g0 + e) : T(0);
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int e = e0 + u * nt;
        if (e < tot) {
          const int l = e / nin, p = e - l * nin;
          s[p * ld + l] = v[u];
        }
      }
    }
  } else {
    // each thread owns one line of the tile (nt is a multiple of LT)
    const int l = tid % LT;
    const int L = L0 + l;
    const bool ok = L < nlines;
    const int64_t base = ok ? line_base<DIR>(L, nin, io.n1) : 0;
    const int step = nt / LT;
    for (int p0 = tid / LT; p0 < nin; p0 += kStageBatch * step) {
      T v[kStageBatch];
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int p = p0 + u * step;
        v[u] = (ok && p < nin) ? eval_expr(io, base + p * ps) : T(0);
      }
#pragma unroll
      for (int u = 0; u < kStageBatch; ++u) {
        const int p = p0 + u * step;
        if (p < nin) s[p * ld + l] = v[u];
      }
    }
  }
  for (int p = tid; p < nout; p += nt) {
    if (P.tdma) {
      sa[p] = T(table[P.la + p]);
      sc[p] = T(table[P.lc + p]);
      sd[p] = T(table[P.ld + p]);
      sx[p] = T(table[P.lx1 + p]);
    }
    if (P.lmap >= 0) sm[p] = T(table[P.lmap + p]);
  }
  __syncthreads();

  const T dd = T(P.dd), r1 = T(P.r1), r2 = T(P.r2);
  if (P.tdma) {
    // ---- compact scheme: one thread per line builds the RHS (5-point register window) and runs
    // the Thomas forward sweep in place, then the backward sweep and the cyclic closure
    const int l = tid;
    const int L = L0 + l;
    if (l < LT && L < nlines) {
      T* col = s + l;
      T sv[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) sv[k] = k < P.nspec ? special_at(P.sp[k], col, ld, io.fbc, nlines, L) * dd : T(0);
      const int nsw = (P.tdma == 2) ? nout - 1 : nout;
      T w0 = T(0), w1 = T(0), w2 = col[0], w3 = col[ld], w4;
      T yprev = T(0);
      const T b1 = T(P.b1);
      // shared-memory values are loaded one or two rows ahead of the recurrence (the input rows
      // i + 3 and i + 4 are not yet overwritten at row i), so that no load sits on its chain
      T wa = (2 < nin) ? col[2 * ld] : T(0), wb = (3 < nin) ? col[3 * ld] : T(0);
      T a1 = sa[0], d1 = sd[0];  // a_i, 1/pivot_i of the current row (row 0 divides by b_1)
      for (int i = 0; i < nout; ++i) {
        w4 = wa;
        wa = wb;
        wb = (i + 4 < nin) ? col[(i + 4) * ld] : T(0);
        const T ai = a1, di = d1;
        if (i + 1 < nsw) {
          a1 = sa[i + 1];
          d1 = sd[i + 1];
        }
        T r;
        if (i >= P.b_lo && i <= P.b_hi) {
          if (FAM == M1P2C) r = r1 * (w2 + w3) + r2 * (w1 + w4);
          else if (FAM == M1C2P) r = r1 * (w2 + w1) + r2 * (w3 + w0);
          else if (FAM == D1C2C || FAM == D1P2P) r = r1 * (w3 - w1) + r2 * (w4 - w0);
          else if (FAM == D1C2P) r = r1 * (w2 - w1) + r2 * (w3 - w0);
          else r = r1 * (w3 - w2) + r2 * (w4 - w1);
          r = r * dd;
        } else {
          r = T(0);
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (k < P.nspec && P.sp[k].row == i) r = sv[k];
        }
        T y = r;
        if (i < nsw) {
          y = (i == 0) ? r / b1 : (r - ai * yprev) * di;
          yprev = y;
        }
        col[i * ld] = y;
        w0 = w1; w1 = w2; w2 = w3; w3 = w4;
      }
      T xn = col[(nsw - 1) * ld];
      T cv = nsw >= 2 ? col[(nsw - 2) * ld] : T(0), cc = nsw >= 2 ? sc[nsw - 2] : T(0);
      for (int i = nsw - 2; i >= 0; --i) {
        const T vi = cv, ci = cc;
        if (i > 0) {
          cv = col[(i - 1) * ld];
          cc = sc[i - 1];
        }
        const T x = vi - ci * xn;
        col[i * ld] = x;
        xn = x;
      }
      if (P.tdma == 2) {
        const T rn = col[(nout - 1) * ld];
        col[(nout - 1) * ld] = (rn - T(P.cn) * col[0] - T(P.an) * col[(nout - 2) * ld]) * T(P.inv_den);
      }
    }
    __syncthreads();
  }

  // ---- store (explicit schemes compute every row here, in parallel)
  auto finish = [&](int l, int p, int L) -> T {
    T v;
    if (P.tdma) {
      v = s[p * ld + l];
      if (P.tdma == 2 && p < nout - 1) v += sx[p] * s[(nout - 1) * ld + l];
    } else {
      const T* col = s + l;
      if (p >= P.b_lo && p <= P.b_hi) {
        v = bulk_at<FAM>(col, ld, p, r1, r2) * dd;
      } else {
        v = T(0);
        for (int k = 0; k < P.nspec; ++k)
          if (P.sp[k].row == p) v = special_at(P.sp[k], col, ld, io.fbc, nlines, L) * dd;
      }
    }
    if (P.lmap >= 0) v *= sm[p];
    if (P.neu1 && p == 0) v = io.fbc[L];
    if (P.neu2 && p == nout - 1) v = io.fbc[nlines + L];
    return v;
  };
  const T g = T(io.g);
  if (DIR == 0) {
    const int tot = LT * nout;
    const int64_t g0 = (int64_t)L0 * nout;
    for (int e = tid; e < tot; e += nt) {
      const int l = e / nout, p = e - l * nout;
      const int L = L0 + l;
      if (L >= nlines) break;
      const T v = finish(l, p, L);
      const int64_t a = g0 + e;
      store_out(io, a, g, v);
    }
  } else {
    const int l = tid % LT;
    const int L = L0 + l;
    if (L < nlines) {
      const int64_t base = line_base<DIR>(L, nout, io.n1);
      for (int p = tid / LT; p < nout; p += nt / LT) {
        const T v = finish(l, p, L);
        const int64_t a = base + p * ps;
        store_out(io, a, g, v);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Explicit operators (no line solve): one thread per output value, flattened over the output
// array in memory order so that loads and stores are coalesced.  Neighbour values along the
// line come from L1/L2; every row is independent.
// ---------------------------------------------------------------------------

// Each thread owns one (i, j) position of the output plane and kStencilPlanes consecutive k
// planes, so the index decomposition and the per-launch constants are paid once per
// kStencilPlanes outputs and the loads of the planes are independent.
constexpr int kStencilPlanes = 1;

template <typename T, int DIR, int FAM>
__global__ void __launch_bounds__(512) stencil_op_kernel(const __grid_constant__ OpPlan P,
                                                         const __grid_constant__ LineIOT<T> io,
                                                         const double* __restrict__ table, int nlines, int m1,
                                                         int m2, int m3) {
  // output array (m1, m2, m3), x fastest: blockIdx.y covers groups of k planes, the x grid the
  // (i, j) plane
  const int nin = P.nin, nout = P.nout;
  const int plane = m1 * m2;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= plane) return;
  const int j = q / m1;
  const int i = q - j * m1;
  const T dd = T(P.dd), r1 = T(P.r1), r2 = T(P.r2), g = T(io.g);
  const int k0 = blockIdx.y * kStencilPlanes;
  // all planes' values first, then the stores: the inputs never alias the output, so the loads of
  // the kStencilPlanes planes are all in flight together
  T vals[kStencilPlanes];
  int Ls[kStencilPlanes], ps[kStencilPlanes];
#pragma unroll
  for (int kk = 0; kk < kStencilPlanes; ++kk) {
    const int k = k0 + kk < m3 ? k0 + kk : m3 - 1;
    int p, L, ibase, istride;
    if (DIR == 0) {
      p = i;
      L = j + m2 * k;
      ibase = L * nin;
      istride = 1;
    } else if (DIR == 1) {
      p = j;
      L = i + m1 * k;
      ibase = k * nin * m1 + i;
      istride = m1;
    } else {
      p = k;
      L = q;
      ibase = q;
      istride = plane;
    }
    auto f = [&](int qq) -> T { return eval_expr32(io, ibase + qq * istride); };
    T v;
    if (P.wrap) {
      auto fw = [&](int qq) -> T { return f(qq < 0 ? qq + nin : (qq >= nin ? qq - nin : qq)); };
      v = bulk_fn<FAM>(fw, p, r1, r2) * dd;
    } else if (p >= P.b_lo && p <= P.b_hi) {
      v = bulk_fn<FAM>(f, p, r1, r2) * dd;
    } else {
      v = T(0);
      for (int s = 0; s < P.nspec; ++s) {
        if (P.sp[s].row != p) continue;
        const SpecialRow& R = P.sp[s];
        T acc = T(0);
        for (int t = 0; t < R.nt; ++t) acc += T(R.w[t]) * f(R.idx[t]);
        for (int u = 0; u < 4; ++u)
          if (R.wb[u] != 0.0) acc += T(R.wb[u]) * io.fbc[u * nlines + L];
        v = acc * dd;
      }
    }
    vals[kk] = v;
    Ls[kk] = L;
    ps[kk] = p;
  }
#pragma unroll
  for (int kk = 0; kk < kStencilPlanes; ++kk) {
    const int k = k0 + kk;
    if (k >= m3) break;
    const int p = ps[kk], L = Ls[kk];
    T v = vals[kk];
    if (P.lmap >= 0) v *= T(table[P.lmap + p]);
    if (P.neu1 && p == 0) v = io.fbc[L];
    if (P.neu2 && p == nout - 1) v = io.fbc[nlines + L];
    store_out(io, (int64_t)(plane * k + q), g, v);
  }
}

template <typename T, int DIR>
static void launch_stencil_dir(const OpPlan& P, const LineIOT<T>& io, const double* table, cudaStream_t st,
                               int nlines) {
  int m[3] = {io.n1, io.n2, io.n3};
  m[DIR] = P.nout;
  const int64_t nin_tot = (int64_t)io.n1 * io.n2 * io.n3, nout_tot = (int64_t)m[0] * m[1] * m[2];
  if (nin_tot >= 0x7fffffff || nout_tot >= 0x7fffffff)
    throw std::runtime_error("explicit operator: arrays of 2^31 or more values are not supported");
  if (io.block == 0 && try_launch_win<T, DIR>(P, io, table, st, nlines)) return;
  const int plane = m[0] * m[1];
  const int bs = (io.block == 128 || io.block == 512) ? io.block : 256;  // tunable CTA size
  dim3 grid((unsigned)((plane + bs - 1) / bs), (unsigned)((m[2] + kStencilPlanes - 1) / kStencilPlanes));
  switch (P.fam) {
#define CHS_CASE(F)                                                                                 \
  case F:                                                                                           \
    stencil_op_kernel<T, DIR, F><<<grid, bs, 0, st>>>(P, io, table, nlines, m[0], m[1], m[2]);      \
    break;
    CHS_CASE(D1C2C)
    CHS_CASE(D1P2P)
    CHS_CASE(D1C2P)
    CHS_CASE(D1P2C)
    CHS_CASE(M1C2P)
    CHS_CASE(M1P2C)
#undef CHS_CASE
    default: throw std::runtime_error("bad family");
  }
}

// ---------------------------------------------------------------------------
// Fused explicit operators: one pass computes sum_m g_m op_m(in_m) at every output value and
// applies the epilogue (store, RK3 fractional step, or the energy update with the property
// lookup).  Each term is evaluated like stencil_op_kernel evaluates one output value.
// ---------------------------------------------------------------------------
template <typename T, int DIR, int FAM>
__device__ __forceinline__ T fused_term_at(const FusedTerm<T>& ft, const double* __restrict__ table, int i, int j,
                                           int k) {
  const OpPlan& P = ft.P;
  const int nin = P.nin, nout = P.nout;
  int p, L, ibase, istride;
  if (DIR == 0) {
    p = i;
    L = j + ft.n2 * k;
    ibase = L * nin;
    istride = 1;
  } else if (DIR == 1) {
    p = j;
    L = i + ft.n1 * k;
    ibase = k * nin * ft.n1 + i;
    istride = ft.n1;
  } else {
    p = k;
    L = i + ft.n1 * j;
    ibase = L;
    istride = ft.n1 * ft.n2;
  }
  auto f = [&](int qq) -> T {
    const int a = ibase + qq * istride;
    T v = eval_term32(ft.t[0], a);
    if (ft.t[1].mode != T_NONE) v += eval_term32(ft.t[1], a);
    return v;
  };
  const T dd = T(P.dd);
  T v;
  if (p >= P.b_lo && p <= P.b_hi) {
    v = bulk_fn<FAM>(f, p, T(P.r1), T(P.r2)) * dd;
  } else {
    v = T(0);
    for (int s = 0; s < P.nspec; ++s) {
      if (P.sp[s].row != p) continue;
      const SpecialRow& R = P.sp[s];
      T acc = T(0);
      for (int t = 0; t < R.nt; ++t) acc += T(R.w[t]) * f(R.idx[t]);
      for (int u = 0; u < 4; ++u)
        if (R.wb[u] != 0.0) acc += T(R.wb[u]) * ft.fbc[u * ft.nlines + L];
      v = acc * dd;
    }
  }
  if (P.lmap >= 0) v *= T(table[P.lmap + p]);
  if (P.neu1 && p == 0) v = ft.fbc[L];
  if (P.neu2 && p == nout - 1) v = ft.fbc[ft.nlines + L];
  return v;
}

template <typename T>
__global__ void __launch_bounds__(256) fused_kernel(const __grid_constant__ FusedIO<T> F,
                                                    const double* __restrict__ table) {
  const int plane = F.m1 * F.m2;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= plane) return;
  const int k = blockIdx.y;
  const int j = q / F.m1;
  const int i = q - j * F.m1;
  T sum0 = T(0), sum1 = T(0);
  for (int mt = 0; mt < F.nterm; ++mt) {
    const FusedTerm<T>& ft = F.term[mt];
    T v;
    switch (ft.dir * 8 + ft.P.fam) {
      case 0 * 8 + D1C2P: v = fused_term_at<T, 0, D1C2P>(ft, table, i, j, k); break;
      case 1 * 8 + D1C2P: v = fused_term_at<T, 1, D1C2P>(ft, table, i, j, k); break;
      case 2 * 8 + D1C2P: v = fused_term_at<T, 2, D1C2P>(ft, table, i, j, k); break;
      case 0 * 8 + D1P2C: v = fused_term_at<T, 0, D1P2C>(ft, table, i, j, k); break;
      case 1 * 8 + D1P2C: v = fused_term_at<T, 1, D1P2C>(ft, table, i, j, k); break;
      case 2 * 8 + D1P2C: v = fused_term_at<T, 2, D1P2C>(ft, table, i, j, k); break;
      default: v = T(0);
    }
    const T gv = T(ft.g) * v;
    if (ft.group == 0) sum0 = sum0 + gv;
    else sum1 = sum1 + gv;
  }
  const int64_t o = (int64_t)plane * k + q;
  if (F.epilogue == EP_STORE) {
    F.out[o] = sum0;
  } else if (F.epilogue == EP_ACCUM) {
    F.out[o] = F.out[o] + sum0;
  } else if (F.epilogue == EP_FRAC) {
    const T last = F.rhs0[o];
    T tot = T(F.gam) * sum0 + T(F.zeta) * last;
    F.rhs0[o] = sum0;
    tot = tot + T(F.alpha) * sum1;
    F.out[o] = T(F.dt) * tot;
  } else {  // EP_ENERGY
    const T last = F.rhs0[o];
    const T tot = T(F.gam) * sum0 + T(F.zeta) * last;
    F.rhs0[o] = sum0;
    const T r1 = T(F.dt) * tot;
    const T rh = F.rhoh[o] + r1;
    F.rhoh[o] = rh;
    if (F.props) {
      const CellProps pr = props_from_dh(F.tab, (double)rh);
      F.h[o] = T(pr.h);
      F.t[o] = T(pr.t);
      F.k[o] = T(pr.k);
      F.d[o] = T(pr.d);
      F.m[o] = T(pr.m);
    }
  }
}

// input-expression term with its mode known at compile time
template <int M, typename T>
__device__ __forceinline__ T eval_term_ct(const TermT<T>& t, int a) {
  if (M == T_X) return T(t.s) * t.X[a];
  if (M == T_XY) return T(t.s) * (t.X[a] * t.Y[a]);
  if (M == T_XpY) return T(t.s) * (t.X[a] + T(t.c) * t.Y[a]);
  if (M == T_XpYZ) return T(t.s) * (t.X[a] + T(t.c) * t.Y[a]) * t.Z[a];
  return T(0);
}

// bulk row of one term (the caller has checked that p is a bulk row): straight-line code with
// unconditional loads, the second stencil pair only when R2
template <typename T, int DIR, int FAM, bool R2, int M0, int M1>
__device__ __forceinline__ T bulk_term(const FusedTerm<T>& ft, const double* __restrict__ table, int i, int j,
                                       int k) {
  const OpPlan& P = ft.P;
  const int nin = P.nin;
  int p, ibase, istride;
  if (DIR == 0) {
    p = i;
    ibase = (j + ft.n2 * k) * nin;
    istride = 1;
  } else if (DIR == 1) {
    p = j;
    ibase = k * nin * ft.n1 + i;
    istride = ft.n1;
  } else {
    p = k;
    ibase = i + ft.n1 * j;
    istride = ft.n1 * ft.n2;
  }
  const bool wrap = P.wrap;
  auto f = [&](int qq) -> T {
    if (wrap) qq = qq < 0 ? qq + nin : (qq >= nin ? qq - nin : qq);
    const int a = ibase + qq * istride;
    T v = eval_term_ct<M0>(ft.t[0], a);
    if (M1 != T_NONE) v += eval_term_ct<M1>(ft.t[1], a);
    return v;
  };
  const T r1 = T(P.r1), r2 = T(P.r2);
  T v;
  if (FAM == D1C2P) {
    v = r1 * (f(p) - f(p - 1));
    if (R2) v += r2 * (f(p + 1) - f(p - 2));
  } else {  // D1P2C
    v = r1 * (f(p + 1) - f(p));
    if (R2) v += r2 * (f(p + 2) - f(p - 1));
  }
  v = v * T(P.dd);
  if (P.lmap >= 0) v *= T(table[P.lmap + p]);
  return v;
}

template <int DIR>
__device__ __forceinline__ int term_pos(int i, int j, int k) {
  return DIR == 0 ? i : (DIR == 1 ? j : k);
}

// epilogue shared by the generic and the specialised fused kernels
template <typename T>
__device__ __forceinline__ void fused_epilogue(const FusedIO<T>& F, int64_t o, T sum0, T sum1) {
  if (F.epilogue == EP_STORE) {
    F.out[o] = sum0;
  } else if (F.epilogue == EP_ACCUM) {
    F.out[o] = F.out[o] + sum0;
  } else if (F.epilogue == EP_FRAC) {
    const T last = F.rhs0[o];
    T tot = T(F.gam) * sum0 + T(F.zeta) * last;
    F.rhs0[o] = sum0;
    tot = tot + T(F.alpha) * sum1;
    F.out[o] = T(F.dt) * tot;
  } else {
    const T last = F.rhs0[o];
    const T tot = T(F.gam) * sum0 + T(F.zeta) * last;
    F.rhs0[o] = sum0;
    const T r1 = T(F.dt) * tot;
    const T rh = F.rhoh[o] + r1;
    F.rhoh[o] = rh;
    if (F.props) {
      const CellProps pr = props_from_dh(F.tab, (double)rh);
      F.h[o] = T(pr.h);
      F.t[o] = T(pr.t);
      F.k[o] = T(pr.k);
      F.d[o] = T(pr.d);
      F.m[o] = T(pr.m);
    }
  }
}

// Specialisation for a term list known at compile time (the signatures the substep uses): every
// term is evaluated inline, so the loads of all terms can be in flight together.
template <int D, int FM, int M0, int M1 = T_NONE>
struct TermSig {
  static constexpr int dir = D, fam = FM, m0 = M0, m1 = M1;
};

template <typename T, bool R2, typename... S>
__global__ void __launch_bounds__(256) fused_kernel_sig(const __grid_constant__ FusedIO<T> F,
                                                        const double* __restrict__ table) {
  const int plane = F.m1 * F.m2;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= plane) return;
  const int k = blockIdx.y;
  const int j = q / F.m1;
  const int i = q - j * F.m1;
  constexpr int N = sizeof...(S);
  T v[N];
  // bulk rows of every term (nearly all outputs): branch-free evaluation so the loads of all
  // terms can be issued together; boundary rows take the general path
  bool bulk = true;
  {
    int idx = 0;
    ((bulk = bulk && (F.term[idx].P.wrap || (term_pos<S::dir>(i, j, k) >= F.term[idx].P.b_lo &&
                                              term_pos<S::dir>(i, j, k) <= F.term[idx].P.b_hi &&
                                              !F.term[idx].P.neu1 && !F.term[idx].P.neu2)),
      ++idx),
     ...);
  }
  if (bulk) {
    int idx = 0;
    ((v[idx] = bulk_term<T, S::dir, S::fam, R2, S::m0, S::m1>(F.term[idx], table, i, j, k), ++idx), ...);
  } else {
    int idx = 0;
    ((v[idx] = fused_term_at<T, S::dir, S::fam>(F.term[idx], table, i, j, k), ++idx), ...);
  }
  T sum0 = T(0), sum1 = T(0);
#pragma unroll
  for (int t = 0; t < N; ++t) {
    const T gv = T(F.term[t].g) * v[t];
    if (F.term[t].group == 0) sum0 = sum0 + gv;
    else sum1 = sum1 + gv;
  }
  fused_epilogue(F, (int64_t)plane * k + q, sum0, sum1);
}

template <typename T, typename... S>
static bool try_sig(const FusedIO<T>& f, const double* table, cudaStream_t st, dim3 grid) {
  constexpr int N = sizeof...(S);
  if (f.nterm != N) return false;
  const int dirs[N] = {S::dir...};
  const int fams[N] = {S::fam...};
  const int m0s[N] = {S::m0...};
  const int m1s[N] = {S::m1...};
  bool r2 = false;
  for (int t = 0; t < N; ++t) {
    if (f.term[t].dir != dirs[t] || f.term[t].P.fam != fams[t]) return false;
    if (f.term[t].t[0].mode != m0s[t] || f.term[t].t[1].mode != m1s[t]) return false;
    if (f.term[t].P.r2 != 0.0) r2 = true;
  }
  if (r2) fused_kernel_sig<T, true, S...><<<grid, 256, 0, st>>>(f, table);
  else fused_kernel_sig<T, false, S...><<<grid, 256, 0, st>>>(f, table);
  return true;
}

template <typename T>
void launch_fused(const FusedIO<T>& f, const double* table, cudaStream_t st) {
  if (f.nterm < 1 || f.nterm > kMaxFusedTerms) throw std::runtime_error("fused operator: bad term count");
  if ((int64_t)f.m1 * f.m2 * f.m3 >= 0x7fffffff || f.m3 > 65535)
    throw std::runtime_error("fused operator: array extents out of range");
  for (int t = 0; t < f.nterm; ++t) {
    const FusedTerm<T>& ft = f.term[t];
    if (ft.P.tdma) throw std::runtime_error("fused operator: compact (line-solve) plans cannot be fused");
    if (ft.P.fam != D1C2P && ft.P.fam != D1P2C) throw std::runtime_error("fused operator: unsupported family");
    if ((int64_t)ft.n1 * ft.n2 * ft.n3 >= 0x7fffffff) throw std::runtime_error("fused operator: input too large");
  }
  const int plane = f.m1 * f.m2;
  dim3 grid((unsigned)((plane + 255) / 256), (unsigned)f.m3);
  // momentum terms: conv (X*Y) + diffusion (X + cY, times mu for variable properties); pressure
  // gradient (X); divergence (X); energy conv and diffusion (X*Y)
  using XC0 = TermSig<0, D1C2P, T_XY, T_XpY>;
  using XC1 = TermSig<1, D1C2P, T_XY, T_XpY>;
  using XC2 = TermSig<2, D1C2P, T_XY, T_XpY>;
  using XP0 = TermSig<0, D1P2C, T_XY, T_XpY>;
  using XP1 = TermSig<1, D1P2C, T_XY, T_XpY>;
  using XP2 = TermSig<2, D1P2C, T_XY, T_XpY>;
  using ZC0 = TermSig<0, D1C2P, T_XY, T_XpYZ>;
  using ZC1 = TermSig<1, D1C2P, T_XY, T_XpYZ>;
  using ZC2 = TermSig<2, D1C2P, T_XY, T_XpYZ>;
  using ZP0 = TermSig<0, D1P2C, T_XY, T_XpYZ>;
  using ZP1 = TermSig<1, D1P2C, T_XY, T_XpYZ>;
  using ZP2 = TermSig<2, D1P2C, T_XY, T_XpYZ>;
  using GC0 = TermSig<0, D1C2P, T_X>;
  using GC1 = TermSig<1, D1C2P, T_X>;
  using GC2 = TermSig<2, D1C2P, T_X>;
  using DP0 = TermSig<0, D1P2C, T_X>;
  using DP1 = TermSig<1, D1P2C, T_X>;
  using DP2 = TermSig<2, D1P2C, T_X>;
  using EP0 = TermSig<0, D1P2C, T_XY, T_XY>;
  using EP1 = TermSig<1, D1P2C, T_XY>;
  using EP2 = TermSig<2, D1P2C, T_XY, T_XY>;
  if (try_sig<T, XC0, XP1, XP2, GC0>(f, table, st, grid)) return;
  if (try_sig<T, XP0, XC1, XP2, GC1>(f, table, st, grid)) return;
  if (try_sig<T, XP0, XP1, XC2, GC2>(f, table, st, grid)) return;
  if (try_sig<T, ZC0, ZP1, ZP2, GC0>(f, table, st, grid)) return;
  if (try_sig<T, ZP0, ZC1, ZP2, GC1>(f, table, st, grid)) return;
  if (try_sig<T, ZP0, ZP1, ZC2, GC2>(f, table, st, grid)) return;
  if (try_sig<T, DP0, DP1, DP2>(f, table, st, grid)) return;
  if (try_sig<T, EP0, EP1, EP1, EP2>(f, table, st, grid)) return;
  fused_kernel<T><<<grid, 256, 0, st>>>(f, table);
}
template void launch_fused<double>(const FusedIO<double>&, const double*, cudaStream_t);
template void launch_fused<float>(const FusedIO<float>&, const double*, cudaStream_t);

constexpr int kLineSmemMax = 200 * 1024;

template <typename T, int DIR>
static void launch_dir(const OpPlan& P, const LineIOT<T>& io, const double* table, cudaStream_t st, int nlines,
                       int LT, size_t shm) {
  dim3 grid((unsigned)((nlines + LT - 1) / LT));
  dim3 block(256);
  switch (P.fam) {
#define CHS_CASE(F)                                                                                   \
  case F: {                                                                                           \
    static bool attr_set = false;                                                                     \
    if (!attr_set) {                                                                                  \
      cudaFuncSetAttribute(line_op_kernel<T, DIR, F>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                           kLineSmemMax);                                                             \
      attr_set = true;                                                                                \
    }                                                                                                 \
    line_op_kernel<T, DIR, F><<<grid, block, shm, st>>>(P, io, table, nlines, LT);                    \
    break;                                                                                            \
  }
    CHS_CASE(D1C2C)
    CHS_CASE(D1P2P)
    CHS_CASE(D1C2P)
    CHS_CASE(D1P2C)
    CHS_CASE(M1C2P)
    CHS_CASE(M1P2C)
#undef CHS_CASE
    default: throw std::runtime_error("bad family");
  }
}

template <typename T>
void launch_line_op_t(int d, const OpPlan& P, const LineIOT<T>& io, const double* table, cudaStream_t st) {
  int n_in3[3] = {io.n1, io.n2, io.n3};
  if (n_in3[d] != P.nin) throw std::runtime_error("line operator: input extent does not match the plan");
  const int64_t nl = num_lines(d, io.n1, io.n2, io.n3);
  if (nl > 0x7fffffff) throw std::runtime_error("line operator: too many lines");
  const int nlines = (int)nl;
  if (!P.tdma) {
    // explicit scheme: every output row is independent
    if (d == 0) launch_stencil_dir<T, 0>(P, io, table, st, nlines);
    else if (d == 1) launch_stencil_dir<T, 1>(P, io, table, st, nlines);
    else launch_stencil_dir<T, 2>(P, io, table, st, nlines);
    return;
  }
  const int nmax = P.nin > P.nout ? P.nin : P.nout;
  // up to 64 lines per CTA, fewer while the tile exceeds ~45 KB so that four or more CTAs
  // (32+ warps) stay resident per SM
  int LT = (io.lt_max == 16 || io.lt_max == 32) ? io.lt_max : 64;  // tunable lines per CTA
  while (LT > 16 && ((size_t)nmax * (LT + 1) + 5 * (size_t)nmax) * sizeof(T) > 45 * 1024) LT /= 2;
  // and fewer while the grid would not give every SM two CTAs (small grids: a CTA's sweep is the
  // latency of its lines' recurrences, whatever their number)
  while (LT > 16 && (nlines + LT - 1) / LT < 2 * 148) LT /= 2;
  const size_t shm = ((size_t)nmax * (LT + 1) + 5 * (size_t)nmax) * sizeof(T);
  if (shm > (size_t)kLineSmemMax) throw std::runtime_error("line operator: line too long for the shared-memory tile");
  if (d == 0) launch_dir<T, 0>(P, io, table, st, nlines, LT, shm);
  else if (d == 1) launch_dir<T, 1>(P, io, table, st, nlines, LT, shm);
  else launch_dir<T, 2>(P, io, table, st, nlines, LT, shm);
}

void launch_line_op(int d, const OpPlan& P, const LineIO& io, const double* table, cudaStream_t st) {
  launch_line_op_t<double>(d, P, io, table, st);
}
void launch_line_op(int d, const OpPlan& P, const LineIOT<float>& io, const double* table, cudaStream_t st) {
  launch_line_op_t<float>(d, P, io, table, st);
}

// ===========================================================================
// Stockham FFT in shared memory (radix 2, 3, 4), several lines per CTA
// ===========================================================================
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// complex element type of the transforms: double2 (the FP64 path) or float2 (the FP32 spectrum of the
// mixed-precision FISHPACK solver); S its scalar, mk its constructor, tw the plan's twiddles
template <typename C>
struct Cplx;
template <>
struct Cplx<double2> {
  using S = double;
  __device__ static double2 mk(double x, double y) { return make_double2(x, y); }
  __device__ static const double2* tw(const FftPlan& fp) { return fp.tw; }
};
template <>
struct Cplx<float2> {
  using S = float;
  __device__ static float2 mk(float x, float y) { return make_float2(x, y); }
  __device__ static const float2* tw(const FftPlan& fp) { return fp.twf; }
};

// x / d for 0 <= x < 2^23 from a float reciprocal of d with one correction step (the float
// estimate is within one of the quotient there); avoids an integer division per butterfly
__device__ __forceinline__ int fast_div(int x, int d, float inv) {
  int q = __float2int_rz((float)x * inv);
  const int r = x - q * d;
  if (r >= d) ++q;
  else if (r < 0) --q;
  return q;
}

// one radix-R butterfly column of a Stockham stage: column j = jq * ns + k (k < ns), input stride
// n / R, twiddle step n / (ns R); k * r * tstep < n, so the twiddle index needs no reduction
template <int R, typename C>
__device__ __forceinline__ void stockham_bfly(const C* in, C* out, int j, int jq, int k, int stride, int ns,
                                              int tstep, const C* tw, int sign) {
  using S = typename Cplx<C>::S;
  C v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    C x = in[j + r * stride];
    if (r > 0 && k > 0) {
      C t = tw[k * r * tstep];
      if (sign > 0) t.y = -t.y;
      x = cmul(x, t);
    }
    v[r] = x;
  }
  const S sg = (S)sign;
  if (R == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    C b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
    C ib1 = Cplx<C>::mk(-sg * b1.y, sg * b1.x);  // (i*sign) * b1
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, ib1);
    v[3] = csub(a1, ib1);
  } else {  // R == 3
    const S h = (S)0.86602540378443864676;  // sqrt(3)/2
    C t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    C m = Cplx<C>::mk(v[0].x - (S)0.5 * t1.x, v[0].y - (S)0.5 * t1.y);
    C it2 = Cplx<C>::mk(-sg * h * t2.y, sg * h * t2.x);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, it2);
    v[2] = csub(m, it2);
  }
  const int idxd = jq * ns * R + k;
#pragma unroll
  for (int r = 0; r < R; ++r) out[idxd + r * ns] = v[r];
}

// FFT of `nl` lines of length n stored in buf0 with line stride ls (n, or n + 1 where the line
// loads and stores run across lines: the padding moves consecutive lines to different banks);
// result in buf0 or buf1 (returned).  All threads of the CTA take part.
template <typename C>
__device__ C* smem_fft(C* buf0, C* buf1, int nl, const FftPlan& fp, int sign, int ls = 0) {
  const int n = fp.n;
  if (ls == 0) ls = n;
  int ns = 1;
  C* in = buf0;
  C* out = buf1;
  const C* tw = Cplx<C>::tw(fp);
  for (int s = 0; s < fp.nst; ++s) {
    const int R = fp.radix[s];
    const int nb = n / R, tstep = n / (ns * R);
    const float inb = 1.0f / (float)nb, ins = 1.0f / (float)ns;
    for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
      const int line = fast_div(t, nb, inb), j = t - line * nb;
      const int jq = fast_div(j, ns, ins), k = j - jq * ns;
      const C* li = in + line * ls;
      C* lo = out + line * ls;
      if (R == 4) stockham_bfly<4, C>(li, lo, j, jq, k, nb, ns, tstep, tw, sign);
      else if (R == 2) stockham_bfly<2, C>(li, lo, j, jq, k, nb, ns, tstep, tw, sign);
      else stockham_bfly<3, C>(li, lo, j, jq, k, nb, ns, tstep, tw, sign);
    }
    __syncthreads();
    ns *= R;
    C* tmp = in; in = out; out = tmp;
  }
  return in;
}

static int fft_lines_per_cta(int n) {
  int l = 2048 / n;
  if (l < 1) l = 1;
  if (l > 32) l = 32;
  return l;
}

// real rows -> half spectra; two real rows per complex transform (rows of type R, FP64 transform)
template <typename R, typename C>
__global__ void rfft_x_kernel(const __grid_constant__ FftPlan fp, const R* __restrict__ in, C* __restrict__ out,
                              int nrows, int lpc) {
  using S = typename Cplx<C>::S;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  C* sh = reinterpret_cast<C*>(fft_smem);
  const int n = fp.n, nh = n / 2 + 1;
  C* b0 = sh;
  C* b1 = sh + (size_t)lpc * n;
  const int pair0 = blockIdx.x * lpc;
  const float inn = 1.0f / (float)n, innh = 1.0f / (float)nh;
  for (int t0 = threadIdx.x; t0 < lpc * n; t0 += 4 * blockDim.x) {
    S a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      a[u] = S(0);
      b[u] = S(0);
      if (t < lpc * n) {
        const int l = fast_div(t, n, inn), p = t - l * n;
        const int ra = 2 * (pair0 + l), rb = ra + 1;
        if (ra < nrows) a[u] = (S)in[(int64_t)ra * n + p];
        if (rb < nrows) b[u] = (S)in[(int64_t)rb * n + p];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < lpc * n) b0[t] = Cplx<C>::mk(a[u], b[u]);
    }
  }
  __syncthreads();
  C* r = smem_fft(b0, b1, lpc, fp, -1);
  for (int t = threadIdx.x; t < lpc * nh; t += blockDim.x) {
    const int l = fast_div(t, nh, innh), k = t - l * nh;
    const int ra = 2 * (pair0 + l), rb = ra + 1;
    const C z = r[l * n + k];
    C zc = r[l * n + (k == 0 ? 0 : n - k)];
    zc.y = -zc.y;
    const C xa = Cplx<C>::mk((S)0.5 * (z.x + zc.x), (S)0.5 * (z.y + zc.y));
    const C d = csub(z, zc);
    const C xb = Cplx<C>::mk((S)0.5 * d.y, (S)-0.5 * d.x);
    if (ra < nrows) out[(int64_t)ra * nh + k] = xa;
    if (rb < nrows) out[(int64_t)rb * nh + k] = xb;
  }
}

template <typename R, typename C>
__global__ void irfft_x_kernel(const __grid_constant__ FftPlan fp, const C* __restrict__ in, R* __restrict__ out,
                               int nrows, double scale, int lpc) {
  using S = typename Cplx<C>::S;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  C* sh = reinterpret_cast<C*>(fft_smem);
  const int n = fp.n, nh = n / 2 + 1;
  C* b0 = sh;
  C* b1 = sh + (size_t)lpc * n;
  const int pair0 = blockIdx.x * lpc;
  const float inn = 1.0f / (float)n;
  for (int t0 = threadIdx.x; t0 < lpc * n; t0 += 4 * blockDim.x) {
    C xa[4], xb[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      xa[u] = Cplx<C>::mk(S(0), S(0));
      xb[u] = Cplx<C>::mk(S(0), S(0));
      if (t < lpc * n) {
        const int l = fast_div(t, n, inn), k = t - l * n;
        const int ra = 2 * (pair0 + l), rb = ra + 1;
        const int kk = k > n / 2 ? n - k : k;
        if (ra < nrows) xa[u] = in[(int64_t)ra * nh + kk];
        if (rb < nrows) xb[u] = in[(int64_t)rb * nh + kk];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < lpc * n) {
        const int k = t - fast_div(t, n, inn) * n;
        const bool hi = k > n / 2;
        const int kk = hi ? n - k : k;
        C A = xa[u], B = xb[u];
        if (kk == 0 || 2 * kk == n) { A.y = S(0); B.y = S(0); }
        if (hi) { A.y = -A.y; B.y = -B.y; }
        b0[t] = Cplx<C>::mk(A.x - B.y, A.y + B.x);  // xa + i*xb
      }
    }
  }
  __syncthreads();
  C* r = smem_fft(b0, b1, lpc, fp, +1);
  const S sc = (S)scale;
  for (int t = threadIdx.x; t < lpc * n; t += blockDim.x) {
    const int l = fast_div(t, n, inn), p = t - l * n;
    const int ra = 2 * (pair0 + l), rb = ra + 1;
    const C z = r[t];
    if (ra < nrows) out[(int64_t)ra * n + p] = R(z.x * sc);
    if (rb < nrows) out[(int64_t)rb * n + p] = R(z.y * sc);
  }
}

template <typename C>
__global__ void cfft_axis_kernel(const __grid_constant__ FftPlan fp, C* __restrict__ data, int na, int nb,
                                 int64_t bstride, int64_t stride, int sign, int lpc) {
  using S = typename Cplx<C>::S;
  extern __shared__ __align__(16) unsigned char fft_smem[];
  C* sh = reinterpret_cast<C*>(fft_smem);
  __shared__ int64_t lbase[32];  // start of each of the CTA's lines (lpc <= 32), -1 past the end
  const int n = fp.n, ls = n + 1;  // padded line stride: the loads and stores run across lines
  C* b0 = sh;
  C* b1 = sh + (size_t)lpc * ls;
  const int64_t g0 = (int64_t)blockIdx.x * lpc;
  const int64_t nlines = (int64_t)na * nb;
  if (threadIdx.x < lpc) {
    const int64_t g = g0 + threadIdx.x;
    if (g < nlines) {
      const int64_t b = g / na, a = g - b * na;
      lbase[threadIdx.x] = a + b * bstride;
    } else {
      lbase[threadIdx.x] = -1;
    }
  }
  __syncthreads();
  const float ilpc = 1.0f / (float)lpc;
  for (int t0 = threadIdx.x; t0 < lpc * n; t0 += 4 * blockDim.x) {
    C v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      v[u] = Cplx<C>::mk(S(0), S(0));
      if (t < lpc * n) {
        const int p = fast_div(t, lpc, ilpc), l = t - p * lpc;
        const int64_t base = lbase[l];
        if (base >= 0) v[u] = data[base + p * stride];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < lpc * n) {
        const int p = fast_div(t, lpc, ilpc), l = t - p * lpc;
        b0[l * ls + p] = v[u];
      }
    }
  }
  __syncthreads();
  C* r = smem_fft(b0, b1, lpc, fp, sign, ls);
  for (int t = threadIdx.x; t < lpc * n; t += blockDim.x) {
    const int p = fast_div(t, lpc, ilpc), l = t - p * lpc;
    const int64_t base = lbase[l];
    if (base >= 0) data[base + p * stride] = r[l * ls + p];
  }
}

template <typename R, typename C>
void launch_rfft_x(const FftPlan& fp, const R* in, C* out, int nrows, cudaStream_t st) {
  const int lpc = fft_lines_per_cta(fp.n);
  const int npairs = (nrows + 1) / 2;
  const size_t shm = 2 * (size_t)lpc * fp.n * sizeof(C);
  cudaFuncSetAttribute(rfft_x_kernel<R, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  rfft_x_kernel<R, C><<<(npairs + lpc - 1) / lpc, 256, shm, st>>>(fp, in, out, nrows, lpc);
}

template <typename R, typename C>
void launch_irfft_x(const FftPlan& fp, const C* in, R* out, int nrows, double scale, cudaStream_t st) {
  const int lpc = fft_lines_per_cta(fp.n);
  const int npairs = (nrows + 1) / 2;
  const size_t shm = 2 * (size_t)lpc * fp.n * sizeof(C);
  cudaFuncSetAttribute(irfft_x_kernel<R, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  irfft_x_kernel<R, C><<<(npairs + lpc - 1) / lpc, 256, shm, st>>>(fp, in, out, nrows, scale, lpc);
}
template void launch_rfft_x<double, double2>(const FftPlan&, const double*, double2*, int, cudaStream_t);
template void launch_rfft_x<float, double2>(const FftPlan&, const float*, double2*, int, cudaStream_t);
template void launch_rfft_x<float, float2>(const FftPlan&, const float*, float2*, int, cudaStream_t);
template void launch_irfft_x<double, double2>(const FftPlan&, const double2*, double*, int, double, cudaStream_t);
template void launch_irfft_x<float, double2>(const FftPlan&, const double2*, float*, int, double, cudaStream_t);
template void launch_irfft_x<float, float2>(const FftPlan&, const float2*, float*, int, double, cudaStream_t);

template <typename C>
void launch_cfft_axis(const FftPlan& fp, C* data, int na, int nb, int64_t bstride, int64_t stride, int sign,
                      cudaStream_t st) {
  const int lpc = fft_lines_per_cta(fp.n);
  const int64_t nlines = (int64_t)na * nb;
  const size_t shm = 2 * (size_t)lpc * (fp.n + 1) * sizeof(C);
  cudaFuncSetAttribute(cfft_axis_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
  cfft_axis_kernel<C><<<(unsigned)((nlines + lpc - 1) / lpc), 256, shm, st>>>(fp, data, na, nb, bstride, stride,
                                                                               sign, lpc);
}
template void launch_cfft_axis<double2>(const FftPlan&, double2*, int, int, int64_t, int64_t, int, cudaStream_t);
template void launch_cfft_axis<float2>(const FftPlan&, float2*, int, int, int64_t, int64_t, int, cudaStream_t);

// ===========================================================================
// FISHPACK y solve: TRID0 (src/poisson_fishpack.f90:20-57) per (kx, kz) on complex data
// laid out (kz, j, kx) with kx fastest.
// ===========================================================================
// The forward-sweep factors of TRID0 depend only on (kx, kz), not on the right-hand side, so
// they are computed once: Zr[j] = 1/pivot_j (j < ny-1), D[j] = c_j * Zr[j], and for the last
// row the pivot itself, or 0 when it is pinned (|pivot| <= 1e-10).  Layout (kz, j, kx) like the
// spectrum.  The arithmetic is TRID0's, in its order, so the solve is bitwise the same.
__global__ void ysolve_factor_kernel(double* __restrict__ Zr, double* __restrict__ D, int nxh, int ny, int nz,
                                     const double* __restrict__ pa, const double* __restrict__ pb,
                                     const double* __restrict__ pc, const double* __restrict__ lamx,
                                     const double* __restrict__ lamz) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nxh * nz) return;
  const int kz = (int)(g / nxh), kx = (int)(g - (int64_t)kz * nxh);
  const double lx = lamx[kx], lz = lamz[kz];
  const int64_t base = (int64_t)kz * ny * nxh + kx;
  double bb = (pb[0] + lx) + lz;
  double Z = 1.0 / bb;
  double d = pc[0] * Z;
  Zr[base] = Z;
  D[base] = d;
  for (int j = 1; j < ny - 1; ++j) {
    bb = (pb[j] + lx) + lz;
    Z = 1.0 / (bb - pa[j] * d);
    d = pc[j] * Z;
    Zr[base + (int64_t)j * nxh] = Z;
    D[base + (int64_t)j * nxh] = d;
  }
  bb = (pb[ny - 1] + lx) + lz;
  Z = bb - pa[ny - 1] * d;
  Zr[base + (int64_t)(ny - 1) * nxh] = fabs(Z) > 1.0e-10 ? Z : 0.0;
  D[base + (int64_t)(ny - 1) * nxh] = 0.0;
}

void launch_ysolve_factor(double* Zr, double* D, int nxh, int ny, int nz, const double* pa, const double* pb,
                          const double* pc, const double* lamx, const double* lamz, cudaStream_t st) {
  if (ny < 2) throw std::runtime_error("ysolve: ny must be at least 2");
  const int64_t n = (int64_t)nxh * nz;
  ysolve_factor_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(Zr, D, nxh, ny, nz, pa, pb, pc, lamx, lamz);
}

// One CTA per `lt` consecutive (kx, kz) columns: the columns and their precomputed factors are
// staged in shared memory with coalesced row loads by all threads (eight loads in flight per
// thread), swept by `lt` threads (one column each), and written back.
// The spectrum is double2 (FP64 path) or float2 (the FP32 spectrum of the mixed-precision path); the
// solve itself always runs in FP64.
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
template <typename C>
__device__ __forceinline__ C from_d2(double2 v);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

template <typename C>
__global__ void __launch_bounds__(128) ysolve_kernel(C* __restrict__ data, int nxh, int ny, int nz,
                                                     const double* __restrict__ Zr, const double* __restrict__ D,
                                                     const double* __restrict__ pa, int lt) {
  extern __shared__ __align__(16) double2 sT[];  // [ny][lt] right-hand sides / solution
  double2* sF = sT + (size_t)ny * lt;            // [ny][lt] (Zr, D) pairs
  const int tid = threadIdx.x;
  const int l = tid % lt;
  const int64_t nl = (int64_t)nxh * nz;
  const int64_t g = (int64_t)blockIdx.x * lt + l;
  const bool ok = g < nl;
  const int kz = ok ? (int)(g / nxh) : 0;
  const int kx = ok ? (int)(g - (int64_t)kz * nxh) : 0;
  const int64_t base = (int64_t)kz * ny * nxh + kx;
  C* col = data + base;
  const int jstep = blockDim.x / lt;
  if (ok) {
    for (int j0 = tid / lt; j0 < ny; j0 += 4 * jstep) {
      double2 v[4];
      double z[4], d[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int j = j0 + u * jstep;
        if (j < ny) {
          v[u] = to_d2(col[(int64_t)j * nxh]);
          z[u] = Zr[base + (int64_t)j * nxh];
          d[u] = D[base + (int64_t)j * nxh];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int j = j0 + u * jstep;
        if (j < ny) {
          sT[j * lt + l] = v[u];
          sF[j * lt + l] = make_double2(z[u], d[u]);
        }
      }
    }
  }
  __syncthreads();
  if (tid < lt && ok) {
    double2* T = sT + l;
    const double2* F = sF + l;
    double2 tp = T[0];
    const double Z0 = F[0].x;
    tp.x *= Z0; tp.y *= Z0;
    T[0] = tp;
    for (int j = 1; j < ny - 1; ++j) {
      const double z = F[j * lt].x, a = pa[j];
      double2 v = T[j * lt];
      v.x = (v.x - a * tp.x) * z;
      v.y = (v.y - a * tp.y) * z;
      T[j * lt] = v;
      tp = v;
    }
    const double zl = F[(ny - 1) * lt].x;
    double2 v = T[(ny - 1) * lt];
    // TRID0's singular-pivot pin: the last unknown is zero when the pivot vanishes
    if (zl != 0.0) {
      v.x = (v.x - pa[ny - 1] * tp.x) / zl;
      v.y = (v.y - pa[ny - 1] * tp.y) / zl;
    } else {
      v.x = 0.0;
      v.y = 0.0;
    }
    T[(ny - 1) * lt] = v;
    for (int j = ny - 2; j >= 0; --j) {
      const double d = F[j * lt].y;
      double2 u = T[j * lt];
      u.x = u.x - d * v.x;
      u.y = u.y - d * v.y;
      T[j * lt] = u;
      v = u;
    }
  }
  __syncthreads();
  if (ok)
    for (int j = tid / lt; j < ny; j += jstep) col[(int64_t)j * nxh] = from_d2<C>(sT[j * lt + l]);
}

// The same solve with one thread per (kx, kz) line working in place in global memory: at a fixed
// row j the threads of a warp (consecutive kx) read and write consecutive values, and each thread
// loads eight rows ahead of its sweep, so the sequential recurrences of many lines overlap.  The
// arithmetic and its order are those of ysolve_kernel.
constexpr int kYsBatch = 8;
template <typename C>
__global__ void __launch_bounds__(128) ysolve_lines_kernel(C* __restrict__ data, int nxh, int ny, int nz,
                                                           const double* __restrict__ Zr,
                                                           const double* __restrict__ D,
                                                           const double* __restrict__ pa) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (int64_t)nxh * nz) return;
  const int kz = (int)(g / nxh), kx = (int)(g - (int64_t)kz * nxh);
  const int64_t base = (int64_t)kz * ny * nxh + kx;
  C* col = data + base;
  const double* zr = Zr + base;
  const double* dd = D + base;
  const int64_t s = nxh;
  double2 tp = to_d2(col[0]);
  const double Z0 = zr[0];
  tp.x *= Z0;
  tp.y *= Z0;
  col[0] = from_d2<C>(tp);
  for (int j0 = 1; j0 < ny - 1; j0 += kYsBatch) {
    double2 v[kYsBatch];
    double z[kYsBatch];
#pragma unroll
    for (int u = 0; u < kYsBatch; ++u)
      if (j0 + u < ny - 1) {
        v[u] = to_d2(col[(j0 + u) * s]);
        z[u] = zr[(j0 + u) * s];
      }
#pragma unroll
    for (int u = 0; u < kYsBatch; ++u)
      if (j0 + u < ny - 1) {
        const double a = __ldg(pa + j0 + u);
        v[u].x = (v[u].x - a * tp.x) * z[u];
        v[u].y = (v[u].y - a * tp.y) * z[u];
        tp = v[u];
      }
#pragma unroll
    for (int u = 0; u < kYsBatch; ++u)
      if (j0 + u < ny - 1) col[(j0 + u) * s] = from_d2<C>(v[u]);
  }
  const double zl = zr[(ny - 1) * s];
  double2 v = to_d2(col[(ny - 1) * s]);
  // TRID0's singular-pivot pin: the last unknown is zero when the pivot vanishes
  if (zl != 0.0) {
    v.x = (v.x - __ldg(pa + ny - 1) * tp.x) / zl;
    v.y = (v.y - __ldg(pa + ny - 1) * tp.y) / zl;
  } else {
    v.x = 0.0;
    v.y = 0.0;
  }
  col[(ny - 1) * s] = from_d2<C>(v);
  for (int j0 = ny - 2; j0 >= 0; j0 -= kYsBatch) {
    double2 w[kYsBatch];
    double d[kYsBatch];
#pragma unroll
    for (int u = 0; u < kYsBatch; ++u)
      if (j0 - u >= 0) {
        w[u] = to_d2(col[(j0 - u) * s]);
        d[u] = dd[(j0 - u) * s];
      }
#pragma unroll
    for (int u = 0; u < kYsBatch; ++u)
      if (j0 - u >= 0) {
        w[u].x = w[u].x - d[u] * v.x;
        w[u].y = w[u].y - d[u] * v.y;
        v = w[u];
      }
#pragma unroll
    for (int u = 0; u < kYsBatch; ++u)
      if (j0 - u >= 0) col[(j0 - u) * s] = from_d2<C>(w[u]);
  }
}

template <typename C>
void launch_ysolve(C* data, int nxh, int ny, int nz, const double* Zr, const double* D, const double* pa,
                   cudaStream_t st) {
  if (ny < 2) throw std::runtime_error("ysolve: ny must be at least 2");
  if (ny > 160) {
    // tall columns: the shared-memory tile leaves too few solving threads per SM
    const int64_t n = (int64_t)nxh * nz;
    ysolve_lines_kernel<C><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(data, nxh, ny, nz, Zr, D, pa);
    return;
  }
  // 16 columns per CTA: a CTA's load, sweep and store phases run one after another, so several
  // CTAs per SM are needed to keep loads in flight while others sweep
  int lt = 16;
  while (lt > 4 && (size_t)ny * lt * 32 > 110 * 1024) lt /= 2;
  const size_t shm = (size_t)ny * lt * 32;
  if (shm > 200 * 1024) throw std::runtime_error("ysolve: ny too large for the shared-memory tile");
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(ysolve_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  const int64_t n = (int64_t)nxh * nz;
  ysolve_kernel<C><<<(unsigned)((n + lt - 1) / lt), 128, shm, st>>>(data, nxh, ny, nz, Zr, D, pa, lt);
}
template void launch_ysolve<double2>(double2*, int, int, int, const double*, const double*, const double*,
                                     cudaStream_t);
template void launch_ysolve<float2>(float2*, int, int, int, const double*, const double*, const double*,
                                    cudaStream_t);

__global__ void spectral_divide_kernel(double2* __restrict__ data, int nxh, int ny, int nz,
                                       const double* __restrict__ k2x, const double* __restrict__ k2y,
                                       const double* __restrict__ k2z, double norm) {
  const int64_t n = (int64_t)nxh * ny * nz;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
    const int kx = (int)(g % nxh);
    const int64_t r = g / nxh;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    double2 v = data[g];
    v.x *= norm;
    v.y *= norm;
    const double kk = k2x[kx] + k2y[j] + k2z[k];
    if (kk < 1.0e-16) { v.x = 0.0; v.y = 0.0; }
    else { v.x = v.x / (-kk); v.y = v.y / (-kk); }
    data[g] = v;
  }
}

void launch_spectral_divide(double2* data, int nxh, int ny, int nz, const double* k2x, const double* k2y,
                            const double* k2z, double norm, cudaStream_t st) {
  spectral_divide_kernel<<<148 * 8, 256, 0, st>>>(data, nxh, ny, nz, k2x, k2y, k2z, norm);
}

// ===========================================================================
// poisson_010 y stage (src/poisson_1stderivcomp.f90:1457-1816) per (kx, kz) column of the
// x/z spectrum (layout (kz, j, kx)): the even/odd reordering in y (:1491-1501), the y FFT, the
// cosine post-processing (:1557-1575), then either the wavenumber division (uniform grid,
// :1591-1613) or the pentadiagonal solves of the odd and even cosine modes (matrice_refinement
// :2718-3039 and inversion5_v1 :420-561), the backward post-processing (:1717-1735), the
// inverse y FFT and the inverse reordering (:1772-1782).  The column stays in shared memory
// from the first load to the last store.
//
// The x and z half-cell phase factors of the reference (:1527-1553, :1740-1767) multiply a
// column by e^{-i theta} before this stage and by e^{+i theta} after it; the stage applies one
// real operator to the real and the imaginary parts, so they cancel and are not applied.
// ===========================================================================
constexpr double kInv5Eps = 1.0e-16;  // epsilon of inversion5_v1 with DOUBLE_PREC

template <int MODE>  // 0: uniform grid (wavenumber division), 1: stretched grid (pentadiagonal)
__global__ void __launch_bounds__(256) dct_y_kernel(const __grid_constant__ FftPlan fp, double2* __restrict__ data,
                                                    int nxh, int nz, int lpc, const double* __restrict__ ayby,
                                                    const double* __restrict__ k2x, const double* __restrict__ k2z,
                                                    const double* __restrict__ k2y, const double* __restrict__ ptab,
                                                    const double* __restrict__ pfac, double scale) {
  extern __shared__ double2 sh[];
  __shared__ int64_t lbase[32];
  __shared__ double lkx[32], lkz[32];
  __shared__ int64_t lfoff[32];  // start of the column's elimination factors in pfac, -1 past the end
  const int ny = fp.n, h = ny / 2;
  const int ls = ny + 1;  // padded line stride: loads, stores and post-processing run across lines
  double2* b0 = sh;
  double2* b1 = sh + (size_t)lpc * ls;
  const int64_t g0 = (int64_t)blockIdx.x * lpc;
  const int64_t nlines = (int64_t)nxh * nz;
  if (threadIdx.x < lpc) {
    const int64_t g = g0 + threadIdx.x;
    if (g < nlines) {
      const int kz = (int)(g / nxh), kx = (int)(g - (int64_t)kz * nxh);
      lbase[threadIdx.x] = kx + (int64_t)kz * nxh * ny;
      lkx[threadIdx.x] = k2x[kx];
      lkz[threadIdx.x] = k2z[kz];
      const int kzf = kz <= nz - kz ? kz : nz - kz;
      lfoff[threadIdx.x] = (int64_t)kzf * h * 8 * nxh + kx;
    } else {
      lbase[threadIdx.x] = -1;
      lfoff[threadIdx.x] = -1;
      lkx[threadIdx.x] = 0.0;
      lkz[threadIdx.x] = 0.0;
    }
  }
  __syncthreads();
  const int ntot = lpc * ny;
  const float ilpc = 1.0f / (float)lpc;
  // load: row p of a column goes to position q of the reordered line (q < ny/2: row 2q;
  // q >= ny/2: row 2ny-1-2q)
  for (int t0 = threadIdx.x; t0 < ntot; t0 += 4 * blockDim.x) {
    double2 v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      v[u] = make_double2(0.0, 0.0);
      if (t < ntot) {
        const int p = fast_div(t, lpc, ilpc), l = t - p * lpc;
        const int64_t base = lbase[l];
        if (base >= 0) v[u] = data[base + (int64_t)p * nxh];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < ntot) {
        const int p = fast_div(t, lpc, ilpc), l = t - p * lpc;
        const int q = (p & 1) ? ny - 1 - (p >> 1) : (p >> 1);
        b0[l * ls + q] = v[u];
      }
    }
  }
  __syncthreads();
  double2* r = smem_fft(b0, b1, lpc, fp, -1, ls);
  double2* o = (r == b0) ? b1 : b0;
  const double* ay = ayby;
  const double* by = ayby + ny;
  // forward post-processing into o, layout [j][l]
  for (int t = threadIdx.x; t < ntot; t += blockDim.x) {
    const int j = fast_div(t, lpc, ilpc), l = t - j * lpc;
    const double2 c = r[l * ls + j];
    double2 v;
    if (j == 0) {
      v = make_double2(c.x * scale, c.y * scale);
    } else {
      const double2 d = r[l * ls + (ny - j)];
      const double t1 = c.x * scale, t2 = c.y * scale, t3 = d.x * scale, t4 = d.y * scale;
      const double yb = by[j], ya = ay[j];
      const double xx1 = t1 * yb, xx2 = t1 * ya, xx3 = t2 * yb, xx4 = t2 * ya;
      const double xx5 = t3 * yb, xx6 = t3 * ya, xx7 = t4 * yb, xx8 = t4 * ya;
      v = make_double2(0.5 * (xx1 + xx4 + xx5 - xx8), 0.5 * (-xx2 + xx3 + xx6 + xx7));
    }
    if (MODE == 0) {
      const double kk = lkx[l] + k2y[j] + lkz[l];
      if (fabs(kk) < 1.0e-16) v = make_double2(0.0, 0.0);
      else v = make_double2(v.x / (-kk), v.y / (-kk));
    }
    o[j * lpc + l] = v;
  }
  __syncthreads();
  if (MODE == 1) {
    // one thread per (column, parity): inversion5_v1 on rows r = 0..h-1 (mode j = 2r + s) with
    // the elimination factors of the column's matrix (dct_y_factor_kernel).  The factors are
    // staged in the free FFT buffer r by all threads (coalesced across kx): the forward
    // multipliers for the forward sweep, then the back-substitution factors, layout
    // [row][field][thread] with thread = 2 l + s.
    double* fs = reinterpret_cast<double*>(r);
    const int nt = 2 * lpc;
    const float intt = 1.0f / (float)nt;
    auto stage = [&](int f0) {
      // fields f0, f0+1 of every row for every (column, parity)
      const int tot = h * 2 * nt;
      constexpr int kB = 8;  // loads in flight per thread
      for (int t0 = threadIdx.x; t0 < tot; t0 += kB * blockDim.x) {
        double v[kB];
#pragma unroll
        for (int u = 0; u < kB; ++u) {
          const int t = t0 + u * blockDim.x;
          v[u] = 0.0;
          if (t < tot) {
            const int rf = fast_div(t, nt, intt), c = t - rf * nt;  // rf = row * 2 + field
            const int row = rf >> 1, fld = f0 + (rf & 1);
            const int64_t off = lfoff[c >> 1];
            if (off >= 0) v[u] = __ldg(pfac + off + ((size_t)(row * 4 + fld) * 2 + (c & 1)) * nxh);
          }
        }
#pragma unroll
        for (int u = 0; u < kB; ++u) {
          const int t = t0 + u * blockDim.x;
          if (t < tot) fs[t] = v[u];
        }
      }
    };
    stage(0);
    __syncthreads();
    const int tid = threadIdx.x;
    const int l = tid >> 1, s = tid & 1;
    const bool act = tid < nt && lbase[l] >= 0;  // l < lpc <= 32 whenever tid < nt
    auto E = [&](int row) -> double2& { return o[(2 * row + s) * lpc + l]; };
    auto FS = [&](int row, int fld) { return fs[(row * 2 + fld) * nt + tid]; };
    double2 e0 = make_double2(0.0, 0.0), e1 = e0;
    if (act) {
      e0 = E(0);
      e1 = E(1);
      double2 e2 = E(2);
      for (int m = 0; m <= h - 3; ++m) {
        const double L1 = FS(m, 0), L2 = FS(m, 1);
        const double2 e3 = m + 3 < h ? E(m + 3) : make_double2(0.0, 0.0);
        e1.x = e1.x - L1 * e0.x;
        e1.y = e1.y - L1 * e0.y;
        e2.x = e2.x - L2 * e0.x;
        e2.y = e2.y - L2 * e0.y;
        E(m) = e0;
        e0 = e1;
        e1 = e2;
        e2 = e3;
      }
    }
    __syncthreads();
    stage(2);
    __syncthreads();
    if (act) {
      // rows h-1 and h-2: (b1, tmp1/b1) and (1/a3, a4/a3) of the reference's last two steps
      const double bb = FS(h - 1, 0), t1 = FS(h - 1, 1);
      double2 eh = make_double2(0.0, 0.0);
      if (fabs(bb) > kInv5Eps) eh = make_double2(e1.x / bb - t1 * e0.x, e1.y / bb - t1 * e0.y);
      const double q2 = FS(h - 2, 0), a2 = FS(h - 2, 1);
      const double2 ehm = make_double2(e0.x * q2 - a2 * eh.x, e0.y * q2 - a2 * eh.y);
      E(h - 1) = eh;
      E(h - 2) = ehm;
      const double* A5 = ptab + (size_t)s * 6 * h + 5 * h;
      const bool pin = s == 0 && lkx[l] == 0.0 && lkz[l] == 0.0;
      double2 x1 = ehm, x2 = eh;
      for (int i = h - 3; i >= 0; --i) {
        const double q = FS(i, 0), a1 = FS(i, 1);
        const double b1 = ((pin && i == 0) ? 0.0 : __ldg(A5 + i)) * q;
        double2 ei = E(i);
        ei.x = ei.x * q - a1 * x1.x - b1 * x2.x;
        ei.y = ei.y * q - a1 * x1.y - b1 * x2.y;
        E(i) = ei;
        x2 = x1;
        x1 = ei;
      }
    }
  }
  __syncthreads();
  // backward post-processing from o ([j][l]) into r (line layout)
  for (int t = threadIdx.x; t < ntot; t += blockDim.x) {
    const int j = fast_div(t, lpc, ilpc), l = t - j * lpc;
    const double2 c = o[j * lpc + l];
    double2 v;
    if (j == 0) {
      v = c;
    } else {
      const double2 d = o[(ny - j) * lpc + l];
      const double t1 = c.x, t2 = c.y, t3 = d.x, t4 = d.y;
      const double yb = by[j], ya = ay[j];
      const double xx1 = t1 * yb, xx2 = t1 * ya, xx3 = t2 * yb, xx4 = t2 * ya;
      const double xx5 = t3 * yb, xx6 = t3 * ya, xx7 = t4 * yb, xx8 = t4 * ya;
      v = make_double2(xx1 - xx4 + xx6 + xx7, -(-xx2 - xx3 + xx5 - xx8));
    }
    r[l * ls + j] = v;
  }
  __syncthreads();
  double2* w = smem_fft(r, o, lpc, fp, +1, ls);
  // store: row p of the column takes position q of the line (the inverse reordering)
  for (int t = threadIdx.x; t < ntot; t += blockDim.x) {
    const int p = fast_div(t, lpc, ilpc), l = t - p * lpc;
    const int64_t base = lbase[l];
    const int q = (p & 1) ? ny - 1 - (p >> 1) : (p >> 1);
    if (base >= 0) data[base + (int64_t)p * nxh] = w[l * ls + q];
  }
}

// The elimination of inversion5_v1 depends on the column only through the main-diagonal shift
// kx2 + kz2 (and the zero-mode pin), not on the right-hand side, so it is done once per
// (kx, |kz|) and parity: per row r the forward multipliers of the step with pivot r (fields 0, 1;
// a zero pivot keeps the previous multiplier, as the reference does), and the back-substitution
// factors 1/a3 and a4/a3 (fields 2, 3; 0 for a pivot within eps), for the last row b1 and
// tmp1/b1 of the reference's closing 2x2 step.  The arithmetic is the reference's, in its order.
__global__ void dct_y_factor_kernel(double* __restrict__ pfac, int nxh, int nzh, int nz, int h,
                                    const double* __restrict__ k2x, const double* __restrict__ k2z,
                                    const double* __restrict__ ptab) {
  const int64_t n = (int64_t)nxh * nzh * 2;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const int kx = (int)(g % nxh);
  const int64_t rr = g / nxh;
  const int s = (int)(rr % 2);
  const int kzf = (int)(rr / 2);
  (void)nz;
  double* F = pfac + ((size_t)kzf * h * 8 + s) * nxh + kx;
  const size_t fst = (size_t)2 * nxh;
  const double* A1 = ptab + (size_t)s * 6 * h;
  const double* A2 = A1 + h;
  const double* T1 = A1 + 2 * h;
  const double* T2 = A1 + 3 * h;
  const double* A4 = A1 + 4 * h;
  const double* A5 = A1 + 5 * h;
  const double sxz = k2x[kx] + k2z[kzf];
  const bool pin = s == 0 && k2x[kx] == 0.0 && k2z[kzf] == 0.0;
  auto diag = [&](int row) { return -((sxz + T1[row]) + T2[row]); };
  auto sup2 = [&](int row) { return (pin && row == 0) ? 0.0 : A5[row]; };
  auto put = [&](int row, int field, double v) { F[(size_t)row * 4 * fst + field * fst] = v; };
  double P3 = pin ? 1.0 : diag(0), P4 = pin ? 0.0 : A4[0];
  double R12 = A2[1], R13 = diag(1), R14 = A4[1];
  double R21 = A1[2], R22 = A2[2], R23 = diag(2), R24 = A4[2];
  double tmp = 0.0;
  for (int m = 0; m <= h - 3; ++m) {
    const double P5 = sup2(m);
    if (P3 != 0.0) tmp = R12 / P3;
    put(m, 0, tmp);
    R13 = R13 - tmp * P4;
    R14 = R14 - tmp * P5;
    if (P3 != 0.0) tmp = R21 / P3;
    put(m, 1, tmp);
    R22 = R22 - tmp * P4;
    R23 = R23 - tmp * P5;
    const double q = fabs(P3) > kInv5Eps ? 1.0 / P3 : 0.0;
    put(m, 2, q);
    put(m, 3, P4 * q);
    P3 = R13; P4 = R14;
    R12 = R22; R13 = R23; R14 = R24;
    if (m + 3 < h) { R21 = A1[m + 3]; R22 = A2[m + 3]; R23 = diag(m + 3); R24 = A4[m + 3]; }
  }
  double t1 = fabs(P3) > kInv5Eps ? R12 / P3 : 0.0;
  const double sr = t1;
  const double bb = R13 - t1 * P4;
  t1 = fabs(bb) > kInv5Eps ? sr / bb : 0.0;
  put(h - 1, 2, bb);
  put(h - 1, 3, t1);
  const double q = fabs(P3) > kInv5Eps ? 1.0 / P3 : 0.0;
  put(h - 2, 2, q);
  put(h - 2, 3, P4 * q);
}

void launch_dct_y_factor(double* pfac, int nxh, int nz, int ny, const double* k2x, const double* k2z,
                         const double* ptab, cudaStream_t st) {
  const int nzh = nz / 2 + 1;
  const int64_t n = (int64_t)nxh * nzh * 2;
  dct_y_factor_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(pfac, nxh, nzh, nz, ny / 2, k2x, k2z, ptab);
}

void launch_dct_y(const FftPlan& fp, double2* data, int nxh, int nz, const double* ayby, const double* k2x,
                  const double* k2z, const double* k2y, const double* ptab, const double* pfac, double scale,
                  cudaStream_t st) {
  const int ny = fp.n;
  if (ny % 2 || ny < 8) throw std::runtime_error("dct_y: ny must be even and at least 8");
  // tall columns: half the FFT kernels' lines per CTA.  The serial sweeps of a CTA leave most
  // of its warps waiting, and smaller CTAs keep more sweeps in flight per SM (384x256x384:
  // 1.06 -> 0.99 ms; at 96 rows the halving is slower, 44 -> 53 us)
  int lpc = fft_lines_per_cta(ny);
  if (ny >= 192 && lpc > 1) lpc /= 2;
  const int64_t nlines = (int64_t)nxh * nz;
  const size_t shm = 2 * (size_t)lpc * (ny + 1) * sizeof(double2);
  const unsigned grid = (unsigned)((nlines + lpc - 1) / lpc);
  if (ptab) {
    if (!pfac) throw std::runtime_error("dct_y: the pentadiagonal factors are missing");
    cudaFuncSetAttribute(dct_y_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    dct_y_kernel<1><<<grid, 256, shm, st>>>(fp, data, nxh, nz, lpc, ayby, k2x, k2z, k2y, ptab, pfac, scale);
  } else {
    cudaFuncSetAttribute(dct_y_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    dct_y_kernel<0><<<grid, 256, shm, st>>>(fp, data, nxh, nz, lpc, ayby, k2x, k2z, k2y, ptab, pfac, scale);
  }
}

// ===========================================================================
// elementwise and reductions.  Field arrays are T (double, or float in the mixed-precision
// form); scalars, reduction accumulators and results stay double.
// ===========================================================================
// 16-byte vectors for the streaming kernels: the elements are processed V at a time where every
// array is 16-byte aligned (the same per-element arithmetic), the remainder one at a time
template <typename T>
struct EVec;
template <>
struct EVec<double> {
  using type = double2;
  static constexpr int n = 2;
};
template <>
struct EVec<float> {
  using type = float4;
  static constexpr int n = 4;
};
__device__ __forceinline__ bool aligned16(const void* a, const void* b = nullptr, const void* c = nullptr,
                                          const void* d = nullptr) {
  return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c) |
           reinterpret_cast<uintptr_t>(d)) & 15) == 0;
}
template <typename T>
__device__ __forceinline__ typename EVec<T>::type vld(const T* p, int64_t iv) {
  return reinterpret_cast<const typename EVec<T>::type*>(p)[iv];
}
template <typename T>
__device__ __forceinline__ void vst(T* p, int64_t iv, const typename EVec<T>::type& v) {
  reinterpret_cast<typename EVec<T>::type*>(p)[iv] = v;
}

template <typename T>
__global__ void fractional_step_kernel(T* __restrict__ rhs1, T* __restrict__ rhs0, const T* __restrict__ pfc,
                                       int64_t n, double dt, double gam, double zeta, double alpha) {
  const T tdt = T(dt), tg = T(gam), tz = T(zeta), ta = T(alpha);
  constexpr int V = EVec<T>::n;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nv = aligned16(rhs1, rhs0, pfc) ? n / V : 0;
  for (int64_t iv = t0; iv < nv; iv += stride) {
    typename EVec<T>::type c = vld(rhs1, iv), l = vld(rhs0, iv), f = vld(pfc, iv), o;
    const T* cp = reinterpret_cast<const T*>(&c);
    const T* lp = reinterpret_cast<const T*>(&l);
    const T* fp = reinterpret_cast<const T*>(&f);
    T* op = reinterpret_cast<T*>(&o);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      T tot = tg * cp[e] + tz * lp[e];
      tot = tot + ta * fp[e];
      op[e] = tdt * tot;
    }
    vst(rhs0, iv, c);
    vst(rhs1, iv, o);
  }
  for (int64_t i = nv * V + t0; i < n; i += stride) {
    const T cur = rhs1[i], last = rhs0[i];
    T tot = tg * cur + tz * last;
    rhs0[i] = cur;
    tot = tot + ta * pfc[i];
    rhs1[i] = tdt * tot;
  }
}
template <typename T>
void launch_fractional_step(T* rhs1, T* rhs0, const T* pfc, int64_t n, double dt, double gam, double zeta,
                            double alpha, cudaStream_t st) {
  fractional_step_kernel<T><<<148 * 8, 256, 0, st>>>(rhs1, rhs0, pfc, n, dt, gam, zeta, alpha);
}

template <typename T>
__global__ void weighted_partial_kernel(const T* __restrict__ a, const double* __restrict__ wy, int n1, int n2,
                                        int n3, double* __restrict__ partial) {
  __shared__ double red[256];
  // rows (j, k) in turn, two per CTA pass (threadIdx.x / 128), x strided by 128 within a row
  const int nrow = n2 * n3, half = threadIdx.x >> 7, tx = threadIdx.x & 127;
  double acc = 0.0;
  for (int r = blockIdx.x * 2 + half; r < nrow; r += gridDim.x * 2) {
    const double w = wy[r % n2];
    const T* row = a + (int64_t)r * n1;
    double s = 0.0;
    for (int i = tx; i < n1; i += 128) s += (double)row[i];
    acc += s * w;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}
__global__ void finalize_mean_kernel(const double* __restrict__ partial, int npart, double* __restrict__ out,
                                     double vol) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < npart; i += blockDim.x) acc += partial[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0] / vol;
}
template <typename T>
void launch_weighted_mean(const T* a, const double* wy, int n1, int n2, int n3, double* partial, int npart,
                          double* out, double vol, cudaStream_t st) {
  weighted_partial_kernel<T><<<npart, 256, 0, st>>>(a, wy, n1, n2, n3, partial);
  finalize_mean_kernel<<<1, 256, 0, st>>>(partial, npart, out, vol);
}

template <typename T>
__global__ void update_q_kernel(T* __restrict__ q, const T* __restrict__ rhs, const double* __restrict__ sub,
                                int64_t n) {
  const T s = sub ? T(sub[0]) : T(0);
  constexpr int V = EVec<T>::n;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nv = aligned16(q, rhs) ? n / V : 0;
  for (int64_t iv = t0; iv < nv; iv += stride) {
    typename EVec<T>::type qv = vld(q, iv), rv = vld(rhs, iv);
    T* qp = reinterpret_cast<T*>(&qv);
    const T* rp = reinterpret_cast<const T*>(&rv);
#pragma unroll
    for (int e = 0; e < V; ++e) qp[e] = qp[e] + (rp[e] - s);
    vst(q, iv, qv);
  }
  for (int64_t i = nv * V + t0; i < n; i += stride) q[i] = q[i] + (rhs[i] - s);
}
template <typename T>
void launch_update_q(T* q, const T* rhs, const double* sub, int64_t n, cudaStream_t st) {
  update_q_kernel<T><<<148 * 8, 256, 0, st>>>(q, rhs, sub, n);
}

template <typename T>
__global__ void set_yrows_kernel(T* __restrict__ a, int n1, int n2, int n3, int s0, double v0, int s1, double v1) {
  const int64_t n = (int64_t)n1 * n3;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = g / n1, i = g - k * n1;
    if (s0) a[(k * n2 + 0) * n1 + i] = T(v0);
    if (s1) a[(k * n2 + (n2 - 1)) * n1 + i] = T(v1);
  }
}
template <typename T>
void launch_set_yrows(T* a, int n1, int n2, int n3, int s0, double v0, int s1, double v1, cudaStream_t st) {
  set_yrows_kernel<T><<<148, 256, 0, st>>>(a, n1, n2, n3, s0, v0, s1, v1);
}

template <typename T>
__global__ void fbcy_const_kernel(T* __restrict__ fbc, int64_t nl, double v0, double v1) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < nl; g += (int64_t)gridDim.x * blockDim.x) {
    fbc[g] = T(v0);
    fbc[nl + g] = T(v1);
    fbc[2 * nl + g] = T(v0);
    fbc[3 * nl + g] = T(v1);
  }
}
template <typename T>
void launch_fbcy_const(T* fbc, int n1, int n3, double v0, double v1, cudaStream_t st) {
  fbcy_const_kernel<T><<<148, 256, 0, st>>>(fbc, (int64_t)n1 * n3, v0, v1);
}

// planes [4][n1*n3] from the wall rows of (n1, n2, n3) arrays: v = s*(A + c1*B)*C, C optional (else c2)
template <typename T>
__global__ void fbcy_extract_kernel(T* __restrict__ fbc, const T* __restrict__ A, const T* __restrict__ B,
                                    const T* __restrict__ C, double c1, double s, double c2, int n1, int n2, int n3) {
  const int64_t nl = (int64_t)n1 * n3;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < nl; g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = g / n1, i = g - k * n1;
    for (int side = 0; side < 2; ++side) {
      const int64_t a = (k * n2 + (side == 0 ? 0 : n2 - 1)) * n1 + i;
      T v = A[a];
      if (B) v = v + T(c1) * B[a];
      v = v * T(s);
      v = C ? v * C[a] : v * T(c2);
      fbc[side * nl + g] = v;
      fbc[(side + 2) * nl + g] = v;
    }
  }
}
template <typename T>
void launch_fbcy_extract(T* fbc, const T* A, const T* B, const T* C, double c1, double s, double c2, int n1, int n2,
                         int n3, cudaStream_t st) {
  fbcy_extract_kernel<T><<<148, 256, 0, st>>>(fbc, A, B, C, c1, s, c2, n1, n2, n3);
}

// out = sa*a + sb*b (+ sc*c), the terms added in that order
template <typename T>
__global__ void axpby_kernel(T* __restrict__ out, const T* __restrict__ a, double sa, const T* __restrict__ b,
                             double sb, const T* __restrict__ c, double sc, int64_t n) {
  const T ta = T(sa), tb = T(sb), tc = T(sc);
  constexpr int V = EVec<T>::n;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nv = aligned16(out, a, b, c) ? n / V : 0;
  for (int64_t iv = t0; iv < nv; iv += stride) {
    typename EVec<T>::type av = vld(a, iv), bv = b ? vld(b, iv) : av, cv = c ? vld(c, iv) : av, o;
    const T* ap = reinterpret_cast<const T*>(&av);
    const T* bp = reinterpret_cast<const T*>(&bv);
    const T* cp = reinterpret_cast<const T*>(&cv);
    T* op = reinterpret_cast<T*>(&o);
#pragma unroll
    for (int e = 0; e < V; ++e) {
      T v = ta * ap[e];
      if (b) v += tb * bp[e];
      if (c) v += tc * cp[e];
      op[e] = v;
    }
    vst(out, iv, o);
  }
  for (int64_t i = nv * V + t0; i < n; i += stride) {
    T v = ta * a[i];
    if (b) v += tb * b[i];
    if (c) v += tc * c[i];
    out[i] = v;
  }
}
template <typename T>
void launch_axpby(T* out, const T* a, double sa, const T* b, double sb, int64_t n, cudaStream_t st, const T* c,
                  double sc) {
  axpby_kernel<T><<<148 * 8, 256, 0, st>>>(out, a, sa, b, sb, c, sc, n);
}

// conversion between the double host layout and a float device field
__global__ void convert_kernel_d2f(float* __restrict__ out, const double* __restrict__ in, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
__global__ void convert_kernel_f2d(double* __restrict__ out, const float* __restrict__ in, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}
void launch_convert(float* out, const double* in, int64_t n, cudaStream_t st) {
  convert_kernel_d2f<<<148 * 8, 256, 0, st>>>(out, in, n);
}
void launch_convert(double* out, const float* in, int64_t n, cudaStream_t st) {
  convert_kernel_f2d<<<148 * 8, 256, 0, st>>>(out, in, n);
}

#define CHS_INST_ELEM(T)                                                                                      \
  template void launch_fractional_step<T>(T*, T*, const T*, int64_t, double, double, double, double,          \
                                          cudaStream_t);                                                      \
  template void launch_weighted_mean<T>(const T*, const double*, int, int, int, double*, int, double*, double, \
                                        cudaStream_t);                                                        \
  template void launch_update_q<T>(T*, const T*, const double*, int64_t, cudaStream_t);                       \
  template void launch_set_yrows<T>(T*, int, int, int, int, double, int, double, cudaStream_t);               \
  template void launch_fbcy_const<T>(T*, int, int, double, double, cudaStream_t);                             \
  template void launch_fbcy_extract<T>(T*, const T*, const T*, const T*, double, double, double, int, int, int, \
                                       cudaStream_t);                                                         \
  template void launch_axpby<T>(T*, const T*, double, const T*, double, int64_t, cudaStream_t, const T*, double);
CHS_INST_ELEM(double)
CHS_INST_ELEM(float)
#undef CHS_INST_ELEM

__global__ void absmax_partial_kernel(const double* __restrict__ a, int64_t n, double* __restrict__ partial) {
  __shared__ double red[256];
  __shared__ int bad[256];
  double m = 0.0;
  int nanf = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v = a[i];
    if (!isfinite(v)) nanf = 1;
    else m = fmax(m, fabs(v));
  }
  red[threadIdx.x] = m;
  bad[threadIdx.x] = nanf;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
      bad[threadIdx.x] |= bad[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { partial[2 * blockIdx.x] = red[0]; partial[2 * blockIdx.x + 1] = (double)bad[0]; }
}
__global__ void absmax_final_kernel(const double* __restrict__ partial, int npart, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double m = 0.0, b = 0.0;
    for (int i = 0; i < npart; ++i) { m = fmax(m, partial[2 * i]); b = fmax(b, partial[2 * i + 1]); }
    out[0] = m;
    out[1] = b;
  }
}
void launch_absmax(const double* a, int64_t n, double* partial, int npart, double* out, cudaStream_t st) {
  absmax_partial_kernel<<<npart, 256, 0, st>>>(a, n, partial);
  absmax_final_kernel<<<1, 32, 0, st>>>(partial, npart, out);
}

// the three x-slab maxima of |a| of Check_element_mass_conservation (src/eq_continuity.f90:379-389):
// slabs i in [0, 4), [4, n1 - 4), [n1 - 6, n1) of an (n1, n2, n3) array; out[0..2] hold the bit
// patterns of non-negative doubles (their order is the values' order) and start at zero
__global__ void absmax_slabs_kernel(const double* __restrict__ a, int n1, int64_t nrows,
                                    unsigned long long* __restrict__ out) {
  double m[3] = {0.0, 0.0, 0.0};
  const int64_t n = nrows * n1;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(g % n1);
    const double v = fabs(a[g]);
    if (i < 4) m[0] = fmax(m[0], v);
    if (i >= 4 && i < n1 - 4) m[1] = fmax(m[1], v);
    if (i >= n1 - 6) m[2] = fmax(m[2], v);
  }
  for (int s = 0; s < 3; ++s) {
    double v = m[s];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + s, (unsigned long long)__double_as_longlong(v));
  }
}
void launch_absmax_slabs(const double* a, int n1, int64_t nrows, unsigned long long* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), st);
  absmax_slabs_kernel<<<148 * 4, 256, 0, st>>>(a, n1, nrows, out);
}

__global__ void ke_density_kernel(double* __restrict__ out, const double* __restrict__ u, const double* __restrict__ v,
                                  const double* __restrict__ w, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = 0.5 * (u[i] * u[i] + v[i] * v[i] + w[i] * w[i]);
}
void launch_ke_density(double* out, const double* u, const double* v, const double* w, int64_t n, cudaStream_t st) {
  ke_density_kernel<<<148 * 8, 256, 0, st>>>(out, u, v, w, n);
}

}  // namespace chs

// ===========================================================================
// Variable-property kernels: table lookups of src/input_thermo.f90:345-446 and the energy
// update of src/eq_energy.f90:148-177, :430-440.  Lookups run in FP64 whatever T is.
// ===========================================================================
namespace chs {

template <typename T>
__global__ void property_update_kernel(const __grid_constant__ ThermoTab tb, const T* __restrict__ rhoh,
                                       T* __restrict__ h, T* __restrict__ t, T* __restrict__ k, T* __restrict__ d,
                                       T* __restrict__ m, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const CellProps p = props_from_dh(tb, (double)rhoh[i]);
    h[i] = T(p.h);
    t[i] = T(p.t);
    k[i] = T(p.k);
    d[i] = T(p.d);
    m[i] = T(p.m);
  }
}
template <typename T>
void launch_property_update(const ThermoTab& tb, const T* rhoh, T* h, T* t, T* k, T* d, T* m, int64_t n,
                            cudaStream_t st) {
  property_update_kernel<T><<<148 * 8, 256, 0, st>>>(tb, rhoh, h, t, k, d, m, n);
}

template <typename T>
__global__ void wall_props_kernel(const __grid_constant__ ThermoTab tb, const T* __restrict__ dh, int n1, int n2,
                                  int n3, int s0, int s1, T* __restrict__ fh, T* __restrict__ fk,
                                  T* __restrict__ fm, T* __restrict__ fd) {
  const int64_t nl = (int64_t)n1 * n3;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < 2 * nl; g += (int64_t)gridDim.x * blockDim.x) {
    const int side = g < nl ? 0 : 1;
    if ((side == 0 && !s0) || (side == 1 && !s1)) continue;
    const int64_t L = g - side * nl;
    const int64_t k = L / n1, i = L - k * n1;
    const int j = side == 0 ? 0 : n2 - 1;
    const CellProps p = props_from_dh(tb, (double)dh[(k * n2 + j) * n1 + i]);
    for (int u = side; u < 4; u += 2) {
      fh[u * nl + L] = T(p.h);
      fk[u * nl + L] = T(p.k);
      fm[u * nl + L] = T(p.m);
      fd[u * nl + L] = T(p.d);
    }
  }
}
template <typename T>
void launch_wall_props(const ThermoTab& tb, const T* dh_cpc, int n1, int n2, int n3, int s0, int s1, T* fh, T* fk,
                       T* fm, T* fd, cudaStream_t st) {
  wall_props_kernel<T><<<148, 256, 0, st>>>(tb, dh_cpc, n1, n2, n3, s0, s1, fh, fk, fm, fd);
}

template <typename T>
__global__ void energy_advance_kernel(T* __restrict__ rhs, T* __restrict__ rhs0, T* __restrict__ rhoh, int64_t n,
                                      double dt, double gam, double zeta) {
  const T tdt = T(dt), tg = T(gam), tz = T(zeta);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T cur = rhs[i], last = rhs0[i];
    const T tot = tg * cur + tz * last;
    rhs0[i] = cur;
    const T r1 = tdt * tot;
    rhs[i] = r1;
    rhoh[i] = rhoh[i] + r1;
  }
}
template <typename T>
void launch_energy_advance(T* rhs, T* rhs0, T* rhoh, int64_t n, double dt, double gam, double zeta,
                           cudaStream_t st) {
  energy_advance_kernel<T><<<148 * 8, 256, 0, st>>>(rhs, rhs0, rhoh, n, dt, gam, zeta);
}

// the energy fractional step and rho*h update followed by the property update of the new rho*h,
// one pass (the same arithmetic as energy_advance_kernel then property_update_kernel)
template <typename T>
__global__ void energy_advance_props_kernel(const __grid_constant__ ThermoTab tb, T* __restrict__ rhs,
                                            T* __restrict__ rhs0, T* __restrict__ rhoh, T* __restrict__ h,
                                            T* __restrict__ t, T* __restrict__ k, T* __restrict__ d,
                                            T* __restrict__ m, int64_t n, double dt, double gam, double zeta) {
  const T tdt = T(dt), tg = T(gam), tz = T(zeta);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T cur = rhs[i], last = rhs0[i];
    const T tot = tg * cur + tz * last;
    rhs0[i] = cur;
    const T r1 = tdt * tot;
    rhs[i] = r1;
    const T rn = rhoh[i] + r1;
    rhoh[i] = rn;
    const CellProps p = props_from_dh(tb, (double)rn);
    h[i] = T(p.h);
    t[i] = T(p.t);
    k[i] = T(p.k);
    d[i] = T(p.d);
    m[i] = T(p.m);
  }
}
template <typename T>
void launch_energy_advance_props(const ThermoTab& tb, T* rhs, T* rhs0, T* rhoh, T* h, T* t, T* k, T* d, T* m,
                                 int64_t n, double dt, double gam, double zeta, cudaStream_t st) {
  energy_advance_props_kernel<T><<<148 * 8, 256, 0, st>>>(tb, rhs, rhs0, rhoh, h, t, k, d, m, n, dt, gam, zeta);
}

template <typename T>
__global__ void fill_kernel(T* __restrict__ a, double v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    a[i] = T(v);
}
template <typename T>
void launch_fill(T* a, double v, int64_t n, cudaStream_t st) {
  fill_kernel<T><<<148 * 4, 256, 0, st>>>(a, v, n);
}

template <typename T>
__global__ void stats_update_kernel(const __grid_constant__ StatsIO<T> s) {
  const double ac = s.ac, am = s.am;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < s.n; i += (int64_t)gridDim.x * blockDim.x) {
    const double u0 = (double)s.u[0][i], u1 = (double)s.u[1][i], u2 = (double)s.u[2][i];
    s.pm[i] = am * s.pm[i] + ac * (double)s.p[i];
    s.um[0][i] = am * s.um[0][i] + ac * u0;
    s.um[1][i] = am * s.um[1][i] + ac * u1;
    s.um[2][i] = am * s.um[2][i] + ac * u2;
    s.uu[0][i] = am * s.uu[0][i] + ac * u0 * u0;
    s.uu[1][i] = am * s.uu[1][i] + ac * u1 * u1;
    s.uu[2][i] = am * s.uu[2][i] + ac * u2 * u2;
    s.uu[3][i] = am * s.uu[3][i] + ac * u0 * u1;
    s.uu[4][i] = am * s.uu[4][i] + ac * u0 * u2;
    s.uu[5][i] = am * s.uu[5][i] + ac * u1 * u2;
    if (s.t) {
      const double t = (double)s.t[i];
      s.tm[i] = am * s.tm[i] + ac * t;
      s.ttm[i] = am * s.ttm[i] + ac * t * t;
    }
  }
}
template <typename T>
void launch_stats_update(const StatsIO<T>& s, cudaStream_t st) {
  stats_update_kernel<T><<<148 * 8, 256, 0, st>>>(s);
}

#define CHS_INST_THERMO(T)                                                                                      \
  template void launch_property_update<T>(const ThermoTab&, const T*, T*, T*, T*, T*, T*, int64_t, cudaStream_t); \
  template void launch_wall_props<T>(const ThermoTab&, const T*, int, int, int, int, int, T*, T*, T*, T*,        \
                                     cudaStream_t);                                                             \
  template void launch_energy_advance<T>(T*, T*, T*, int64_t, double, double, double, cudaStream_t); \
  template void launch_energy_advance_props<T>(const ThermoTab&, T*, T*, T*, T*, T*, T*, T*, T*, int64_t, double,    \
                                               double, double, cudaStream_t);                                  \
  template void launch_fill<T>(T*, double, int64_t, cudaStream_t);                                           \
  template void launch_stats_update<T>(const StatsIO<T>&, cudaStream_t);
CHS_INST_THERMO(double)
CHS_INST_THERMO(float)
#undef CHS_INST_THERMO

}  // namespace chs
