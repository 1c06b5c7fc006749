// Fused CD2 substep kernels (see chs_fused.cuh).
//
// Momentum: Compute_momentum_rhs (src/eq_momentum2.f90:101-1571, Cartesian branches) with the
// fractional step Calculate_momentum_fractional_step (:35-71), per output value:
//   x: d/dx[-u u + 2 mu/Re (du/dx - div/3)] + d/dy[-v u + mu/Re (du/dy + dv/dx)]
//      + d/dz[-w u + mu/Re (du/dz + dw/dx)] - dp/dx            (:796-966)
//   y: d/dx[-u v + mu/Re (du/dy + dv/dx)] + d/dy[-v v + 2 mu/Re (dv/dy - div/3)]
//      + d/dz[-w v + mu/Re (dv/dz + dw/dy)] - dp/dy            (:978-1242)
//   z: d/dx[-u w + mu/Re (du/dz + dw/dx)] + d/dy[-v w + mu/Re (dv/dz + dw/dy)]
//      + d/dz[-w w + 2 mu/Re (dw/dz - div/3)] - dp/dz          (:1262-1457)
// with the first velocity factor of each convective product replaced by the interpolated momentum
// g and the viscosity interpolated to the stress points for variable properties (:576-703).
// Energy: Compute_energy_rhs and Calculate_energy_fractional_step (src/eq_energy.f90:148-401).
// Projection: Correct_massflux (src/eq_momentum2.f90:1577-1660) and convert_primary_conservative
// (src/para_conversion.f90:5-227).
#include <cuda_runtime.h>

#include <stdexcept>

#include "chs_fused.cuh"

namespace chs {

namespace {

// Every array of the fused kernels has x extent n0 and z extent n2 (periodic: points = cells) and y
// extent nc1 (cell rows) or np1 (point rows); index (k, j, i), x fastest, below 2^31 values.  The
// FP64 kernels form the index as k * (ny * n0) + (j * n0 + i), whose terms the many stencil loads
// of a thread share (measured 2 % faster per FP64 step; the FP32 kernels keep the nested form,
// which measured faster for them).
template <typename T>
__device__ __forceinline__ T ld(const T* __restrict__ a, int n0, int ny, int i, int j, int k) {
  if (sizeof(T) == 8) return __ldg(a + (k * (ny * n0) + (j * n0 + i)));
  return __ldg(a + (k * ny + j) * n0 + i);
}

// periodic CD2 operator of family FAM at row p: the bulk formula of stencil_op_kernel (bulk_fn with
// r2 = 0) on wrapped indices, times dd
// W false: the caller's rows p-1 .. p+1 lie inside 0 .. n-1 (a CTA away from the periodic seam), so
// the neighbours need no wrap
template <int FAM, typename T, bool W = true, typename F>
__device__ __forceinline__ T fz_per(const FzOp& o, int p, int n, const F& f) {
  const T r1 = T(o.r1);
  const int pp = W ? (p + 1 < n ? p + 1 : 0) : p + 1;
  const int pm = W ? (p > 0 ? p - 1 : n - 1) : p - 1;
  T v;
  if (FAM == M1P2C) v = r1 * (f(p) + f(pp));
  else if (FAM == M1C2P) v = r1 * (f(p) + f(pm));
  else if (FAM == D1C2P) v = r1 * (f(p) - f(pm));
  else v = r1 * (f(pp) - f(p));  // D1P2C
  return v * T(o.dd);
}

// y operator with walls at output row p from its row table
template <typename T, typename F>
__device__ __forceinline__ T fz_row(const FzRow* __restrict__ rows, const FzOp& o, int p, const T* __restrict__ fbc,
                                    int nl, int L, const F& f) {
  const FzRow& r = rows[o.row + p];
  const int fl = r.flags;
  T v = T(r.w[0]) * f(p + r.o[0]);
  v += T(r.w[1]) * f(p + r.o[1]);
  if (fl & 1) v += T(r.w[2]) * f(p + r.o[2]);
  if (fl & 2) v += T(r.wb[0]) * fbc[L];
  if (fl & 4) v += T(r.wb[1]) * fbc[nl + L];
  return v;
}

// input offsets of the two taps of a family's bulk formula (bulk_fn)
template <int FAM>
struct FzTap {
  static constexpr int o0 = FAM == D1P2C ? 1 : 0;
  static constexpr int o1 = (FAM == M1P2C) ? 1 : (FAM == D1P2C ? 0 : -1);
};

// y operator: periodic (PY); with walls in the interior rows (E false: the row's two bulk weights at
// the family's fixed offsets, so loads shared between taps are shared in the code); with walls near
// them (E: the row's own taps and wall planes)
template <int FAM, bool PY, bool E, typename T, typename F>
__device__ __forceinline__ T fz_y(const FzRow* __restrict__ rows, const FzOp& o, int p, int nin,
                                  const T* __restrict__ fbc, int nl, int L, const F& f) {
  if (PY) return fz_per<FAM, T>(o, p, nin, f);
  if (!E) {
    const FzRow& r = rows[o.row + p];
    T v = T(r.w[0]) * f(p + FzTap<FAM>::o0);
    v += T(r.w[1]) * f(p + FzTap<FAM>::o1);
    return v;
  }
  return fz_row<T>(rows, o, p, fbc, nl, L, f);
}

// op(conv) + w*op(visc) of one direction.  x and z are periodic with one bulk formula for both
// terms (checked by the host), so one operator runs on conv + (s*w)*visc; a y pair runs on the
// combined expression when it merges (as the operator path does) and term by term otherwise.
template <int FAM, int DIR, bool PY, bool E, typename T, bool WX = true, bool WZ = true, typename FC, typename FV>
__device__ __forceinline__ T fz_pair(const FzPair<T>& pr, const FzRow* __restrict__ rows, int nl, int n0, int i, int j,
                                     int k, int nin, double sv, double w, const FC& conv, const FV& visc) {
  const double sr = sv * w;
  auto comb = [&](int q) -> T {
    T e = conv(q);
    e += visc(sr, q);
    return e;
  };
  if (DIR == 0) return fz_per<FAM, T, WX>(pr.a, i, nin, comb);
  if (DIR == 2) return fz_per<FAM, T, WZ>(pr.a, k, nin, comb);
  if (PY) return fz_per<FAM, T>(pr.a, j, nin, comb);
  const int L = i + n0 * k;
  // interior rows: both terms' plans share the bulk weights (checked by the host)
  if (!E || pr.merged) return fz_y<FAM, false, E, T>(rows, pr.a, j, nin, pr.fa, nl, L, comb);
  const T va = fz_row<T>(rows, pr.a, j, pr.fa, nl, L, [&](int q) { return conv(q); });
  const T vb = fz_row<T>(rows, pr.b, j, pr.fb, nl, L, [&](int q) { return visc(sv, q); });
  return va + T(w) * vb;
}

// rows at each y wall whose outputs may reach a boundary row of some plan at some level: a block
// whose rows all lie in [kFzEdge, nc1 - kFzEdge) takes the bulk formulas only (the host checked
// that every y plan's bulk range covers rows 2 .. nout-3)
constexpr int kFzEdge = 4;
__device__ __forceinline__ bool fz_interior_block(int nc1) {
  const int j0 = blockIdx.y * blockDim.y;
  return j0 >= kFzEdge && j0 + (int)blockDim.y <= nc1 - kFzEdge;
}

// the inner operators of the momentum equation at one position (E: the row may be near a wall; WX,
// WZ: x / z neighbours may wrap around the periodic seam)
template <typename T, bool TH, bool PY, bool E, bool WX = true, bool WZ = true>
struct FzCtx {
  const FzMomentum<T>& f;
  int nl;  // lines of a y operator (n0 * n2)

  __device__ __forceinline__ T at(const T* a, int ny, int i, int j, int k) const { return ld(a, f.n0, ny, i, j, k); }
#define FZ_X(FAM, S, A, NY) fz_per<FAM, T, WX>(f.in[S], i, f.n0, [&](int q) { return at(A, NY, q, j, k); })
#define FZ_Z(FAM, S, A, NY) fz_per<FAM, T, WZ>(f.in[S], k, f.n2, [&](int q) { return at(A, NY, i, j, q); })
#define FZ_Y(FAM, S, A, NY, FB) \
  fz_y<FAM, PY, E, T>(f.rows, f.in[S], j, NY, FB, nl, i + f.n0 * k, [&](int q) { return at(A, NY, i, q, k); })
  // velocity interpolations and derivatives (src/eq_momentum2.f90:347-508)
  __device__ __forceinline__ T qxix(int i, int j, int k) const { return FZ_X(M1P2C, FI_QX_MX, f.qx, f.nc1); }
  __device__ __forceinline__ T qxdx(int i, int j, int k) const { return FZ_X(D1P2C, FI_QX_DX, f.qx, f.nc1); }
  __device__ __forceinline__ T qxdy(int i, int j, int k) const { return FZ_Y(D1C2P, FI_QX_DY, f.qx, f.nc1, f.fyqx); }
  __device__ __forceinline__ T qxiy(int i, int j, int k) const { return FZ_Y(M1C2P, FI_QX_MY, f.qx, f.nc1, f.fyqx); }
  __device__ __forceinline__ T qxiz(int i, int j, int k) const { return FZ_Z(M1C2P, FI_QX_MZ, f.qx, f.nc1); }
  __device__ __forceinline__ T qxdz(int i, int j, int k) const { return FZ_Z(D1C2P, FI_QX_DZ, f.qx, f.nc1); }
  __device__ __forceinline__ T qydx(int i, int j, int k) const { return FZ_X(D1C2P, FI_QY_DX, f.qy, f.np1); }
  __device__ __forceinline__ T qyix(int i, int j, int k) const { return FZ_X(M1C2P, FI_QY_MX, f.qy, f.np1); }
  __device__ __forceinline__ T qydy(int i, int j, int k) const {
    return FZ_Y(D1P2C, FI_QY_DY, f.qy, f.np1, (const T*)nullptr);
  }
  __device__ __forceinline__ T qyiy(int i, int j, int k) const { return FZ_Y(M1P2C, FI_QY_MY, f.qy, f.np1, f.fyqy); }
  __device__ __forceinline__ T qydz(int i, int j, int k) const { return FZ_Z(D1C2P, FI_QY_DZ, f.qy, f.np1); }
  __device__ __forceinline__ T qyiz(int i, int j, int k) const { return FZ_Z(M1C2P, FI_QY_MZ, f.qy, f.np1); }
  __device__ __forceinline__ T qzdx(int i, int j, int k) const { return FZ_X(D1C2P, FI_QZ_DX, f.qz, f.nc1); }
  __device__ __forceinline__ T qzix(int i, int j, int k) const { return FZ_X(M1C2P, FI_QZ_MX, f.qz, f.nc1); }
  __device__ __forceinline__ T qziy(int i, int j, int k) const { return FZ_Y(M1C2P, FI_QZ_MY, f.qz, f.nc1, f.fyqz); }
  __device__ __forceinline__ T qzdy(int i, int j, int k) const { return FZ_Y(D1C2P, FI_QZ_DY, f.qz, f.nc1, f.fyqz); }
  __device__ __forceinline__ T qziz(int i, int j, int k) const { return FZ_Z(M1P2C, FI_QZ_MZ, f.qz, f.nc1); }
  __device__ __forceinline__ T qzdz(int i, int j, int k) const { return FZ_Z(D1P2C, FI_QZ_DZ, f.qz, f.nc1); }
  // variable properties: interpolated momentum (:576-606) and viscosity (:691-703)
  __device__ __forceinline__ T gxix(int i, int j, int k) const { return FZ_X(M1P2C, FI_GX_MX, f.gx, f.nc1); }
  __device__ __forceinline__ T gxiy(int i, int j, int k) const { return FZ_Y(M1C2P, FI_GX_MY, f.gx, f.nc1, f.fz); }
  __device__ __forceinline__ T gxiz(int i, int j, int k) const { return FZ_Z(M1C2P, FI_GX_MZ, f.gx, f.nc1); }
  __device__ __forceinline__ T gyix(int i, int j, int k) const { return FZ_X(M1C2P, FI_GY_MX, f.gy, f.np1); }
  __device__ __forceinline__ T gyiy(int i, int j, int k) const { return FZ_Y(M1P2C, FI_GY_MY, f.gy, f.np1, f.fz); }
  __device__ __forceinline__ T gyiz(int i, int j, int k) const { return FZ_Z(M1C2P, FI_GY_MZ, f.gy, f.np1); }
  __device__ __forceinline__ T gzix(int i, int j, int k) const { return FZ_X(M1C2P, FI_GZ_MX, f.gz, f.nc1); }
  __device__ __forceinline__ T gziy(int i, int j, int k) const { return FZ_Y(M1C2P, FI_GZ_MY, f.gz, f.nc1, f.fz); }
  __device__ __forceinline__ T gziz(int i, int j, int k) const { return FZ_Z(M1P2C, FI_GZ_MZ, f.gz, f.nc1); }
  __device__ __forceinline__ T muy(int i, int j, int k) const { return FZ_Y(M1C2P, FI_MU_Y, f.mu, f.nc1, f.fm); }
  __device__ __forceinline__ T mux(int i, int j, int k) const { return FZ_X(M1C2P, FI_MU_X, f.mu, f.nc1); }
  __device__ __forceinline__ T muyx(int i, int j, int k) const {
    return fz_per<M1C2P, T, WX>(f.in[FI_MU_YX], i, f.n0, [&](int q) { return muy(q, j, k); });
  }
  __device__ __forceinline__ T muxz(int i, int j, int k) const {
    return fz_per<M1C2P, T, WZ>(f.in[FI_MU_XZ], k, f.n2, [&](int q) { return mux(i, j, q); });
  }
  __device__ __forceinline__ T muyz(int i, int j, int k) const {
    return fz_per<M1C2P, T, WZ>(f.in[FI_MU_YZ], k, f.n2, [&](int q) { return muy(i, j, q); });
  }
#undef FZ_X
#undef FZ_Z
#undef FZ_Y
  __device__ __forceinline__ T pr(int i, int j, int k) const { return at(f.p, f.nc1, i, j, k); }
  __device__ __forceinline__ T muc(int i, int j, int k) const { return at(f.mu, f.nc1, i, j, k); }
  // div = qxdx + qydy + qzdz at a cell centre (the axpby of the operator path)
  __device__ __forceinline__ T divc(T dx, int i, int j, int k) const {
    T v = dx;
    v += qydy(i, j, k);
    v += qzdz(i, j, k);
    return v;
  }
  // s*(a + c*b) (linm; times the viscosity with variable properties)
  __device__ __forceinline__ T lin(double s, T a, double c, T b) const { return T(s) * (a + T(c) * b); }

  // ---- the convective and viscous expressions at the stress points
  // cell centre, component C: conv -(c*qi) with c the interpolated momentum (or qi), visc
  // s*(qidi - div/3)[*mu]
  template <int C>
  __device__ __forceinline__ T conv_c(int i, int j, int k) const {
    if (C == 0) { const T a = qxix(i, j, k); const T b = TH ? gxix(i, j, k) : a; return T(-1.0) * (b * a); }
    if (C == 1) { const T a = qyiy(i, j, k); const T b = TH ? gyiy(i, j, k) : a; return T(-1.0) * (a * b); }
    const T a = qziz(i, j, k);
    const T b = TH ? gziz(i, j, k) : a;
    return T(-1.0) * (b * a);
  }
  template <int C>
  __device__ __forceinline__ T visc_c(double s, int i, int j, int k) const {
    const T dx = qxdx(i, j, k);
    const T d = C == 0 ? dx : (C == 1 ? qydy(i, j, k) : qzdz(i, j, k));
    const T v = lin(s, d, -1.0 / 3.0, divc(dx, i, j, k));
    return TH ? v * muc(i, j, k) : v;
  }
  // xy edge (ppc): x-momentum -(gyix*qxiy), y-momentum -(gxiy*qyix); the viscous part is shared
  template <int C>
  __device__ __forceinline__ T conv_xy(int i, int j, int k) const {
    if (C == 0) { const T a = qxiy(i, j, k); const T b = TH ? gyix(i, j, k) : qyix(i, j, k); return T(-1.0) * (b * a); }
    const T a = qyix(i, j, k);
    const T b = TH ? gxiy(i, j, k) : qxiy(i, j, k);
    return T(-1.0) * (b * a);
  }
  __device__ __forceinline__ T visc_xy(double s, int i, int j, int k) const {
    const T v = lin(s, qxdy(i, j, k), 1.0, qydx(i, j, k));
    return TH ? v * muyx(i, j, k) : v;
  }
  // xz edge (pcp): x-momentum -(gzix*qxiz), z-momentum -(gxiz*qzix)
  template <int C>
  __device__ __forceinline__ T conv_xz(int i, int j, int k) const {
    if (C == 0) { const T a = qxiz(i, j, k); const T b = TH ? gzix(i, j, k) : qzix(i, j, k); return T(-1.0) * (b * a); }
    const T a = qzix(i, j, k);
    const T b = TH ? gxiz(i, j, k) : qxiz(i, j, k);
    return T(-1.0) * (b * a);
  }
  __device__ __forceinline__ T visc_xz(double s, int i, int j, int k) const {
    const T v = lin(s, qxdz(i, j, k), 1.0, qzdx(i, j, k));
    return TH ? v * muxz(i, j, k) : v;
  }
  // yz edge (cpp): y-momentum -(qyiz*gziy), z-momentum -(gyiz*qziy)
  template <int C>
  __device__ __forceinline__ T conv_yz(int i, int j, int k) const {
    if (C == 1) { const T a = qyiz(i, j, k); const T b = TH ? gziy(i, j, k) : qziy(i, j, k); return T(-1.0) * (a * b); }
    const T a = qziy(i, j, k);
    const T b = TH ? gyiz(i, j, k) : qyiz(i, j, k);
    return T(-1.0) * (b * a);
  }
  __device__ __forceinline__ T visc_yz(double s, int i, int j, int k) const {
    const T v = lin(s, qzdy(i, j, k), 1.0, qydz(i, j, k));
    return TH ? v * muyz(i, j, k) : v;
  }

  // the fractional step of the operator path's O_FRAC store (pfc = 1 * v); last = m0[c][a], loaded
  // by the caller before the stencil loads so that no load waits behind the stores
  __device__ __forceinline__ T frac(int c, int a, T F, T v, T last) const {
    const T tdt = T(f.dt), tg = T(f.gam), tz = T(f.zeta), ta = T(f.alpha);
    const T pfc = T(1.0) * v;
    T tot = tg * F + tz * last;
    f.m0[c][a] = F;
    tot = tot + ta * pfc;
    const T r = tdt * tot;
    f.m[c][a] = r;
    return r;
  }
};

// one momentum component C (0 x, 1 y, 2 z) at (i, j, k)
template <typename T, bool TH, bool PY, int C, bool E, bool WX = true, bool WZ = true>
__device__ __forceinline__ T fz_momentum_body(const FzMomentum<T>& f, int i, int j, int k) {
  const int n0 = f.n0, nc1 = f.nc1, np1 = f.np1, n2 = f.n2;
  const FzCtx<T, TH, PY, E, WX, WZ> c{f, n0 * n2};
  const int nl = c.nl, L = i + n0 * k;
  const double r = f.rre;
  const int a = (k * (C == 1 ? np1 : nc1) + j) * n0 + i;
  const T last = f.m0[C][a];
  T F, v;
  if (C == 0) {
    // x-momentum at (i, j, k) of the qx grid
    F = fz_pair<D1C2P, 0, PY, E, T, WX, WZ>(
        f.term[0][0], f.rows, nl, n0, i, j, k, n0, 2.0, r, [&](int q) { return c.template conv_c<0>(q, j, k); },
        [&](double s, int q) { return c.template visc_c<0>(s, q, j, k); });
    F += fz_pair<D1P2C, 1, PY, E, T, WX, WZ>(
        f.term[0][1], f.rows, nl, n0, i, j, k, np1, 1.0, r, [&](int q) { return c.template conv_xy<0>(i, q, k); },
        [&](double s, int q) { return c.visc_xy(s, i, q, k); });
    F += fz_pair<D1P2C, 2, PY, E, T, WX, WZ>(
        f.term[0][2], f.rows, nl, n0, i, j, k, n2, 1.0, r, [&](int q) { return c.template conv_xz<0>(i, j, q); },
        [&](double s, int q) { return c.visc_xz(s, i, j, q); });
    v = fz_per<D1C2P, T, WX>(f.pres[0], i, n0, [&](int q) { return T(-1.0) * c.pr(q, j, k); });
    return c.frac(0, a, F, v, last);
  } else if (C == 1) {
    // y-momentum at (i, j, k) of the qy grid
    F = fz_pair<D1P2C, 0, PY, E, T, WX, WZ>(
        f.term[1][0], f.rows, nl, n0, i, j, k, n0, 1.0, r, [&](int q) { return c.template conv_xy<1>(q, j, k); },
        [&](double s, int q) { return c.visc_xy(s, q, j, k); });
    F += fz_pair<D1C2P, 1, PY, E, T, WX, WZ>(
        f.term[1][1], f.rows, nl, n0, i, j, k, nc1, 2.0, r, [&](int q) { return c.template conv_c<1>(i, q, k); },
        [&](double s, int q) { return c.template visc_c<1>(s, i, q, k); });
    F += fz_pair<D1P2C, 2, PY, E, T, WX, WZ>(
        f.term[1][2], f.rows, nl, n0, i, j, k, n2, 1.0, r, [&](int q) { return c.template conv_yz<1>(i, j, q); },
        [&](double s, int q) { return c.visc_yz(s, i, j, q); });
    v = fz_y<D1C2P, PY, E, T>(f.rows, f.pres[1], j, nc1, f.fpres[1], nl, L,
                           [&](int q) { return T(-1.0) * c.pr(i, q, k); });
    return c.frac(1, a, F, v, last);
  } else {
    // z-momentum at (i, j, k) of the qz grid
    F = fz_pair<D1P2C, 0, PY, E, T, WX, WZ>(
        f.term[2][0], f.rows, nl, n0, i, j, k, n0, 1.0, r, [&](int q) { return c.template conv_xz<2>(q, j, k); },
        [&](double s, int q) { return c.visc_xz(s, q, j, k); });
    F += fz_pair<D1P2C, 1, PY, E, T, WX, WZ>(
        f.term[2][1], f.rows, nl, n0, i, j, k, np1, 1.0, r, [&](int q) { return c.template conv_yz<2>(i, q, k); },
        [&](double s, int q) { return c.visc_yz(s, i, q, k); });
    F += fz_pair<D1C2P, 2, PY, E, T, WX, WZ>(
        f.term[2][2], f.rows, nl, n0, i, j, k, n2, 2.0, r, [&](int q) { return c.template conv_c<2>(i, j, q); },
        [&](double s, int q) { return c.template visc_c<2>(s, i, j, q); });
    v = fz_per<D1C2P, T, WZ>(f.pres[2], k, n2, [&](int q) { return T(-1.0) * c.pr(i, j, q); });
    return c.frac(2, a, F, v, last);
  }
}

// one momentum component C (0 x, 1 y, 2 z) per thread and output value; at most 64 registers, so that
// four CTAs fit an SM (the loads of more warps in flight)
template <typename T, bool TH, bool PY, int C>
__global__ void __launch_bounds__(256, 4) fz_momentum_kernel(const __grid_constant__ FzMomentum<T> f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const bool valid = i < f.n0 && j < (C == 1 ? f.np1 : f.nc1) && k < f.n2;
  T m = T(0);
  if (valid) {
    // CTAs whose x (z) neighbours within two of their rows stay inside the domain skip the wrap
    const int i0 = blockIdx.x * blockDim.x, k0 = blockIdx.z * blockDim.z;
    const bool wx = !(i0 >= 2 && i0 + (int)blockDim.x + 2 <= f.n0);
    const bool wz = !(k0 >= 2 && k0 + (int)blockDim.z + 2 <= f.n2);
    if (PY || fz_interior_block(f.nc1)) {
      if (!wx && !wz) m = fz_momentum_body<T, TH, PY, C, false, false, false>(f, i, j, k);
      else if (!wz) m = fz_momentum_body<T, TH, PY, C, false, true, false>(f, i, j, k);
      else m = fz_momentum_body<T, TH, PY, C, false, true, true>(f, i, j, k);
    } else {
      m = fz_momentum_body<T, TH, PY, C, true>(f, i, j, k);
    }
  }
  if (C == 0 && f.part) {
    // the CTA's share of the mass-flux mean: sum of wy[j] * m (fixed order, so the mean is
    // deterministic), reduced over the warp by shuffles and over the CTA's 8 warps in shared memory
    __shared__ double red[8];
    double s = valid ? f.wy[j] * (double)m : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if ((tid & 31) == 0) red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x * blockDim.y * blockDim.z) / 32; ++w) t += red[w];
      f.part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = t;
    }
  }
}

// the wall rows of the y-viscous boundary value (fbcy_velo: src/eq_momentum2.f90:374-442, :537-546,
// :1156-1171): qxdx_cpc = d/dx qxiy, qydy_cpc = d/dy qyiy, qzdz_cpc = d/dz qziy at the two walls
template <typename T, bool TH>
__global__ void fz_wall_visc_kernel(const __grid_constant__ FzMomentum<T> f, T* __restrict__ fvisc2,
                                    T* __restrict__ fcomb, const T* __restrict__ fconv2) {
  const int nl = f.n0 * f.n2;
  const FzCtx<T, TH, false, true> c{f, nl};
  for (int gs = blockIdx.x * blockDim.x + threadIdx.x; gs < 2 * nl; gs += gridDim.x * blockDim.x) {
    const int side = gs < nl ? 0 : 1, g = gs - side * nl;
    const int k = g / f.n0, i = g - k * f.n0;
    {
      const int j = side == 0 ? 0 : f.np1 - 1;
      const T ddx = fz_per<D1P2C, T>(f.in[FI_W_DX], i, f.n0, [&](int q) { return c.qxiy(q, j, k); });
      const T ddy = fz_row<T>(f.rows, f.in[FI_W_DY], j, f.fyqy, nl, g, [&](int q) { return c.qyiy(i, q, k); });
      const T ddz = fz_per<D1P2C, T>(f.in[FI_W_DZ], k, f.n2, [&](int q) { return c.qziy(i, j, q); });
      T sum = T(1.0) * ddx;
      sum += T(1.0) * ddy;
      sum += T(1.0) * ddz;
      // launch_fbcy_extract(A = qydy_cpc, B = the sum, C = mu_y or none, c1 = -1/3, s, c2 = 2)
      T v = ddy;
      v = v + T(-1.0 / 3.0) * sum;
      v = v * T(TH ? 2.0 : 1.0);
      v = TH ? v * c.muy(i, j, k) : v * T(2.0);
      for (int slot = side; slot < 4; slot += 2) {
        fvisc2[slot * nl + g] = v;
        T cb = T(1.0) * fconv2[slot * nl + g];
        cb += T(f.rre) * v;
        fcomb[slot * nl + g] = cb;
      }
    }
  }
}

template <typename T>
__global__ void fz_update_kernel(T* __restrict__ ux, T* __restrict__ uy, T* __restrict__ uz,
                                 const T* __restrict__ mx, const T* __restrict__ my, const T* __restrict__ mz,
                                 const double* __restrict__ bulk, int n0, int nc1, int np1, int n2, int s0, double v0,
                                 int s1, double v1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int k = blockIdx.z;
  if (i >= n0) return;
  if (j < nc1) {
    const int a = (k * nc1 + j) * n0 + i;
    const T s = bulk ? T(bulk[0]) : T(0);
    ux[a] = ux[a] + (mx[a] - s);
    uz[a] = uz[a] + (mz[a] - T(0));
  }
  const int b = (k * np1 + j) * n0 + i;
  T v = uy[b] + (my[b] - T(0));
  if (s0 && j == 0) v = T(v0);
  if (s1 && j == np1 - 1) v = T(v1);
  uy[b] = v;
}

// ---- energy equation: thread per cell (i, j, k)
template <typename T, bool E>
struct FzECtx {
  const FzEnergy<T>& f;
  int nl;
  __device__ __forceinline__ T at(const T* a, int ny, int i, int j, int k) const { return ld(a, f.n0, ny, i, j, k); }
  template <int FAM>
  __device__ __forceinline__ T xop(int s, const T* a, int i, int j, int k) const {
    return fz_per<FAM, T>(f.in[s], i, f.n0, [&](int q) { return at(a, f.nc1, q, j, k); });
  }
  template <int FAM>
  __device__ __forceinline__ T zop(int s, const T* a, int i, int j, int k) const {
    return fz_per<FAM, T>(f.in[s], k, f.n2, [&](int q) { return at(a, f.nc1, i, j, q); });
  }
  template <int FAM>
  __device__ __forceinline__ T yop(int s, const T* a, const T* fbc, int i, int j, int k) const {
    return fz_y<FAM, false, E, T>(f.rows, f.in[s], j, f.nc1, fbc, nl, i + f.n0 * k,
                                  [&](int q) { return at(a, f.nc1, i, q, k); });
  }
};

template <typename T, bool E>
__device__ __forceinline__ void fz_energy_body(const FzEnergy<T>& f, int i, int j, int k) {
  const int n0 = f.n0, nc1 = f.nc1, np1 = f.np1, n2 = f.n2;
  const FzECtx<T, E> c{f, n0 * n2};
  const int nl = c.nl;
  const int a = (k * nc1 + j) * n0 + i;
  const T last = f.rhs0[a], rh = f.rhoh[a];
  // x: faces (q, j, k) of the qx grid
  T F = fz_pair<D1P2C, 0, false, E, T>(
      f.term[0], f.rows, nl, n0, i, j, k, n0, 1.0, f.rpr,
      [&](int q) { return T(-1.0) * (c.at(f.gx, nc1, q, j, k) * c.template xop<M1C2P>(FE_H_X, f.h, q, j, k)); },
      [&](double s, int q) {
        return T(s) * (c.template xop<D1C2P>(FE_T_X, f.t, q, j, k) * c.template xop<M1C2P>(FE_K_X, f.k, q, j, k));
      });
  // y: faces (i, q, k) of the qy grid
  F += fz_pair<D1P2C, 1, false, E, T>(
      f.term[1], f.rows, nl, n0, i, j, k, np1, 1.0, f.rpr,
      [&](int q) { return T(-1.0) * (c.at(f.gy, np1, i, q, k) * c.template yop<M1C2P>(FE_H_Y, f.h, f.fh, i, q, k)); },
      [&](double s, int q) {
        return T(s) * (c.template yop<D1C2P>(FE_T_Y, f.t, f.fqw, i, q, k) *
                       c.template yop<M1C2P>(FE_K_Y, f.k, f.fk, i, q, k));
      });
  // z: faces (i, j, q) of the qz grid
  F += fz_pair<D1P2C, 2, false, E, T>(
      f.term[2], f.rows, nl, n0, i, j, k, n2, 1.0, f.rpr,
      [&](int q) { return T(-1.0) * (c.at(f.gz, nc1, i, j, q) * c.template zop<M1C2P>(FE_H_Z, f.h, i, j, q)); },
      [&](double s, int q) {
        return T(s) * (c.template zop<D1C2P>(FE_T_Z, f.t, i, j, q) * c.template zop<M1C2P>(FE_K_Z, f.k, i, j, q));
      });
  // energy_advance_kernel: rhs0 = F, rho*h += dt*(gam*F + zeta*rhs0)
  const T tdt = T(f.dt), tg = T(f.gam), tz = T(f.zeta);
  const T tot = tg * F + tz * last;
  f.rhs0[a] = F;
  const T r1 = tdt * tot;
  f.rhoh[a] = rh + r1;
}

// The interior rows of the energy pass with every input loaded up front (27 values of the 3D
// cross around the cell, independent loads in flight together), then the arithmetic of
// fz_energy_body<T, false> in the same order.
template <typename T>
__device__ __forceinline__ void fz_energy_interior(const FzEnergy<T>& f, int i, int j, int k) {
  const int n0 = f.n0, nc1 = f.nc1, np1 = f.np1, n2 = f.n2;
  const int im = i > 0 ? i - 1 : n0 - 1, ip = i + 1 < n0 ? i + 1 : 0;
  const int km = k > 0 ? k - 1 : n2 - 1, kp = k + 1 < n2 ? k + 1 : 0;
  const int c = (k * nc1 + j) * n0 + i;
  const int xm = c - i + im, xp = c - i + ip;
  const int ym = c - n0, yp = c + n0;
  const int zm = c + (km - k) * nc1 * n0, zp = c + (kp - k) * nc1 * n0;
  const int pc = (k * np1 + j) * n0 + i;
  const T last = f.rhs0[c], rh = f.rhoh[c];
  const T h0 = __ldg(f.h + c), hxm = __ldg(f.h + xm), hxp = __ldg(f.h + xp), hym = __ldg(f.h + ym),
          hyp = __ldg(f.h + yp), hzm = __ldg(f.h + zm), hzp = __ldg(f.h + zp);
  const T t0 = __ldg(f.t + c), txm = __ldg(f.t + xm), txp = __ldg(f.t + xp), tym = __ldg(f.t + ym),
          typ = __ldg(f.t + yp), tzm = __ldg(f.t + zm), tzp = __ldg(f.t + zp);
  const T k0 = __ldg(f.k + c), kxm = __ldg(f.k + xm), kxp = __ldg(f.k + xp), kym = __ldg(f.k + ym),
          kyp = __ldg(f.k + yp), kzm = __ldg(f.k + zm), kzp = __ldg(f.k + zp);
  const T gx0 = __ldg(f.gx + c), gx1 = __ldg(f.gx + xp);
  const T gy0 = __ldg(f.gy + pc), gy1 = __ldg(f.gy + pc + n0);
  const T gz0 = __ldg(f.gz + c), gz1 = __ldg(f.gz + zp);
  const FzRow& rh0 = f.rows[f.in[FE_H_Y].row + j];
  const FzRow& rh1 = f.rows[f.in[FE_H_Y].row + j + 1];
  const FzRow& rt0 = f.rows[f.in[FE_T_Y].row + j];
  const FzRow& rt1 = f.rows[f.in[FE_T_Y].row + j + 1];
  const FzRow& rk0 = f.rows[f.in[FE_K_Y].row + j];
  const FzRow& rk1 = f.rows[f.in[FE_K_Y].row + j + 1];
  const FzRow& ro = f.rows[f.term[1].a.row + j];
  const double sr = 1.0 * f.rpr;
  // periodic M1C2P / D1C2P (fz_per): r1*(f(p) + f(p-1))*dd, r1*(f(p) - f(p-1))*dd
  auto m12 = [](const FzOp& o, T a, T b) { return T(o.r1) * (a + b) * T(o.dd); };
  auto d12 = [](const FzOp& o, T a, T b) { return T(o.r1) * (a - b) * T(o.dd); };
  // y with walls, interior (fz_y): w0*f(p) + w1*f(p-1)
  auto y12 = [](const FzRow& r, T a, T b) {
    T v = T(r.w[0]) * a;
    v += T(r.w[1]) * b;
    return v;
  };
  auto face = [&](T g, T hf, T dt, T kf) {
    T e = T(-1.0) * (g * hf);
    e += T(sr) * (dt * kf);
    return e;
  };
  // x: faces i and i+1 (D1P2C: r1*(f(p+1) - f(p))*dd)
  const T ex0 = face(gx0, m12(f.in[FE_H_X], h0, hxm), d12(f.in[FE_T_X], t0, txm), m12(f.in[FE_K_X], k0, kxm));
  const T ex1 = face(gx1, m12(f.in[FE_H_X], hxp, h0), d12(f.in[FE_T_X], txp, t0), m12(f.in[FE_K_X], kxp, k0));
  T F = T(f.term[0].a.r1) * (ex1 - ex0) * T(f.term[0].a.dd);
  // y: faces j and j+1 (D1P2C interior: w0*f(j+1) + w1*f(j))
  const T ey0 = face(gy0, y12(rh0, h0, hym), y12(rt0, t0, tym), y12(rk0, k0, kym));
  const T ey1 = face(gy1, y12(rh1, hyp, h0), y12(rt1, typ, t0), y12(rk1, kyp, k0));
  T vy = T(ro.w[0]) * ey1;
  vy += T(ro.w[1]) * ey0;
  F += vy;
  // z: faces k and k+1
  const T ez0 = face(gz0, m12(f.in[FE_H_Z], h0, hzm), d12(f.in[FE_T_Z], t0, tzm), m12(f.in[FE_K_Z], k0, kzm));
  const T ez1 = face(gz1, m12(f.in[FE_H_Z], hzp, h0), d12(f.in[FE_T_Z], tzp, t0), m12(f.in[FE_K_Z], kzp, k0));
  F += T(f.term[2].a.r1) * (ez1 - ez0) * T(f.term[2].a.dd);
  // energy_advance_kernel: rhs0 = F, rho*h += dt*(gam*F + zeta*rhs0)
  const T tdt = T(f.dt), tg = T(f.gam), tz = T(f.zeta);
  const T tot = tg * F + tz * last;
  f.rhs0[c] = F;
  const T r1 = tdt * tot;
  f.rhoh[c] = rh + r1;
}

template <typename T>
__global__ void __launch_bounds__(256) fz_energy_kernel(const __grid_constant__ FzEnergy<T> f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= f.n0 || j >= f.nc1 || k >= f.n2) return;
  if (fz_interior_block(f.nc1)) fz_energy_interior<T>(f, i, j, k);
  else fz_energy_body<T, true>(f, i, j, k);
}

template <typename T>
__global__ void fz_energy_walls_kernel(const __grid_constant__ FzEnergy<T> f, int mode, T* __restrict__ out) {
  const int nl = f.n0 * f.n2;
  const FzECtx<T, true> c{f, nl};
  for (int gs = blockIdx.x * blockDim.x + threadIdx.x; gs < 2 * nl; gs += gridDim.x * blockDim.x) {
    const int side = gs < nl ? 0 : 1, g = gs - side * nl;
    const int k = g / f.n0, i = g - k * f.n0;
    {
      const int j = side == 0 ? 0 : f.np1 - 1;
      if (mode == 0) {
        // launch_fbcy_extract(A = dT/dy, B none, C = kappa_y, s = 1): (A*1)*C
        T v = c.template yop<D1C2P>(FE_T_Y, f.t, f.fqw, i, j, k);
        v = v * T(1.0);
        v = v * c.template yop<M1C2P>(FE_K_Y, f.k, f.fk, i, j, k);
        out[side * nl + g] = v;
        out[(side + 2) * nl + g] = v;
      } else if (side == 0 ? f.ws0 : f.ws1) {
        // wall_props_kernel on the wall row of rho*h interpolated to the y faces
        const T dh = c.template yop<M1C2P>(FE_RH_Y, f.rhoh, (const T*)nullptr, i, j, k);
        const CellProps p = props_from_dh(f.tab, (double)dh);
        for (int u = side; u < 4; u += 2) {
          f.wh[u * nl + g] = T(p.h);
          f.wk[u * nl + g] = T(p.k);
          f.wm[u * nl + g] = T(p.m);
          f.wd[u * nl + g] = T(p.d);
        }
      }
    }
  }
}

// ---- pressure update, projection and q = g / rho_face: thread per (i, j, k), j over the y points
template <typename T, bool TH>
__global__ void __launch_bounds__(256) fz_project_kernel(const __grid_constant__ FzProject<T> f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int n0 = f.n0, nc1 = f.nc1, np1 = f.np1, n2 = f.n2;
  if (i >= n0 || j >= np1 || k >= n2) return;
  const int nl = n0 * n2, L = i + n0 * k;
  auto phi = [&](int ii, int jj, int kk) { return ld(f.phi, n0, nc1, ii, jj, kk); };
  auto rho = [&](int ii, int jj, int kk) { return ld(f.rho, n0, nc1, ii, jj, kk); };
  const T cf = T(f.coef);
  // every read-modify-write value is loaded before the first store, so that no load waits behind one
  const int b = (k * np1 + j) * n0 + i;
  T uy0 = f.uy[b];
  if (f.upd) uy0 = uy0 + (f.my[b] - T(0));
  if (j < nc1) {
    const int a = (k * nc1 + j) * n0 + i;
    const T p0 = f.p[a];
    T ux0 = f.ux[a], uz0 = f.uz[a];
    if (f.upd) {
      const T s = f.bulk ? T(f.bulk[0]) : T(0);
      ux0 = ux0 + (f.mx[a] - s);
      uz0 = uz0 + (f.mz[a] - T(0));
    }
    // p += phi (axpby with unit weights)
    T pv = T(1.0) * p0;
    pv += T(1.0) * phi(i, j, k);
    f.p[a] = pv;
    const T vx = fz_per<D1C2P, T>(f.in[FP_DX], i, n0, [&](int q) { return phi(q, j, k); });
    const T gxn = ux0 + cf * vx;
    f.ux[a] = gxn;
    const T vz = fz_per<D1C2P, T>(f.in[FP_DZ], k, n2, [&](int q) { return phi(i, j, q); });
    const T gzn = uz0 + cf * vz;
    f.uz[a] = gzn;
    if (TH) {
      f.qx[a] = gxn / (T(1.0) * fz_per<M1C2P, T>(f.in[FP_PX], i, n0, [&](int q) { return rho(q, j, k); }));
      f.qz[a] = gzn / (T(1.0) * fz_per<M1C2P, T>(f.in[FP_PZ], k, n2, [&](int q) { return rho(i, j, q); }));
    }
  }
  T vy;
  if (f.periodic_y) vy = fz_per<D1C2P, T>(f.in[FP_DY], j, nc1, [&](int q) { return phi(i, q, k); });
  else vy = fz_row<T>(f.rows, f.in[FP_DY], j, f.fphi, nl, L, [&](int q) { return phi(i, q, k); });
  T gyn = uy0 + cf * vy;
  if (f.s0 && j == 0) gyn = T(f.v0);
  if (f.s1 && j == np1 - 1) gyn = T(f.v1);
  f.uy[b] = gyn;
  if (TH) {
    const T ry = fz_row<T>(f.rows, f.in[FP_PY], j, f.fd, nl, L, [&](int q) { return rho(i, q, k); });
    f.qy[b] = gyn / (T(1.0) * ry);
  }
}

// ---- momentum advance folded into the Poisson right-hand side: thread per cell (i, j, k)
template <typename T>
__global__ void __launch_bounds__(256) fz_update_div_kernel(const __grid_constant__ FzUpdateDiv<T> f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int n0 = f.n0, nc1 = f.nc1, np1 = f.np1, n2 = f.n2;
  if (i >= n0 || j >= nc1 || k >= n2) return;
  const T s = f.bulk ? T(f.bulk[0]) : T(0);
  // u' at a face (fz_update_kernel's arithmetic)
  auto gx = [&](int q) {
    const int a = (k * nc1 + j) * n0 + q;
    return __ldg(f.ux + a) + (__ldg(f.mx + a) - s);
  };
  auto gy = [&](int q) {
    const int b = (k * np1 + q) * n0 + i;
    T v = __ldg(f.uy + b) + (__ldg(f.my + b) - T(0));
    if (f.s0 && q == 0) v = T(f.v0);
    if (f.s1 && q == np1 - 1) v = T(f.v1);
    return v;
  };
  auto gz = [&](int q) {
    const int a = (q * nc1 + j) * n0 + i;
    return __ldg(f.uz + a) + (__ldg(f.mz + a) - T(0));
  };
  const T vx = fz_per<D1P2C, T>(f.dx, i, n0, gx);
  const T vy = fz_row<T>(f.rows, f.dy, j, f.fdy, n0 * n2, i + n0 * k, gy);
  const T vz = fz_per<D1P2C, T>(f.dz, k, n2, gz);
  // run_fused's sum of the three terms with their coefficient
  const T g = T(f.coeff);
  T sum = T(0);
  sum = sum + g * vx;
  sum = sum + g * vy;
  sum = sum + g * vz;
  f.out[(k * nc1 + j) * n0 + i] = sum;
}

// the mass-flux mean from the x pass's per-CTA sums: one CTA, thread t summing parts t, t + 256, ...
// (eight loads in flight), then a tree over the threads; a fixed order, so the mean is deterministic
__global__ void __launch_bounds__(256) fz_finalize_mean_kernel(const double* __restrict__ part, int nblk,
                                                                double* __restrict__ bulk, double vol) {
  __shared__ double acc[256];
  const int tid = threadIdx.x, nthr = blockDim.x;
  double a = 0.0;
  for (int q0 = tid; q0 < nblk; q0 += 8 * nthr) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = q0 + u * nthr < nblk ? part[q0 + u * nthr] : 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (q0 + u * nthr < nblk) a += v[u];
  }
  acc[tid] = a;
  __syncthreads();
  for (int h = nthr / 2; h > 0; h >>= 1) {
    if (tid < h) acc[tid] += acc[tid + h];
    __syncthreads();
  }
  if (tid == 0) bulk[0] = acc[0] / vol;
}

}  // namespace

void launch_fz_finalize_mean(const double* part, int nblk, double* bulk, double vol, cudaStream_t st) {
  fz_finalize_mean_kernel<<<1, 256, 0, st>>>(part, nblk, bulk, vol);
}

int fz_momentum_x_blocks(int n0, int nc1, int n2) { return ((n0 + 31) / 32) * ((nc1 + 3) / 4) * ((n2 + 1) / 2); }

template <typename T, bool TH, bool PY>
void launch_fz_c(const FzMomentum<T>& f, int c, cudaStream_t st) {
  const dim3 bs(32, 4, 2);
  const int ny = c == 1 ? f.np1 : f.nc1;
  const dim3 grid((f.n0 + bs.x - 1) / bs.x, (ny + bs.y - 1) / bs.y, (f.n2 + bs.z - 1) / bs.z);
  if (c == 0) fz_momentum_kernel<T, TH, PY, 0><<<grid, bs, 0, st>>>(f);
  else if (c == 1) fz_momentum_kernel<T, TH, PY, 1><<<grid, bs, 0, st>>>(f);
  else fz_momentum_kernel<T, TH, PY, 2><<<grid, bs, 0, st>>>(f);
}

template <typename T>
void launch_fz_momentum(const FzMomentum<T>& f, int c, cudaStream_t st) {
  if (f.thermo && f.periodic_y) throw std::invalid_argument("fused momentum: variable properties need y walls");
  if (f.thermo) launch_fz_c<T, true, false>(f, c, st);
  else if (f.periodic_y) launch_fz_c<T, false, true>(f, c, st);
  else launch_fz_c<T, false, false>(f, c, st);
}

template <typename T>
void launch_fz_wall_visc(const FzMomentum<T>& f, T* fvisc2, T* fcomb, const T* fconv2, cudaStream_t st) {
  const int nl = f.n0 * f.n2;
  const int blocks = (2 * nl + 127) / 128;
  if (f.thermo) fz_wall_visc_kernel<T, true><<<blocks, 128, 0, st>>>(f, fvisc2, fcomb, fconv2);
  else fz_wall_visc_kernel<T, false><<<blocks, 128, 0, st>>>(f, fvisc2, fcomb, fconv2);
}

template <typename T>
void launch_fz_update(T* ux, T* uy, T* uz, const T* mx, const T* my, const T* mz, const double* bulk, int n0,
                      int nc1, int np1, int n2, int s0, double v0, int s1, double v1, cudaStream_t st) {
  const dim3 grid((n0 + 127) / 128, np1, n2);
  fz_update_kernel<T><<<grid, 128, 0, st>>>(ux, uy, uz, mx, my, mz, bulk, n0, nc1, np1, n2, s0, v0, s1, v1);
}

template <typename T>
void launch_fz_energy(const FzEnergy<T>& f, cudaStream_t st) {
  const dim3 bs(32, 4, 2);
  const dim3 grid((f.n0 + bs.x - 1) / bs.x, (f.nc1 + bs.y - 1) / bs.y, (f.n2 + bs.z - 1) / bs.z);
  fz_energy_kernel<T><<<grid, bs, 0, st>>>(f);
}

template <typename T>
void launch_fz_energy_walls(const FzEnergy<T>& f, int mode, T* out, cudaStream_t st) {
  const int nl = f.n0 * f.n2;
  fz_energy_walls_kernel<T><<<(2 * nl + 127) / 128, 128, 0, st>>>(f, mode, out);
}

template <typename T>
void launch_fz_update_div(const FzUpdateDiv<T>& f, cudaStream_t st) {
  const dim3 bs(32, 4, 2);
  const dim3 grid((f.n0 + bs.x - 1) / bs.x, (f.nc1 + bs.y - 1) / bs.y, (f.n2 + bs.z - 1) / bs.z);
  fz_update_div_kernel<T><<<grid, bs, 0, st>>>(f);
}

template <typename T>
void launch_fz_project(const FzProject<T>& f, cudaStream_t st) {
  const dim3 bs(32, 4, 2);
  const dim3 grid((f.n0 + bs.x - 1) / bs.x, (f.np1 + bs.y - 1) / bs.y, (f.n2 + bs.z - 1) / bs.z);
  if (f.thermo) fz_project_kernel<T, true><<<grid, bs, 0, st>>>(f);
  else fz_project_kernel<T, false><<<grid, bs, 0, st>>>(f);
}

template void launch_fz_momentum<double>(const FzMomentum<double>&, int, cudaStream_t);
template void launch_fz_momentum<float>(const FzMomentum<float>&, int, cudaStream_t);
template void launch_fz_wall_visc<double>(const FzMomentum<double>&, double*, double*, const double*, cudaStream_t);
template void launch_fz_wall_visc<float>(const FzMomentum<float>&, float*, float*, const float*, cudaStream_t);
template void launch_fz_update<double>(double*, double*, double*, const double*, const double*, const double*,
                                       const double*, int, int, int, int, int, double, int, double, cudaStream_t);
template void launch_fz_update<float>(float*, float*, float*, const float*, const float*, const float*,
                                      const double*, int, int, int, int, int, double, int, double, cudaStream_t);
template void launch_fz_energy<double>(const FzEnergy<double>&, cudaStream_t);
template void launch_fz_energy<float>(const FzEnergy<float>&, cudaStream_t);
template void launch_fz_energy_walls<double>(const FzEnergy<double>&, int, double*, cudaStream_t);
template void launch_fz_energy_walls<float>(const FzEnergy<float>&, int, float*, cudaStream_t);
template void launch_fz_update_div<double>(const FzUpdateDiv<double>&, cudaStream_t);
template void launch_fz_update_div<float>(const FzUpdateDiv<float>&, cudaStream_t);
template void launch_fz_project<double>(const FzProject<double>&, cudaStream_t);
template void launch_fz_project<float>(const FzProject<float>&, cudaStream_t);

}  // namespace chs
