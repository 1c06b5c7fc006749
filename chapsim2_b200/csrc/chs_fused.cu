// Fused momentum right-hand side for the explicit schemes (see chs_fused.cuh).
//
// Compute_momentum_rhs (src/eq_momentum2.f90:101-1571, Cartesian branches) with the fractional
// step Calculate_momentum_fractional_step (:35-71), per output value:
//   x: d/dx[-u u + 2 mu/Re (du/dx - div/3)] + d/dy[-v u + mu/Re (du/dy + dv/dx)]
//      + d/dz[-w u + mu/Re (du/dz + dw/dx)] - dp/dx            (:796-966)
//   y: d/dx[-u v + mu/Re (du/dy + dv/dx)] + d/dy[-v v + 2 mu/Re (dv/dy - div/3)]
//      + d/dz[-w v + mu/Re (dv/dz + dw/dy)] - dp/dy            (:978-1242)
//   z: d/dx[-u w + mu/Re (du/dz + dw/dx)] + d/dy[-v w + mu/Re (dv/dz + dw/dy)]
//      + d/dz[-w w + 2 mu/Re (dw/dz - div/3)] - dp/dz          (:1262-1457)
// with the first velocity factor of each convective product replaced by the interpolated momentum
// g and the viscosity interpolated to the stress points for variable properties (:576-703).  Every
// interpolation and derivative is the plan the operator path launches (same coefficients, same
// boundary rows, same arithmetic order), evaluated in registers where the sum needs it.
#include <cuda_runtime.h>

#include <stdexcept>

#include "chs_fused.cuh"
#include "chs_stencil_dev.cuh"

namespace chs {

namespace {

// CD2 bulk formula of family FAM at row p (bulk_fn with r2 = 0)
template <int FAM, typename T, typename F>
__device__ __forceinline__ T fz_bulk(const F& f, int p, T r1) {
  if (FAM == M1P2C) return r1 * (f(p) + f(p + 1));
  if (FAM == M1C2P) return r1 * (f(p) + f(p - 1));
  if (FAM == D1C2P) return r1 * (f(p) - f(p - 1));
  return r1 * (f(p + 1) - f(p));  // D1P2C
}

// periodic line: every row the bulk formula with wrapped indices (the plan's wrap flag)
template <int FAM, typename T, typename F>
__device__ __forceinline__ T fz_per(const FzOp& o, int p, int nin, const F& f) {
  auto w = [&](int q) -> T { return f(q < 0 ? q + nin : (q >= nin ? q - nin : q)); };
  return fz_bulk<FAM, T>(w, p, T(o.r1)) * T(o.dd);
}

// the plan's boundary row p over the input f and the boundary planes (out of line: boundary rows are
// a few wall rows, and inlining them into every composed expression multiplies the code)
template <typename T, typename F>
__device__ __forceinline__ T fz_special(const OpPlan* __restrict__ P, int p, const T* __restrict__ fbc, int nl, int L,
                                     F f) {
  T v = T(0);
  const int ns = P->nspec;
  for (int s = 0; s < ns; ++s) {
    if (P->sp[s].row != p) continue;
    const SpecialRow& R = P->sp[s];
    T acc = T(0);
    const int nt = R.nt;
    for (int t = 0; t < nt; ++t) acc += T(R.w[t]) * f(R.idx[t]);
    for (int u = 0; u < 4; ++u)
      if (R.wb[u] != 0.0) acc += T(R.wb[u]) * fbc[u * nl + L];
    v = acc * T(P->dd);
  }
  return v;
}

// the y metric and the Neumann overrides of stencil_op_kernel
template <typename T>
__device__ __forceinline__ T fz_finish(const FzOp& o, const double* __restrict__ table, const T* __restrict__ fbc,
                                       int nl, int L, int p, T v) {
  if (o.lmap >= 0) v *= T(table[o.lmap + p]);
  if ((o.neu & 1) && p == 0) v = fbc[L];
  if ((o.neu & 2) && p == o.nout - 1) v = fbc[nl + L];
  return v;
}

// y line with walls, a row in the bulk range: the bulk formula and the y metric
template <int FAM, typename T, typename F>
__device__ __forceinline__ T fz_ybulk(const FzOp& o, const double* __restrict__ table, int p, const F& f) {
  T v = fz_bulk<FAM, T>(f, p, T(o.r1)) * T(o.dd);
  if (o.lmap >= 0) v *= T(table[o.lmap + p]);
  return v;
}

// y line with walls: bulk rows or the plan's boundary rows
template <int FAM, typename T, typename F>
__device__ __forceinline__ T fz_wall(const FzOp& o, const OpPlan* __restrict__ plans, const double* __restrict__ table,
                                     const T* __restrict__ fbc, int nl, int L, int p, const F& f) {
  T v;
  if (p >= o.b_lo && p <= o.b_hi) v = fz_bulk<FAM, T>(f, p, T(o.r1)) * T(o.dd);
  else v = fz_special<T>(plans + o.plan, p, fbc, nl, L, f);
  return fz_finish<T>(o, table, fbc, nl, L, p, v);
}

// The inner operators at one position.  Arrays all have x extent n0 and z extent n2; their y
// extent is nc1 (cell rows: qx, qz, p, gx, gz, mu) or np1 (point rows: qy, gy).  PY: periodic y.
// E: rows near the walls, where y operators may take their plans' boundary rows; the interior rows
// (every y operator of every level in its bulk range, checked by the host) compile without them.
template <typename T, bool TH, bool PY, bool E>
struct FzCtx {
  const FzMomentum<T>& f;
  int nl;  // lines of a y operator (n0 * n2)

  __device__ __forceinline__ T at(const T* a, int ny, int i, int j, int k) const {
    return __ldg(a + ((int64_t)k * ny + j) * f.n0 + i);
  }
  template <int FAM, typename F>
  __device__ __forceinline__ T xop(int s, int i, const F& g) const { return fz_per<FAM, T>(f.in[s], i, f.n0, g); }
  template <int FAM, typename F>
  __device__ __forceinline__ T zop(int s, int k, const F& g) const { return fz_per<FAM, T>(f.in[s], k, f.n2, g); }
  template <int FAM, typename F>
  __device__ __forceinline__ T yop(int s, const T* fbc, int i, int j, int k, int nin, const F& g) const {
    if (PY) return fz_per<FAM, T>(f.in[s], j, nin, g);
    if (!E) return fz_ybulk<FAM, T>(f.in[s], f.table, j, g);
    return fz_wall<FAM, T>(f.in[s], f.plans, f.table, fbc, nl, i + f.n0 * k, j, g);
  }
#define FZ_X(FAM, S, A, NY) xop<FAM>(S, i, [&](int q) { return at(A, NY, q, j, k); })
#define FZ_Z(FAM, S, A, NY) zop<FAM>(S, k, [&](int q) { return at(A, NY, i, j, q); })
#define FZ_Y(FAM, S, A, NY, FB) yop<FAM>(S, FB, i, j, k, NY, [&](int q) { return at(A, NY, i, q, k); })
  // velocity interpolations and derivatives (src/eq_momentum2.f90:347-508)
  __device__ __forceinline__ T qxix(int i, int j, int k) const { return FZ_X(M1P2C, FI_QX_MX, f.qx, f.nc1); }
  __device__ __forceinline__ T qxdx(int i, int j, int k) const { return FZ_X(D1P2C, FI_QX_DX, f.qx, f.nc1); }
  __device__ __forceinline__ T qxdy(int i, int j, int k) const { return FZ_Y(D1C2P, FI_QX_DY, f.qx, f.nc1, f.fyqx); }
  __device__ __forceinline__ T qxiy(int i, int j, int k) const { return FZ_Y(M1C2P, FI_QX_MY, f.qx, f.nc1, f.fyqx); }
  __device__ __forceinline__ T qxiz(int i, int j, int k) const { return FZ_Z(M1C2P, FI_QX_MZ, f.qx, f.nc1); }
  __device__ __forceinline__ T qxdz(int i, int j, int k) const { return FZ_Z(D1C2P, FI_QX_DZ, f.qx, f.nc1); }
  __device__ __forceinline__ T qydx(int i, int j, int k) const { return FZ_X(D1C2P, FI_QY_DX, f.qy, f.np1); }
  __device__ __forceinline__ T qyix(int i, int j, int k) const { return FZ_X(M1C2P, FI_QY_MX, f.qy, f.np1); }
  __device__ __forceinline__ T qydy(int i, int j, int k) const { return FZ_Y(D1P2C, FI_QY_DY, f.qy, f.np1, (const T*)nullptr); }
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
    return xop<M1C2P>(FI_MU_YX, i, [&](int q) { return muy(q, j, k); });
  }
  __device__ __forceinline__ T muxz(int i, int j, int k) const {
    return zop<M1C2P>(FI_MU_XZ, k, [&](int q) { return mux(i, j, q); });
  }
  __device__ __forceinline__ T muyz(int i, int j, int k) const {
    return zop<M1C2P>(FI_MU_YZ, k, [&](int q) { return muy(i, j, q); });
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
  // s*(a + c*b), times m with variable properties (linm)
  __device__ __forceinline__ T lin(double s, T a, double c, T b) const { return T(s) * (a + T(c) * b); }

  // ---- the viscous and convective expressions at the stress points
  // cell centre, component c (0 x, 1 y, 2 z): conv -(ci*qi), visc s*(qidi - div/3)[*mu]
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
    T d;
    T dv;
    if (C == 0) { d = qxdx(i, j, k); dv = divc(d, i, j, k); }
    else if (C == 1) { d = qydy(i, j, k); dv = divc(qxdx(i, j, k), i, j, k); }
    else { d = qzdz(i, j, k); dv = divc(qxdx(i, j, k), i, j, k); }
    const T v = lin(s, d, -1.0 / 3.0, dv);
    return TH ? v * muc(i, j, k) : v;
  }
  // xy point (ppc): conv of x-momentum -(gyix*qxiy), of y-momentum -(gxiy*qyix); visc shared
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
  // xz point (pcp): x-momentum -(gzix*qxiz), z-momentum -(gxiz*qzix)
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
  // yz point (cpp): y-momentum -(qyiz*gziy), z-momentum -(gyiz*qziy)
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

  // op(conv) + rre*op(visc) of one direction, added to acc (`first`: stored).  x and z are periodic
  // with identical bulk plans for both terms, so one operator runs on conv + (s*rre)*visc; in y the
  // bulk rows do the same, and a boundary row applies each term's own plan (the combined planes
  // when the pair merges, as the operator path does)
  template <int FAM, int DIR, typename FC, typename FV>
  __device__ __forceinline__ T pair(const FzPair<T>& pr, T acc, bool first, int i, int j, int k, int nin, double sv,
                                    const FC& conv, const FV& visc) const {
    const double sr = sv * f.rre;
    auto comb = [&](int q) -> T {
      T e = conv(q);
      e += visc(sr, q);
      return e;
    };
    T v;
    if (DIR != 1 || PY) {
      v = fz_per<FAM, T>(pr.a, DIR == 0 ? i : (DIR == 1 ? j : k), nin, comb);
    } else if (!E) {
      v = fz_ybulk<FAM, T>(pr.a, f.table, j, comb);
    } else {
      const int L = i + f.n0 * k;
      if (j >= pr.a.b_lo && j <= pr.a.b_hi) {
        v = fz_finish<T>(pr.a, f.table, pr.fa, nl, L, j, fz_bulk<FAM, T>(comb, j, T(pr.a.r1)) * T(pr.a.dd));
      } else if (pr.merged) {
        v = fz_finish<T>(pr.a, f.table, pr.fa, nl, L, j, fz_special<T>(f.plans + pr.a.plan, j, pr.fa, nl, L, comb));
      } else {
        const T va = fz_finish<T>(pr.a, f.table, pr.fa, nl, L, j,
                                  fz_special<T>(f.plans + pr.a.plan, j, pr.fa, nl, L, [&](int q) { return conv(q); }));
        const T vb = fz_finish<T>(pr.b, f.table, pr.fb, nl, L, j,
                                  fz_special<T>(f.plans + pr.b.plan, j, pr.fb, nl, L, [&](int q) { return visc(sv, q); }));
        v = va + T(f.rre) * vb;
      }
    }
    return first ? v : acc + v;
  }

  // the fractional step of the operator path's O_FRAC store (pfc = 1 * v)
  __device__ __forceinline__ void frac(int c, int64_t a, T F, T v) const {
    const T tdt = T(f.dt), tg = T(f.gam), tz = T(f.zeta), ta = T(f.alpha);
    const T pfc = T(1.0) * v;
    const T last = f.m0[c][a];
    T tot = tg * F + tz * last;
    f.m0[c][a] = F;
    tot = tot + ta * pfc;
    f.m[c][a] = tdt * tot;
  }
};

// one momentum component C (0 x, 1 y, 2 z) per thread and output value.  Interior launch (E
// false): rows [row0, row0 + gridDim.y * blockDim.y) of the component's grid; edge launch (E
// true): blockIdx.y indexes the edge rows, [0, row0) then [row1, ny).
template <typename T, bool TH, bool PY, int C, bool E>
__global__ void __launch_bounds__(256) fz_momentum_kernel(const __grid_constant__ FzMomentum<T> f, int row0, int row1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int n0 = f.n0, nc1 = f.nc1, np1 = f.np1, n2 = f.n2;
  int j;
  if (E) j = blockIdx.y < row0 ? (int)blockIdx.y : row1 + ((int)blockIdx.y - row0);
  else j = row0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= n0 || j >= (E ? (C == 1 ? np1 : nc1) : row1) || k >= n2) return;
  const FzCtx<T, TH, PY, E> c{f, n0 * n2};
  const int L = i + n0 * k;
  T F, v;
  if (C == 0) {
    // x-momentum at (i, j, k) of the qx grid
    F = c.template pair<D1C2P, 0>(
        f.term[0][0], T(0), true, i, j, k, n0, 2.0, [&](int q) { return c.template conv_c<0>(q, j, k); },
        [&](double s, int q) { return c.template visc_c<0>(s, q, j, k); });
    F = c.template pair<D1P2C, 1>(
        f.term[0][1], F, false, i, j, k, np1, 1.0, [&](int q) { return c.template conv_xy<0>(i, q, k); },
        [&](double s, int q) { return c.visc_xy(s, i, q, k); });
    F = c.template pair<D1P2C, 2>(
        f.term[0][2], F, false, i, j, k, n2, 1.0, [&](int q) { return c.template conv_xz<0>(i, j, q); },
        [&](double s, int q) { return c.visc_xz(s, i, j, q); });
    v = fz_per<D1C2P, T>(f.pres[0], i, n0, [&](int q) { return T(-1.0) * c.pr(q, j, k); });
    c.frac(0, ((int64_t)k * nc1 + j) * n0 + i, F, v);
  } else if (C == 1) {
    // y-momentum at (i, j, k) of the qy grid
    F = c.template pair<D1P2C, 0>(
        f.term[1][0], T(0), true, i, j, k, n0, 1.0, [&](int q) { return c.template conv_xy<1>(q, j, k); },
        [&](double s, int q) { return c.visc_xy(s, q, j, k); });
    F = c.template pair<D1C2P, 1>(
        f.term[1][1], F, false, i, j, k, nc1, 2.0, [&](int q) { return c.template conv_c<1>(i, q, k); },
        [&](double s, int q) { return c.template visc_c<1>(s, i, q, k); });
    F = c.template pair<D1P2C, 2>(
        f.term[1][2], F, false, i, j, k, n2, 1.0, [&](int q) { return c.template conv_yz<1>(i, j, q); },
        [&](double s, int q) { return c.visc_yz(s, i, j, q); });
    auto pf = [&](int q) { return T(-1.0) * c.pr(i, q, k); };
    if (PY) v = fz_per<D1C2P, T>(f.pres[1], j, nc1, pf);
    else if (!E) v = fz_ybulk<D1C2P, T>(f.pres[1], f.table, j, pf);
    else v = fz_wall<D1C2P, T>(f.pres[1], f.plans, f.table, f.fpres[1], c.nl, L, j, pf);
    c.frac(1, ((int64_t)k * np1 + j) * n0 + i, F, v);
  } else {
    // z-momentum at (i, j, k) of the qz grid
    F = c.template pair<D1P2C, 0>(
        f.term[2][0], T(0), true, i, j, k, n0, 1.0, [&](int q) { return c.template conv_xz<2>(q, j, k); },
        [&](double s, int q) { return c.visc_xz(s, q, j, k); });
    F = c.template pair<D1P2C, 1>(
        f.term[2][1], F, false, i, j, k, np1, 1.0, [&](int q) { return c.template conv_yz<2>(i, q, k); },
        [&](double s, int q) { return c.visc_yz(s, i, q, k); });
    F = c.template pair<D1C2P, 2>(
        f.term[2][2], F, false, i, j, k, n2, 2.0, [&](int q) { return c.template conv_c<2>(i, j, q); },
        [&](double s, int q) { return c.template visc_c<2>(s, i, j, q); });
    v = fz_per<D1C2P, T>(f.pres[2], k, n2, [&](int q) { return T(-1.0) * c.pr(i, j, q); });
    c.frac(2, ((int64_t)k * nc1 + j) * n0 + i, F, v);
  }
}

// the wall rows of the y-viscous boundary value (fbcy_velo: src/eq_momentum2.f90:374-442, :537-546,
// :1156-1171): qxdx_cpc = d/dx qxiy, qydy_cpc = d/dy qyiy, qzdz_cpc = d/dz qziy at the two walls
template <typename T, bool TH>
__global__ void fz_wall_visc_kernel(const __grid_constant__ FzMomentum<T> f, T* __restrict__ fvisc2,
                                    T* __restrict__ fcomb, const T* __restrict__ fconv2) {
  const int nl = f.n0 * f.n2;
  const FzCtx<T, TH, false, true> c{f, nl};
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nl; g += gridDim.x * blockDim.x) {
    const int k = g / f.n0, i = g - k * f.n0;
    for (int side = 0; side < 2; ++side) {
      const int j = side == 0 ? 0 : f.np1 - 1;
      const T ddx = fz_per<D1P2C, T>(f.in[FI_W_DX], i, f.n0, [&](int q) { return c.qxiy(q, j, k); });
      const T ddy = fz_wall<D1C2P, T>(f.in[FI_W_DY], f.plans, f.table, f.fyqy, nl, g, j,
                                      [&](int q) { return c.qyiy(i, q, k); });
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
    const int64_t a = ((int64_t)k * nc1 + j) * n0 + i;
    const T s = bulk ? T(bulk[0]) : T(0);
    ux[a] = ux[a] + (mx[a] - s);
    uz[a] = uz[a] + (mz[a] - T(0));
  }
  const int64_t b = ((int64_t)k * np1 + j) * n0 + i;
  T v = uy[b] + (my[b] - T(0));
  if (s0 && j == 0) v = T(v0);
  if (s1 && j == np1 - 1) v = T(v1);
  uy[b] = v;
}

}  // namespace

template <typename T, bool TH, bool PY, int C>
void launch_fz_c(const FzMomentum<T>& f, cudaStream_t st) {
  const int ny = C == 1 ? f.np1 : f.nc1;
  // interior rows [m, ny - m) without boundary-row code (all rows when y is periodic); the host
  // checked that every y plan's bulk range covers rows 2 .. n-3 of its output
  const int m = PY ? 0 : (ny > 2 * kFzEdge ? kFzEdge : ny / 2);
  const int r0 = m, r1 = ny - m;
  if (r1 > r0) {
    const dim3 bs(32, 4, 2);
    const dim3 grid((f.n0 + bs.x - 1) / bs.x, (r1 - r0 + bs.y - 1) / bs.y, (f.n2 + bs.z - 1) / bs.z);
    fz_momentum_kernel<T, TH, PY, C, false><<<grid, bs, 0, st>>>(f, r0, r1);
  }
  if (!PY && m > 0) {
    const dim3 bs(32, 1, 8);
    const dim3 grid((f.n0 + bs.x - 1) / bs.x, r0 + (ny - r1), (f.n2 + bs.z - 1) / bs.z);
    fz_momentum_kernel<T, TH, PY, C, true><<<grid, bs, 0, st>>>(f, r0, r1);
  }
}

template <typename T, bool TH, bool PY>
void launch_fz_c(const FzMomentum<T>& f, int c, cudaStream_t st) {
  if (c == 0) launch_fz_c<T, TH, PY, 0>(f, st);
  else if (c == 1) launch_fz_c<T, TH, PY, 1>(f, st);
  else launch_fz_c<T, TH, PY, 2>(f, st);
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
  const int blocks = (nl + 255) / 256 < 148 ? (nl + 255) / 256 : 148;
  if (f.thermo) fz_wall_visc_kernel<T, true><<<blocks, 256, 0, st>>>(f, fvisc2, fcomb, fconv2);
  else fz_wall_visc_kernel<T, false><<<blocks, 256, 0, st>>>(f, fvisc2, fcomb, fconv2);
}

template <typename T>
void launch_fz_update(T* ux, T* uy, T* uz, const T* mx, const T* my, const T* mz, const double* bulk, int n0,
                      int nc1, int np1, int n2, int s0, double v0, int s1, double v1, cudaStream_t st) {
  const dim3 grid((n0 + 127) / 128, np1, n2);
  fz_update_kernel<T><<<grid, 128, 0, st>>>(ux, uy, uz, mx, my, mz, bulk, n0, nc1, np1, n2, s0, v0, s1, v1);
}

template void launch_fz_momentum<double>(const FzMomentum<double>&, int, cudaStream_t);
template void launch_fz_momentum<float>(const FzMomentum<float>&, int, cudaStream_t);
template void launch_fz_wall_visc<double>(const FzMomentum<double>&, double*, double*, const double*, cudaStream_t);
template void launch_fz_wall_visc<float>(const FzMomentum<float>&, float*, float*, const float*, cudaStream_t);
template void launch_fz_update<double>(double*, double*, double*, const double*, const double*, const double*,
                                       const double*, int, int, int, int, int, double, int, double, cudaStream_t);
template void launch_fz_update<float>(float*, float*, float*, const float*, const float*, const float*,
                                      const double*, int, int, int, int, int, double, int, double, cudaStream_t);

}  // namespace chs
