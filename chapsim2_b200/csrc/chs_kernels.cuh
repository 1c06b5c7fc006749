// Device kernels of the B200 CHAPSim2 hot path (declarations and launch helpers).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "chs_plan.h"

namespace chs {

// Input expression of a line operator, evaluated while a tile is staged:
// f = term0 + term1, each term one of
//   T_X     s * X
//   T_XY    s * (X * Y)
//   T_XpY   s * (X + c * Y)
//   T_XpYZ  s * (X + c * Y) * Z
enum TermMode { T_NONE = 0, T_X = 1, T_XY = 2, T_XpY = 3, T_XpYZ = 4 };
// Output of a line operator with result v: O_STORE out = g*v (or out += g*v when accumulating),
// O_DIV out = num / (g*v), O_MUL out = num * (g*v)
enum OutMode { O_STORE = 0, O_DIV = 1, O_MUL = 2, O_FRAC = 3 };
// O_FRAC: the operator value is the pressure-gradient term of the RK3 fractional step
// (Calculate_momentum_fractional_step): with cur = out, last = rhs0,
// rhs0 = cur, out = dt*(gam*cur + zeta*last + alpha*g*v), and, when qupd is set, qupd += out

template <typename T>
struct TermT {
  const T* X;
  const T* Y;
  int mode;
  double s, c;
  const T* Z;
};
using Term = TermT<double>;

template <typename T>
struct LineIOT {
  TermT<T> t[2];
  const T* fbc;       // boundary values, layout [4][nlines] (line order of the kernel), or null
  T* out;
  int accumulate;     // 0: out = g * r ; 1: out += g * r
  double g;
  int n1, n2, n3;     // extents of the INPUT array (x fastest)
  int omode;          // OutMode
  const T* onum;      // numerator / factor of O_DIV / O_MUL (output layout)
  int block;          // launch shape chosen by the autotuner: explicit-operator CTA size (0 = 256)
  int lt_max;         // and lines per CTA of the compact-scheme tile kernel (0 = 64)
  T* rhs0;            // O_FRAC: previous right-hand side (updated)
  T* qupd;            // O_FRAC: field advanced by the new right-hand side, or null
  double dt, gam, zeta, alpha;  // O_FRAC: RK3 coefficients of the substep
};
using LineIO = LineIOT<double>;

// Launch one plan over all lines of direction d.  `table` holds the LHS/mapping arrays.
void launch_line_op(int d, const OpPlan& plan, const LineIO& io, const double* table, cudaStream_t st);
void launch_line_op(int d, const OpPlan& plan, const LineIOT<float>& io, const double* table, cudaStream_t st);

// nondimensional property table on the device, sorted by T (FP64 columns)
struct ThermoTab {
  const double *t, *h, *d, *m, *k, *rhoh;
  int n;
  double dhmin, dhmax;
  // bracket index of the rho*h (0) and h (1) columns: for each of ix_nb uniform bins over
  // [ix_lo, ix_hi], the bisection state (a, b) that every value of the bin reaches, so the search
  // starts there and takes the same path as from (0, n-1); null: full bisection
  const int2* ix[2];
  double ix_lo[2], ix_hi[2], ix_iw[2];
  int ix_nb;
};

// ---- fused explicit operators: out(i,j,k) = sum over terms of g_m * op_m(in_m)(i,j,k) ----
// Every term is an explicit (no line solve) D1C2P or D1P2C plan of any direction whose output
// array has the shape of `out`; the sum is formed per output value, so the partial results never
// go through HBM.  Epilogues fold the RK3 fractional step (and, for the energy equation, the
// rho*h update and the table property update) into the same pass.
constexpr int kMaxFusedTerms = 6;
template <typename T>
struct FusedTerm {
  OpPlan P;
  int dir;
  TermT<T> t[2];      // input expression
  const T* fbc;       // boundary planes [4][nlines] or null
  int n1, n2, n3;     // input extents
  int nlines;
  double g;           // weight
  int group;          // 0: the flux sum F, 1: the pressure-gradient sum (EP_FRAC)
};
enum FusedEpilogue { EP_STORE = 0, EP_ACCUM = 1, EP_FRAC = 2, EP_ENERGY = 3 };
template <typename T>
struct FusedIO {
  FusedTerm<T> term[kMaxFusedTerms];
  int nterm;
  T* out;
  int m1, m2, m3;     // output extents
  int epilogue;
  // EP_FRAC: out = dt*(gam*F + zeta*rhs0 + alpha*pfc), rhs0 = F.
  // EP_ENERGY: r1 = dt*(gam*F + zeta*rhs0), rhs0 = F, rhoh += r1, then (props) h, T, kappa, rho,
  // mu from the table; out is unused
  T* rhs0;
  double dt, gam, zeta, alpha;
  T* rhoh;
  int props;
  T *h, *t, *k, *d, *m;
  ThermoTab tab;
};
template <typename T>
void launch_fused(const FusedIO<T>& f, const double* table, cudaStream_t st);

// number of lines of a direction for an input array of extents n1 x n2 x n3
inline int64_t num_lines(int d, int n1, int n2, int n3) {
  return d == 0 ? (int64_t)n2 * n3 : (d == 1 ? (int64_t)n1 * n3 : (int64_t)n1 * n2);
}

// ---- Poisson building blocks (double2 = complex) ----
struct FftPlan {
  int n;            // transform length (2^a 3^b)
  int nst;          // number of radix stages
  int radix[16];
  const double2* tw;  // exp(-2 pi i m / n), m = 0..n-1 (device)
  const float2* twf;  // the same rounded to FP32 (device; the FP32 spectrum of the mixed form), or null
};

// real x-lines (rows of length nx, R = double or float) -> half spectra (rows of nx/2+1) of
// complex type C (double2: FP64 transforms; float2: FP32 transforms of float rows)
template <typename R, typename C>
void launch_rfft_x(const FftPlan& fp, const R* in, C* out, int nrows, cudaStream_t st);
// half spectra -> real x-lines, scaled by `scale`
template <typename R, typename C>
void launch_irfft_x(const FftPlan& fp, const C* in, R* out, int nrows, double scale, cudaStream_t st);
// complex FFT along a strided axis: element (line, p) at base(line) + p*stride,
// line = a + na*b with base = a + b*bstride (a fastest); sign -1 forward, +1 backward
template <typename C>
void launch_cfft_axis(const FftPlan& fp, C* data, int na, int nb, int64_t bstride, int64_t stride, int sign,
                      cudaStream_t st);
// forward-sweep factors of the FISHPACK y solve per (kx, kz), computed once (layout (kz, j, kx))
void launch_ysolve_factor(double* Zr, double* D, int nxh, int ny, int nz, const double* pa, const double* pb,
                          const double* pc, const double* lamx, const double* lamz, cudaStream_t st);
// y tridiagonal solve per (kx, kz) of the FISHPACK path (TRID0 with the singular-pivot pin), in
// FP64 on a double2 or float2 spectrum
template <typename C>
void launch_ysolve(C* data, int nxh, int ny, int nz, const double* Zr, const double* D, const double* pa,
                   cudaStream_t st);
// poisson_010 y stage per (kx, kz) column: reordering, y FFT, cosine post-processing, the
// pentadiagonal solves (ptab: per system s = 0 odd / 1 even cosine modes and row r < ny/2 the
// rows [6][ny/2] sub-2, sub-1, t1, t2, super-1, super-2 with main diagonal
// -(((kx2 + kz2) + t1) + t2)) or, with ptab null, the division by -(kx2 + k2y + kz2), and the
// inverse steps; ayby holds sin and cos of (j pi / 2 ny), j < ny; scale the FFT normalisation
// (pfac: the elimination factors of the pentadiagonal systems from launch_dct_y_factor)
void launch_dct_y(const FftPlan& fp, double2* data, int nxh, int nz, const double* ayby, const double* k2x,
                  const double* k2z, const double* k2y, const double* ptab, const double* pfac, double scale,
                  cudaStream_t st);
// elimination factors of the poisson_010 pentadiagonal systems per (kx, |kz|) and parity, computed
// once: 8 * (ny/2) * (nz/2+1) * nxh doubles
void launch_dct_y_factor(double* pfac, int nxh, int nz, int ny, const double* k2x, const double* k2z,
                         const double* ptab, cudaStream_t st);
// 3D spectral division by -(kx'^2 + ky'^2 + kz'^2) (zero mode -> 0), with normalisation
void launch_spectral_divide(double2* data, int nxh, int ny, int nz, const double* k2x, const double* k2y,
                            const double* k2z, double norm, cudaStream_t st);

// ---- elementwise and reductions (T = double, or float in the mixed-precision form) ----
// rhs1 <- dt*(gamma*rhs1 + zeta*rhs0 + alpha*pfc); rhs0 <- old rhs1
template <typename T>
void launch_fractional_step(T* rhs1, T* rhs0, const T* pfc, int64_t n, double dt, double gam, double zeta,
                            double alpha, cudaStream_t st);
// weighted sum over (n1, n2, n3) with weight w[j] (double accumulation) -> partial sums;
// finalize writes out[0] = sum/vol
template <typename T>
void launch_weighted_mean(const T* a, const double* wy, int n1, int n2, int n3, double* partial, int npart,
                          double* out, double vol, cudaStream_t st);
// q <- q + rhs - (sub ? *sub : 0)
template <typename T>
void launch_update_q(T* q, const T* rhs, const double* sub, int64_t n, cudaStream_t st);
// set rows j = 0 and j = n2-1 of an (n1, n2, n3) array to v0 / v1 (flags select sides)
template <typename T>
void launch_set_yrows(T* a, int n1, int n2, int n3, int s0, double v0, int s1, double v1, cudaStream_t st);
// fbc planes [4][n1*n3] for y-lines: constant wall values
template <typename T>
void launch_fbcy_const(T* fbc, int n1, int n3, double v0, double v1, cudaStream_t st);
// fbc planes from the first/last y rows of `a` (extract_dirichlet_fbcy): out = s*(A_wall + c1*B_wall)*C
template <typename T>
void launch_fbcy_extract(T* fbc, const T* A, const T* B, const T* C, double c1, double s, double c2, int n1, int n2,
                         int n3, cudaStream_t st);
// out = sa*a + sb*b (b optional)
template <typename T>
void launch_axpby(T* out, const T* a, double sa, const T* b, double sb, int64_t n, cudaStream_t st,
                  const T* c = nullptr, double sc = 0.0);
// float <-> double field conversion
void launch_convert(float* out, const double* in, int64_t n, cudaStream_t st);
void launch_convert(double* out, const float* in, int64_t n, cudaStream_t st);
// ---- variable-property (thermal) kernels ----
// per-cell update from rho*h: h, T, kappa, rho, mu (ftp_refresh_thermal_properties_from_DH)
template <typename T>
void launch_property_update(const ThermoTab& tb, const T* rhoh, T* h, T* t, T* k, T* d, T* m, int64_t n,
                            cudaStream_t st);
// wall states from the wall rows (j = 0 and n2-1) of rho*h interpolated to the y faces:
// planes [4][n1*n3] of h, kappa, mu, rho; side s fills planes s and s+2; flags select sides
template <typename T>
void launch_wall_props(const ThermoTab& tb, const T* dh_cpc, int n1, int n2, int n3, int s0, int s1, T* fh, T* fk,
                       T* fm, T* fd, cudaStream_t st);
// energy fractional step and update: r1 = dt*(gam*r + zeta*r0); r0 = r; rhoh += r1
template <typename T>
void launch_energy_advance(T* rhs, T* rhs0, T* rhoh, int64_t n, double dt, double gam, double zeta,
                           cudaStream_t st);

// launch_energy_advance followed by launch_property_update of the new rho*h, in one pass
template <typename T>
void launch_energy_advance_props(const ThermoTab& tb, T* rhs, T* rhs0, T* rhoh, T* h, T* t, T* k, T* d, T* m,
                                 int64_t n, double dt, double gam, double zeta, cudaStream_t st);

// a[i] = v
template <typename T>
void launch_fill(T* a, double v, int64_t n, cudaStream_t st);

// running means of the flow and thermal statistics (update_statistics_flow/thermo,
// src/post_statistics.f90:152-283): with ac = 1/nstat, am = (nstat-1)/nstat,
// mean = am*mean + ac*x and product means am*m + (ac*a)*b; inputs at cell centres, FP64 sums
template <typename T>
struct StatsIO {
  const T* p;
  const T* u[3];   // cell-centre velocities (P2C interpolations)
  const T* t;      // temperature or null
  double* pm;
  double* um[3];
  double* uu[6];   // uu, vv, ww, uv, uw, vw
  double* tm;
  double* ttm;
  double ac, am;
  int64_t n;
};
template <typename T>
void launch_stats_update(const StatsIO<T>& s, cudaStream_t st);

// max |a| and NaN flag into out[0], out[1] (two-pass with partials)
void launch_absmax(const double* a, int64_t n, double* partial, int npart, double* out, cudaStream_t st);
// max |a| over the x slabs [0, 4), [4, n1 - 4), [n1 - 6, n1) of nrows rows of length n1 (the three
// monitors of Check_element_mass_conservation) as the bit patterns of the three doubles in out
void launch_absmax_slabs(const double* a, int n1, int64_t nrows, unsigned long long* out, cudaStream_t st);
// 0.5*(u^2+v^2+w^2) over ccc
void launch_ke_density(double* out, const double* u, const double* v, const double* w, int64_t n, cudaStream_t st);

}  // namespace chs
