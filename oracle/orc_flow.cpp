// ORACLE (test infrastructure only; never linked into the product library).
//
// CPU FP64 restatement of CHAPSim2's Cartesian RK3 substep, flow-only and variable-property:
//   geometry            src/geometry.f90:151-269, :410-530
//   boundary conditions src/bc_general.f90:137-248, :455-760, src/bc_dirichlet.f90:206-231, :461-516
//   momentum RHS        src/eq_momentum2.f90:101-1571 (Cartesian branches)
//   fractional step     src/eq_momentum2.f90:35-71, RK3 constants src/input_general.f90:851-886
//   mass-flux driving   src/eq_momentum2.f90:1547-1562, src/tools_general.f90:1202-1268
//   Poisson RHS         src/eq_momentum2.f90:1663-1718, src/eq_continuity.f90:91-161
//   FISHPACK Poisson    src/poisson_fishpack.f90:20-490 with the RFFTF/RFFTB sums documented in
//                       lib/fishpack4.1/fftpack.f:129-224 (evaluated here as direct DFT sums)
//   3D-FFT Poisson      src/poisson_1stderivcomp.f90:1016-1195 (poisson_000), :2343-2714
//   3FMD Poisson        src/poisson_1stderivcomp.f90:1457-1816 (poisson_010), :2718-3039
//                       (matrice_refinement), :420-561 (inversion5_v1); the 3FMD mapping
//                       src/geometry.f90:287-408
//   correction          src/eq_momentum2.f90:1577-1660, :1799-1932
//   KE monitor          src/io_monitor.f90:209-241
//   energy equation     src/eq_energy.f90:148-458 (Compute_energy_rhs, Solve_energy_eq)
//   property update     src/eq_energy.f90:14-146, src/input_thermo.f90:272-446 (table lookups)
//   q <-> g conversion  src/para_conversion.f90:5-227
//   momentum, thermal   src/eq_momentum2.f90:576-703 (g and mu interpolations) and the
//                       is_thermo branches of :796-1457, :1577-1660, :1799-1932
// Restriction: x and z must be periodic (the channel and Taylor-Green configurations).
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "orc_domain.h"

namespace orc {

static const double PI = 3.141592653589793238462643383279502884;

struct Arr {
  int n[3] = {0, 0, 0};
  std::vector<double> v;
  Arr() = default;
  Arr(int a, int b, int c, double val = 0.0) { n[0] = a; n[1] = b; n[2] = c; v.assign((size_t)a * b * c, val); }
  size_t size() const { return v.size(); }
  double& at(int i, int j, int k) { return v[((size_t)k * n[1] + j) * n[0] + i]; }
  double at(int i, int j, int k) const { return v[((size_t)k * n[1] + j) * n[0] + i]; }
};

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
static void tanh_mapping(const Domain& dm, bool node, int n, std::vector<double>& y, std::vector<double>& mp) {
  // Buildup_grid_mapping_1D_tanh (geometry.f90:151-269)
  double eta_shift = 0.0, eta_delta = 1.0;
  if (node) { eta_shift = 0.0; eta_delta = 1.0 / double(n - 1); }
  else { eta_shift = 1.0 / double(n) * 0.5; eta_delta = 1.0 / double(n); }
  std::vector<double> eta(n);
  eta[0] = 0.0 + eta_shift;
  for (int j = 2; j <= n; ++j) eta[j - 1] = eta[0] + double(j - 1) * eta_delta;
  double gamma = 1.0, delta = 0.0, ymin = 0.0, ymax = 0.0;
  if (dm.istret == 2) { gamma = 0.5; delta = 0.5; ymin = -1.0; ymax = 1.0; }
  else if (dm.istret == 3) { gamma = -1.0; delta = 1.0; ymin = 0.0; ymax = 1.0; }
  else if (dm.istret == 4) { gamma = 1.0; delta = 0.0; ymin = 0.0; ymax = 1.0; }
  else throw std::runtime_error("unsupported istret");
  const double beta = dm.rstret * 20.0;
  const double mm = std::tanh(beta * gamma);
  y.assign(n, 0.0);
  mp.assign(n, 0.0);
  for (int j = 0; j < n; ++j) {
    double yy = std::tanh(beta * (eta[j] - delta)) / mm;
    double m1 = 1.0 - yy * yy * mm * mm;
    if (m1 < 1.0e-20 && m1 > -1.0e-20) m1 = 1.0;
    else m1 = mm / beta / m1;
    const double ff = (dm.lyt - dm.lyb) / (ymax - ymin);
    yy = (yy - ymin) * ff + dm.lyb;
    m1 = m1 / ff;
    y[j] = yy;
    mp[j] = m1;
  }
}

// heaviside_step (modules.f90:960-971)
static double heaviside(double r) {
  if (r > 1.0e-20) return 1.0;
  if (r < -1.0e-20) return 0.0;
  return 0.5;
}

static void fmd_mapping(const Domain& dm, bool node, int n, std::vector<double>& y, std::vector<double>& mp) {
  // Buildup_grid_mapping_1D_3fmd (geometry.f90:287-408): the analytic stretching whose metric
  // 1/h' has a single cosine mode, as the 3D-FFT Poisson solver requires
  double eta_shift = 0.0, eta_delta = 1.0;
  if (node) { eta_shift = 0.0; eta_delta = 1.0 / double(n - 1); }
  else { eta_shift = 1.0 / double(n) * 0.5; eta_delta = 1.0 / double(n); }
  std::vector<double> eta(n);
  eta[0] = 0.0 + eta_shift;
  for (int j = 2; j <= n; ++j) eta[j - 1] = eta[0] + double(j - 1) * eta_delta;
  double gamma = 1.0, delta = 0.0;
  if (dm.istret == 1) { gamma = 1.0; delta = 0.0; }
  else if (dm.istret == 2) { gamma = 1.0; delta = 0.5; }
  else if (dm.istret == 3) { gamma = 0.5; delta = 0.5; }
  else if (dm.istret == 4) { gamma = 0.5; delta = 0.0; }
  else throw std::runtime_error("unsupported istret");
  const double beta = dm.rstret;
  const double alpha = (-1.0 + std::sqrt(1.0 + 4.0 * PI * PI * beta * beta)) / beta * 0.5;
  const double cc = std::sqrt(alpha * beta + 1.0) / std::sqrt(beta);
  const double dd = cc / std::sqrt(alpha);
  const double ee = cc * std::sqrt(alpha);
  const double st1 = (1.0 - 2.0 * delta) / gamma * 0.5;
  const double st2 = (3.0 - 2.0 * delta) / gamma * 0.5;
  y.assign(n, 0.0);
  mp.assign(n, 0.0);
  for (int j = 1; j <= n; ++j) {
    const double mm = PI * (gamma * eta[j - 1] + delta);
    double yy = std::atan(dd * std::tan(mm)) - std::atan(dd * std::tan(PI * delta)) +
                PI * (heaviside(eta[j - 1] - st1) + heaviside(eta[j - 1] - st2));
    yy = 1.0 / (gamma * ee) * yy;
    if (node && j == 1) yy = 0.0;
    if (node && j == n) yy = 1.0;
    y[j - 1] = yy * (dm.lyt - dm.lyb) + dm.lyb;
    mp[j - 1] = (alpha / PI + std::sin(mm) * std::sin(mm) / PI / beta) / (dm.lyt - dm.lyb);
  }
}

static void build_geometry(Domain& dm) {
  for (int d = 0; d < 3; ++d) {
    dm.np_geo[d] = dm.nc[d] + 1;
    dm.np[d] = dm.periodic[d] ? dm.nc[d] : dm.np_geo[d];
  }
  dm.h[0] = dm.lxx / double(dm.nc[0]);
  dm.h[2] = dm.lzz / double(dm.nc[2]);
  dm.h[1] = (dm.lyt - dm.lyb) / double(dm.nc[1]);
  dm.yp.assign(dm.np_geo[1], 0.0);
  dm.yc.assign(dm.nc[1], 0.0);
  dm.mppt.assign(dm.np_geo[1], 1.0);
  dm.mpcc.assign(dm.nc[1], 1.0);
  if (dm.stretch_y) {
    dm.h[1] = 1.0 / double(dm.nc[1]);
    // the 3D-FFT solver selects the 3FMD mapping, FISHPACK the tanh one (input_general.f90:552-553)
    if (dm.ifft == 3) {
      fmd_mapping(dm, true, dm.np_geo[1], dm.yp, dm.mppt);
      fmd_mapping(dm, false, dm.nc[1], dm.yc, dm.mpcc);
    } else {
      tanh_mapping(dm, true, dm.np_geo[1], dm.yp, dm.mppt);
      tanh_mapping(dm, false, dm.nc[1], dm.yc, dm.mpcc);
    }
  } else {
    for (int j = 0; j < dm.np_geo[1]; ++j) dm.yp[j] = double(j) * dm.h[1] + dm.lyb;
    for (int j = 0; j < dm.nc[1]; ++j) dm.yc[j] = double(j) * dm.h[1] + dm.h[1] * 0.5 + dm.lyb;
  }
  for (int d = 0; d < 3; ++d) {
    dm.h2r[d] = 1.0 / (dm.h[d] * dm.h[d]);
    dm.h1r[d] = 1.0 / dm.h[d];
  }
}

// ---------------------------------------------------------------------------
// boundary-condition configuration
// ---------------------------------------------------------------------------
enum { JSELF = 0, JGRAD = 1, JPROD = 2 };
// build_bc_symm_operation (bc_general.f90:455-509); mbc[side][j]
static void symm_op(const int ibc[2], int mbc[2][3], const int* jbc) {
  for (int i = 0; i < 2; ++i) mbc[i][0] = mbc[i][1] = mbc[i][2] = ibc[i];
  for (int i = 0; i < 2; ++i) {
    if (jbc) {
      if (ibc[i] == BC_SYMMETRIC && jbc[i] == BC_SYMMETRIC) mbc[i][JPROD] = BC_SYMMETRIC;
      else if (ibc[i] == BC_SYMMETRIC && jbc[i] == BC_ASYMMETRIC) mbc[i][JPROD] = BC_ASYMMETRIC;
      else if (ibc[i] == BC_ASYMMETRIC && jbc[i] == BC_SYMMETRIC) mbc[i][JPROD] = BC_ASYMMETRIC;
      else if (ibc[i] == BC_ASYMMETRIC && jbc[i] == BC_ASYMMETRIC) mbc[i][JPROD] = BC_SYMMETRIC;
      else {
        if (ibc[i] != jbc[i]) {
          if (ibc[i] == BC_DIRICHLET) mbc[i][0] = mbc[i][1] = mbc[i][2] = ibc[i];
          if (jbc[i] == BC_DIRICHLET) mbc[i][0] = mbc[i][1] = mbc[i][2] = jbc[i];
        } else {
          mbc[i][0] = mbc[i][1] = mbc[i][2] = ibc[i];
        }
      }
    } else {
      if (ibc[i] == BC_SYMMETRIC) { mbc[i][JSELF] = ibc[i]; mbc[i][JGRAD] = BC_ASYMMETRIC; mbc[i][JPROD] = ibc[i]; }
      else if (ibc[i] == BC_ASYMMETRIC) {
        mbc[i][JSELF] = ibc[i]; mbc[i][JGRAD] = BC_SYMMETRIC; mbc[i][JPROD] = BC_SYMMETRIC;
      } else mbc[i][0] = mbc[i][1] = mbc[i][2] = ibc[i];
    }
  }
}
static void prod_of(const int a[2], const int* b, int out[2]) {
  int m[2][3];
  symm_op(a, m, b);
  out[0] = m[0][JPROD]; out[1] = m[1][JPROD];
}
static void tau_of(const int var[2], const int ftp[2], int out[2]) {
  int m[2][3];
  symm_op(var, m, nullptr);
  int g[2] = {m[0][JGRAD], m[1][JGRAD]};
  prod_of(ftp, g, out);
}

static void configure_bcs(Domain& dm, const int nom[3][5][2]) {
  int nx[5][2], ny[5][2], nz[5][2];
  std::memcpy(nx, nom[0], sizeof(nx));
  std::memcpy(ny, nom[1], sizeof(ny));
  std::memcpy(nz, nom[2], sizeof(nz));
  for (int n = 0; n < 2; ++n) {  // config_calc_basic_ibc (bc_general.f90:141-150)
    if (nx[V_QX][n] == BC_SYMMETRIC) nx[V_QX][n] = BC_ASYMMETRIC;
    if (ny[V_QY][n] == BC_SYMMETRIC) ny[V_QY][n] = BC_ASYMMETRIC;
    if (nz[V_QZ][n] == BC_SYMMETRIC) nz[V_QZ][n] = BC_ASYMMETRIC;
  }
  std::memcpy(dm.ibcx, nx, sizeof(nx));
  std::memcpy(dm.ibcy, ny, sizeof(ny));
  std::memcpy(dm.ibcz, nz, sizeof(nz));
  int ftpx[2], ftpz[2];
  for (int n = 0; n < 2; ++n) {
    ftpx[n] = dm.ibcx[V_TM][n] == BC_NEUMANN ? BC_DIRICHLET : dm.ibcx[V_TM][n];
    dm.ibcy_ftp[n] = dm.ibcy[V_TM][n] == BC_NEUMANN ? BC_DIRICHLET : dm.ibcy[V_TM][n];
    ftpz[n] = dm.ibcz[V_TM][n] == BC_NEUMANN ? BC_DIRICHLET : dm.ibcz[V_TM][n];
    if (dm.ibcx[V_QX][n] == BC_DIRICHLET) dm.ibcx[V_PR][n] = BC_NEUMANN;
    if (dm.ibcy[V_QY][n] == BC_DIRICHLET) { dm.ibcy[V_PR][n] = BC_NEUMANN; dm.fbcy_const[V_PR][n] = 0.0; }
    if (dm.ibcz[V_QZ][n] == BC_DIRICHLET) dm.ibcz[V_PR][n] = BC_NEUMANN;
  }
  for (int n = 0; n < 2; ++n)
    if (dm.ibcx[V_QX][n] != BC_PERIODIC || dm.ibcz[V_QZ][n] != BC_PERIODIC)
      throw std::runtime_error("oracle: x and z must be periodic");
  // config_calc_eqs_ibc (bc_general.f90:512-677)
  prod_of(dm.ibcx[V_QX], dm.ibcx[V_QX], dm.mbcx_cov1);
  prod_of(dm.ibcy[V_QY], dm.ibcy[V_QX], dm.mbcy_cov1);
  prod_of(dm.ibcz[V_QZ], dm.ibcz[V_QX], dm.mbcz_cov1);
  tau_of(dm.ibcx[V_QX], ftpx, dm.mbcx_tau1);
  tau_of(dm.ibcy[V_QX], dm.ibcy_ftp, dm.mbcy_tau1);
  tau_of(dm.ibcz[V_QX], ftpz, dm.mbcz_tau1);
  prod_of(dm.ibcx[V_QX], dm.ibcx[V_QY], dm.mbcx_cov2);
  prod_of(dm.ibcy[V_QY], dm.ibcy[V_QY], dm.mbcy_cov2);
  prod_of(dm.ibcz[V_QZ], dm.ibcz[V_QY], dm.mbcz_cov2);
  tau_of(dm.ibcx[V_QY], ftpx, dm.mbcx_tau2);
  tau_of(dm.ibcy[V_QY], dm.ibcy_ftp, dm.mbcy_tau2);
  tau_of(dm.ibcz[V_QY], ftpz, dm.mbcz_tau2);
  prod_of(dm.ibcx[V_QX], dm.ibcx[V_QZ], dm.mbcx_cov3);
  prod_of(dm.ibcy[V_QY], dm.ibcy[V_QZ], dm.mbcy_cov3);
  prod_of(dm.ibcz[V_QZ], dm.ibcz[V_QZ], dm.mbcz_cov3);
  tau_of(dm.ibcx[V_QZ], ftpx, dm.mbcx_tau3);
  tau_of(dm.ibcy[V_QZ], dm.ibcy_ftp, dm.mbcy_tau3);
  tau_of(dm.ibcz[V_QZ], ftpz, dm.mbcz_tau3);
  dm.fbcy_velo_required = false;
  for (int v = V_QX; v <= V_QZ; ++v)
    for (int n = 0; n < 2; ++n)
      if (dm.ibcy[v][n] == BC_DIRICHLET || dm.ibcy[v][n] == BC_INTERIOR) dm.fbcy_velo_required = true;
}

// fbcy plane (n1, 4, n3) for a constant wall value: layers 1,3 = side 1, layers 2,4 = side 2
// (initialise_fbcy_given_const, bc_dirichlet.f90:206-231)
static std::vector<double> fbcy_const_plane(int n1, int n3, double v1, double v2) {
  std::vector<double> f((size_t)n1 * 4 * n3);
  for (int k = 0; k < n3; ++k)
    for (int u = 0; u < 4; ++u)
      for (int i = 0; i < n1; ++i) f[((size_t)k * 4 + u) * n1 + i] = (u % 2 == 0) ? v1 : v2;
  return f;
}
// extract_dirichlet_fbcy (bc_dirichlet.f90:42-56): layers 1/2 = first/last y row, 3:4 = 1:2
static std::vector<double> extract_fbcy(const Arr& a) {
  const int n1 = a.n[0], n2 = a.n[1], n3 = a.n[2];
  std::vector<double> f((size_t)n1 * 4 * n3);
  for (int k = 0; k < n3; ++k)
    for (int i = 0; i < n1; ++i) {
      double lo = a.at(i, 0, k), hi = a.at(i, n2 - 1, k);
      f[((size_t)k * 4 + 0) * n1 + i] = lo;
      f[((size_t)k * 4 + 1) * n1 + i] = hi;
      f[((size_t)k * 4 + 2) * n1 + i] = lo;
      f[((size_t)k * 4 + 3) * n1 + i] = hi;
    }
  return f;
}

// ---------------------------------------------------------------------------
// operator helper on Arr
// ---------------------------------------------------------------------------
static Arr op(const Domain& dm, int dir, int fam, const int ibc[2], const std::vector<double>* fbc, const Arr& in) {
  int n3[3] = {in.n[0], in.n[1], in.n[2]};
  int o[3] = {in.n[0], in.n[1], in.n[2]};
  o[dir] = op_out_len(dm, dir, fam);
  Arr out(o[0], o[1], o[2]);
  op3d(dm, dir, fam, ibc, fbc ? fbc->data() : nullptr, in.v.data(), n3, out.v.data());
  return out;
}
static const int PER2[2] = {BC_PERIODIC, BC_PERIODIC};

// Get_volumetric_average_3d_for_var_xcx (tools_general.f90:1202-1268)
static double vol_average(const Domain& dm, const Arr& a) {
  double vol = 0.0, fo = 0.0;
  const double dx = dm.h[0], dz = dm.h[2];
  for (int j = 0; j < a.n[1]; ++j) {
    double dy = dm.h[1];
    if (dm.stretch_y) dy = dm.h[1] / dm.mpcc[j];
    for (int k = 0; k < a.n[2]; ++k)
      for (int i = 0; i < a.n[0]; ++i) {
        fo = fo + a.at(i, j, k) * dy * dx * dz;
        vol = vol + dy * dx * dz;
      }
  }
  return fo / vol;
}

// ---------------------------------------------------------------------------
// momentum RHS (eq_momentum2.f90:101-1571), Cartesian, flow only, periodic x/z
// ---------------------------------------------------------------------------
struct Rhs3 {
  Arr mx, my, mz, px, py, pz;
};

static Arr op(const Domain& dm, int dir, int fam, const int ibc[2], const std::vector<double>* fbc, const Arr& in);
static std::vector<double> fbcy_const_plane(int n1, int n3, double v1, double v2);

static std::vector<double> extract_fbcy(const Arr& a);
// x and z are periodic for every configuration of this build: their property BCs are periodic
static const int* PER2_FTPX(const Domain&) { static const int p[2] = {BC_PERIODIC, BC_PERIODIC}; return p; }
static const int* PER2_FTPZ(const Domain&) { static const int p[2] = {BC_PERIODIC, BC_PERIODIC}; return p; }

// Property-dependent inputs of the momentum RHS (src/eq_momentum2.f90:576-703): interpolated
// momentum g and viscosity.  For constant-property flow every factor is 1 and g = q.
struct ThermoMom {
  Arr gxix_ccc, gxiy_ppc, gxiz_pcp, gyix_ppc, gyiy_ccc, gyiz_cpp, gzix_pcp, gziy_cpp, gziz_ccc;
  Arr mu_ccc, muixy_ppc, muixz_pcp, muiyz_cpp;
  std::vector<double> fbcy_mu;  // mu at the y walls (fbcy_mu_c4c)
};

static void thermo_mom_inputs(const Domain& dm, const Flow& fl, ThermoMom& t) {
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2];
  const int np0 = dm.np[0], np1 = dm.np[1], np2 = dm.np[2];
  const Thermo& th = fl.th;
  Arr gx(np0, nc1, nc2), gy(nc0, np1, nc2), gz(nc0, nc1, np2), mu(nc0, nc1, nc2);
  gx.v = th.gx; gy.v = th.gy; gz.v = th.gz; mu.v = th.mVisc;
  std::vector<double> fbcx_any((size_t)4 * np1 * np2 + 4 * nc1 * np2 + 16, MAXP);
  std::vector<double> fbcz_any((size_t)np0 * np1 * 4 + 16, MAXP);
  // no-slip walls: g = rho * q = 0 there (convert_primary_conservative, src/para_conversion.f90:5-227)
  const auto fg_x = fbcy_const_plane(np0, nc2, dm.fbcy_const[V_QX][0], dm.fbcy_const[V_QX][1]);
  const auto fg_y = fbcy_const_plane(nc0, nc2, dm.fbcy_const[V_QY][0], dm.fbcy_const[V_QY][1]);
  const auto fg_z = fbcy_const_plane(nc0, np2, dm.fbcy_const[V_QZ][0], dm.fbcy_const[V_QZ][1]);
  t.gxix_ccc = op(dm, 0, FAM_M1P2C, dm.ibcx[V_QX], &fbcx_any, gx);
  t.gxiy_ppc = op(dm, 1, FAM_M1C2P, dm.ibcy[V_QX], &fg_x, gx);
  t.gxiz_pcp = op(dm, 2, FAM_M1C2P, dm.ibcz[V_QX], &fbcz_any, gx);
  t.gyix_ppc = op(dm, 0, FAM_M1C2P, dm.ibcx[V_QY], &fbcx_any, gy);
  t.gyiy_ccc = op(dm, 1, FAM_M1P2C, dm.ibcy[V_QY], &fg_y, gy);
  t.gyiz_cpp = op(dm, 2, FAM_M1C2P, dm.ibcz[V_QY], &fbcz_any, gy);
  t.gzix_pcp = op(dm, 0, FAM_M1C2P, dm.ibcx[V_QZ], &fbcx_any, gz);
  t.gziy_cpp = op(dm, 1, FAM_M1C2P, dm.ibcy[V_QZ], &fg_z, gz);
  t.gziz_ccc = op(dm, 2, FAM_M1P2C, dm.ibcz[V_QZ], &fbcz_any, gz);
  // viscosity at the y walls from the wall states (fbcy_ftp%m)
  std::vector<double> fmu((size_t)nc0 * 4 * nc2);
  for (size_t n = 0; n < fmu.size(); ++n) fmu[n] = th.fbcy_ftp[n].m;
  t.mu_ccc = mu;
  Arr muiy_cpc = op(dm, 1, FAM_M1C2P, dm.ibcy_ftp, &fmu, mu);
  t.muixy_ppc = op(dm, 0, FAM_M1C2P, PER2_FTPX(dm), &fbcx_any, muiy_cpc);
  Arr mu_pcc = op(dm, 0, FAM_M1C2P, PER2_FTPX(dm), &fbcx_any, mu);
  t.muixz_pcp = op(dm, 2, FAM_M1C2P, PER2_FTPZ(dm), nullptr, mu_pcc);
  t.muiyz_cpp = op(dm, 2, FAM_M1C2P, PER2_FTPZ(dm), nullptr, muiy_cpc);
  // fbcy_mu_c4c: rows j = 1 and j = np of mu_cpc; planes 3, 4 repeat planes 1, 2
  t.fbcy_mu = extract_fbcy(muiy_cpc);
}

static void momentum_rhs(const Domain& dm, const Flow& fl, Rhs3& out) {
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2];
  const int np0 = dm.np[0], np1 = dm.np[1], np2 = dm.np[2];
  Arr qx(np0, nc1, nc2), qy(nc0, np1, nc2), qz(nc0, nc1, np2), pr(nc0, nc1, nc2);
  qx.v = fl.qx; qy.v = fl.qy; qz.v = fl.qz; pr.v = fl.pres;
  const auto fbcy_qx = fbcy_const_plane(np0, nc2, dm.fbcy_const[V_QX][0], dm.fbcy_const[V_QX][1]);
  const auto fbcy_qy = fbcy_const_plane(nc0, nc2, dm.fbcy_const[V_QY][0], dm.fbcy_const[V_QY][1]);
  const auto fbcy_qz = fbcy_const_plane(nc0, np2, dm.fbcy_const[V_QZ][0], dm.fbcy_const[V_QZ][1]);
  const auto fbcy_pr = fbcy_const_plane(nc0, nc2, dm.fbcy_const[V_PR][0], dm.fbcy_const[V_PR][1]);
  const int* bxqx = dm.ibcx[V_QX]; const int* byqx = dm.ibcy[V_QX]; const int* bzqx = dm.ibcz[V_QX];
  const int* bxqy = dm.ibcx[V_QY]; const int* byqy = dm.ibcy[V_QY]; const int* bzqy = dm.ibcz[V_QY];
  const int* bxqz = dm.ibcx[V_QZ]; const int* byqz = dm.ibcy[V_QZ]; const int* bzqz = dm.ibcz[V_QZ];
  // periodic x/z never read their boundary planes; any plane (here MAXP) stands for "present"
  std::vector<double> fbcx_any((size_t)4 * np1 * np2 + 4 * nc1 * np2 + 16, MAXP);
  std::vector<double> fbcz_any((size_t)np0 * np1 * 4 + 16, MAXP);

  // qx derived quantities (eq_momentum2.f90:347-383)
  Arr qxix_ccc = op(dm, 0, FAM_M1P2C, bxqx, &fbcx_any, qx);
  Arr qxdx_ccc = op(dm, 0, FAM_D1P2C, bxqx, &fbcx_any, qx);
  Arr qxdy_ppc = op(dm, 1, FAM_D1C2P, byqx, &fbcy_qx, qx);
  Arr qxiy_ppc = op(dm, 1, FAM_M1C2P, byqx, &fbcy_qx, qx);
  Arr qxiz_pcp = op(dm, 2, FAM_M1C2P, bzqx, &fbcz_any, qx);
  Arr qxdz_pcp = op(dm, 2, FAM_D1C2P, bzqx, &fbcz_any, qx);
  Arr qxdx_cpc;
  if (dm.fbcy_velo_required) qxdx_cpc = op(dm, 0, FAM_D1P2C, bxqx, nullptr, qxiy_ppc);
  // qy (eq_momentum2.f90:395-442)
  Arr qydx_ppc = op(dm, 0, FAM_D1C2P, bxqy, &fbcx_any, qy);
  Arr qyix_ppc = op(dm, 0, FAM_M1C2P, bxqy, &fbcx_any, qy);
  Arr qydy_ccc = op(dm, 1, FAM_D1P2C, byqy, nullptr, qy);
  Arr qyiy_ccc = op(dm, 1, FAM_M1P2C, byqy, &fbcy_qy, qy);
  Arr qydz_cpp = op(dm, 2, FAM_D1C2P, bzqy, &fbcz_any, qy);
  Arr qyiz_cpp = op(dm, 2, FAM_M1C2P, bzqy, &fbcz_any, qy);
  Arr qydy_cpc;
  if (dm.fbcy_velo_required) {
    Arr t = op(dm, 1, FAM_M1P2C, byqy, &fbcy_qy, qy);
    qydy_cpc = op(dm, 1, FAM_D1C2P, byqy, &fbcy_qy, t);
  }
  // qz (eq_momentum2.f90:454-508)
  Arr qzdx_pcp = op(dm, 0, FAM_D1C2P, bxqz, &fbcx_any, qz);
  Arr qzix_pcp = op(dm, 0, FAM_M1C2P, bxqz, &fbcx_any, qz);
  Arr qziy_cpp = op(dm, 1, FAM_M1C2P, byqz, &fbcy_qz, qz);
  Arr qzdy_cpp = op(dm, 1, FAM_D1C2P, byqz, &fbcy_qz, qz);
  Arr qziz_ccc = op(dm, 2, FAM_M1P2C, bzqz, &fbcz_any, qz);
  Arr qzdz_ccc = op(dm, 2, FAM_D1P2C, bzqz, nullptr, qz);
  Arr qzdz_cpc;
  if (dm.fbcy_velo_required) {
    Arr t = op(dm, 1, FAM_M1C2P, byqz, &fbcy_qz, qz);
    qzdz_cpc = op(dm, 2, FAM_D1P2C, bzqz, nullptr, t);
  }
  // divergence (eq_momentum2.f90:512-558)
  Arr div(nc0, nc1, nc2);
  for (size_t n = 0; n < div.size(); ++n) div.v[n] = ((0.0 + qxdx_ccc.v[n]) + qydy_ccc.v[n]) + qzdz_ccc.v[n];
  std::vector<double> fbcy_div;
  if (dm.fbcy_velo_required) {
    fbcy_div.assign((size_t)nc0 * 4 * nc2, 0.0);
    for (int k = 0; k < nc2; ++k)
      for (int i = 0; i < nc0; ++i)
        for (int side = 0; side < 2; ++side) {
          int j = side == 0 ? 0 : np1 - 1;
          double s = qxdx_cpc.at(i, j, k) + qydy_cpc.at(i, j, k) + qzdz_cpc.at(i, j, k);
          fbcy_div[((size_t)k * 4 + side) * nc0 + i] = s;
          fbcy_div[((size_t)k * 4 + side + 2) * nc0 + i] = s;
        }
  }
  const double rre = dm.rre;
  const double THIRD = 1.0 / 3.0;
  // first factors of the convection products (g for variable properties, q otherwise) and the
  // viscosity factors of the stresses (1 for constant properties)
  ThermoMom tmo;
  if (fl.thermo) thermo_mom_inputs(dm, fl, tmo);
  const bool TH = fl.thermo;
  const Arr& c_xix = TH ? tmo.gxix_ccc : qxix_ccc;
  const Arr& c_yix = TH ? tmo.gyix_ppc : qyix_ppc;
  const Arr& c_zix = TH ? tmo.gzix_pcp : qzix_pcp;
  const Arr& c_xiy = TH ? tmo.gxiy_ppc : qxiy_ppc;
  const Arr& c_yiy = TH ? tmo.gyiy_ccc : qyiy_ccc;
  const Arr& c_ziy = TH ? tmo.gziy_cpp : qziy_cpp;
  const Arr& c_xiz = TH ? tmo.gxiz_pcp : qxiz_pcp;
  const Arr& c_yiz = TH ? tmo.gyiz_cpp : qyiz_cpp;
  const Arr& c_ziz = TH ? tmo.gziz_ccc : qziz_ccc;
  auto MU = [&](const Arr& m, size_t n) { return TH ? m.v[n] : 1.0; };

  // ---- x-momentum (eq_momentum2.f90:796-966)
  Arr mx(np0, nc1, nc2), mxy(np0, nc1, nc2), mxz(np0, nc1, nc2), px(np0, nc1, nc2);
  {
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -c_xix.v[n] * qxix_ccc.v[n];
    Arr r = op(dm, 0, FAM_D1C2P, dm.mbcx_cov1, &fbcx_any, a);
    for (size_t n = 0; n < mx.size(); ++n) mx.v[n] = mx.v[n] + r.v[n];
  }
  {
    Arr a(np0, np1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -c_yix.v[n] * qxiy_ppc.v[n];
    Arr r = op(dm, 1, FAM_D1P2C, dm.mbcy_cov1, nullptr, a);
    for (size_t n = 0; n < mxy.size(); ++n) mxy.v[n] = mxy.v[n] + r.v[n];
  }
  {
    Arr a(np0, nc1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -c_zix.v[n] * qxiz_pcp.v[n];
    Arr r = op(dm, 2, FAM_D1P2C, dm.mbcz_cov1, nullptr, a);
    for (size_t n = 0; n < mxz.size(); ++n) mxz.v[n] = mxz.v[n] + r.v[n];
  }
  {
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -pr.v[n];
    Arr r = op(dm, 0, FAM_D1C2P, dm.ibcx[V_PR], &fbcx_any, a);
    for (size_t n = 0; n < px.size(); ++n) px.v[n] = px.v[n] + r.v[n];
  }
  {
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = 2.0 * MU(tmo.mu_ccc, n) * (qxdx_ccc.v[n] - THIRD * div.v[n]);
    Arr r = op(dm, 0, FAM_D1C2P, dm.mbcx_tau1, &fbcx_any, a);
    for (size_t n = 0; n < mx.size(); ++n) mx.v[n] = mx.v[n] + r.v[n] * rre;
  }
  {
    Arr a(np0, np1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qxdy_ppc.v[n] + qydx_ppc.v[n]) * MU(tmo.muixy_ppc, n);
    Arr r = op(dm, 1, FAM_D1P2C, dm.mbcy_tau1, nullptr, a);
    for (size_t n = 0; n < mxy.size(); ++n) mxy.v[n] = mxy.v[n] + r.v[n] * rre;
  }
  {
    Arr a(np0, nc1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qxdz_pcp.v[n] + qzdx_pcp.v[n]) * MU(tmo.muixz_pcp, n);
    Arr r = op(dm, 2, FAM_D1P2C, dm.mbcz_tau1, nullptr, a);
    for (size_t n = 0; n < mxz.size(); ++n) mxz.v[n] = mxz.v[n] + r.v[n] * rre;
  }
  for (size_t n = 0; n < mx.size(); ++n) mx.v[n] = mx.v[n] + mxy.v[n];
  for (size_t n = 0; n < mx.size(); ++n) mx.v[n] = mx.v[n] + mxz.v[n];

  // ---- y-momentum (eq_momentum2.f90:978-1242)
  Arr my(nc0, np1, nc2), myy(nc0, np1, nc2), myz(nc0, np1, nc2), py(nc0, np1, nc2);
  {
    Arr a(np0, np1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -c_xiy.v[n] * qyix_ppc.v[n];
    Arr r = op(dm, 0, FAM_D1P2C, dm.mbcx_cov2, nullptr, a);
    for (size_t n = 0; n < my.size(); ++n) my.v[n] = my.v[n] + r.v[n];
  }
  {
    std::vector<double> fb;
    if (dm.fbcy_velo_required) {
      // -fbcy_qy * fbcy_gy (thermo) or -fbcy_qy * fbcy_qy; the walls are at rest or moving with
      // a constant velocity, and fbcy_gy = fbcy_qy * rho there (src/para_conversion.f90:157-169)
      fb = fbcy_qy;
      for (size_t n = 0; n < fb.size(); ++n) {
        const double g = TH ? fb[n] * fl.th.fbcy_ftp[n].d : fb[n];
        fb[n] = -fb[n] * g;
      }
    } else fb.assign(fbcy_qy.size(), MAXP);
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -qyiy_ccc.v[n] * c_yiy.v[n];
    Arr r = op(dm, 1, FAM_D1C2P, dm.mbcy_cov2, &fb, a);
    for (size_t n = 0; n < myy.size(); ++n) myy.v[n] = myy.v[n] + r.v[n];
  }
  {
    Arr a(nc0, np1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -qyiz_cpp.v[n] * c_ziy.v[n];
    Arr r = op(dm, 2, FAM_D1P2C, dm.mbcz_cov2, nullptr, a);
    for (size_t n = 0; n < myz.size(); ++n) myz.v[n] = myz.v[n] + r.v[n];
  }
  {
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -pr.v[n];
    std::vector<double> fb = fbcy_pr;
    for (auto& v : fb) v = -v;
    Arr r = op(dm, 1, FAM_D1C2P, dm.ibcy[V_PR], &fb, a);
    for (size_t n = 0; n < py.size(); ++n) py.v[n] = py.v[n] + r.v[n];
  }
  {
    Arr a(np0, np1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qxdy_ppc.v[n] + qydx_ppc.v[n]) * MU(tmo.muixy_ppc, n);
    Arr r = op(dm, 0, FAM_D1P2C, dm.mbcx_tau2, nullptr, a);
    for (size_t n = 0; n < my.size(); ++n) my.v[n] = my.v[n] + r.v[n] * rre;
  }
  {
    std::vector<double> fb;
    if (dm.fbcy_velo_required) {
      fb = extract_fbcy(qydy_cpc);
      for (size_t n = 0; n < fb.size(); ++n) fb[n] = (fb[n] - THIRD * fbcy_div[n]) * 2.0 * (TH ? tmo.fbcy_mu[n] : 1.0);
    } else fb.assign(fbcy_qy.size(), MAXP);
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qydy_ccc.v[n] - THIRD * div.v[n]) * 2.0 * MU(tmo.mu_ccc, n);
    Arr r = op(dm, 1, FAM_D1C2P, dm.mbcy_tau2, &fb, a);
    for (size_t n = 0; n < myy.size(); ++n) myy.v[n] = myy.v[n] + r.v[n] * rre;
  }
  {
    Arr a(nc0, np1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qzdy_cpp.v[n] + qydz_cpp.v[n] - 0.0) * MU(tmo.muiyz_cpp, n);
    Arr r = op(dm, 2, FAM_D1P2C, dm.mbcz_tau2, nullptr, a);
    for (size_t n = 0; n < myz.size(); ++n) myz.v[n] = myz.v[n] + r.v[n] * rre;
  }
  for (size_t n = 0; n < my.size(); ++n) my.v[n] = my.v[n] + myy.v[n];
  for (size_t n = 0; n < my.size(); ++n) my.v[n] = my.v[n] + myz.v[n];

  // ---- z-momentum (eq_momentum2.f90:1262-1457)
  Arr mz(nc0, nc1, np2), mzy(nc0, nc1, np2), mzz(nc0, nc1, np2), pz(nc0, nc1, np2);
  {
    Arr a(np0, nc1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -c_xiz.v[n] * qzix_pcp.v[n];
    Arr r = op(dm, 0, FAM_D1P2C, dm.mbcx_cov3, nullptr, a);
    for (size_t n = 0; n < mz.size(); ++n) mz.v[n] = mz.v[n] + r.v[n];
  }
  {
    Arr a(nc0, np1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -c_yiz.v[n] * qziy_cpp.v[n];
    Arr r = op(dm, 1, FAM_D1P2C, dm.mbcy_cov3, nullptr, a);
    for (size_t n = 0; n < mzy.size(); ++n) mzy.v[n] = mzy.v[n] + r.v[n];
  }
  {
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -c_ziz.v[n] * qziz_ccc.v[n];
    Arr r = op(dm, 2, FAM_D1C2P, dm.mbcz_cov3, &fbcz_any, a);
    for (size_t n = 0; n < mzz.size(); ++n) mzz.v[n] = mzz.v[n] + r.v[n];
  }
  {
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = -pr.v[n];
    Arr r = op(dm, 2, FAM_D1C2P, dm.ibcz[V_PR], &fbcz_any, a);
    for (size_t n = 0; n < pz.size(); ++n) pz.v[n] = pz.v[n] + r.v[n];
  }
  {
    Arr a(np0, nc1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qxdz_pcp.v[n] + qzdx_pcp.v[n]) * MU(tmo.muixz_pcp, n);
    Arr r = op(dm, 0, FAM_D1P2C, dm.mbcx_tau3, nullptr, a);
    for (size_t n = 0; n < mz.size(); ++n) mz.v[n] = mz.v[n] + r.v[n] * rre;
  }
  {
    Arr a(nc0, np1, np2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qzdy_cpp.v[n] + qydz_cpp.v[n]) * MU(tmo.muiyz_cpp, n);
    Arr r = op(dm, 1, FAM_D1P2C, dm.mbcy_tau3, nullptr, a);
    for (size_t n = 0; n < mzy.size(); ++n) mzy.v[n] = mzy.v[n] + r.v[n] * rre;
  }
  {
    Arr a(nc0, nc1, nc2);
    for (size_t n = 0; n < a.size(); ++n) a.v[n] = (qzdz_ccc.v[n] - THIRD * div.v[n] + 0.0) * 2.0 * MU(tmo.mu_ccc, n);
    Arr r = op(dm, 2, FAM_D1C2P, dm.mbcz_tau3, &fbcz_any, a);
    for (size_t n = 0; n < mzz.size(); ++n) mzz.v[n] = mzz.v[n] + r.v[n] * rre;
  }
  for (size_t n = 0; n < mz.size(); ++n) mz.v[n] = mz.v[n] + mzy.v[n];
  for (size_t n = 0; n < mz.size(); ++n) mz.v[n] = mz.v[n] + mzz.v[n];

  out.mx = std::move(mx); out.my = std::move(my); out.mz = std::move(mz);
  out.px = std::move(px); out.py = std::move(py); out.pz = std::move(pz);
}

// Calculate_momentum_fractional_step (eq_momentum2.f90:35-71)
static void fractional_step(const Domain& dm, int isub, std::vector<double>& rhs0, std::vector<double>& rhs1,
                            const std::vector<double>& pfc) {
  for (size_t n = 0; n < rhs1.size(); ++n) {
    double cur = rhs1[n], last = rhs0[n];
    double tot = dm.tGamma[isub] * cur + dm.tZeta[isub] * last;
    rhs0[n] = cur;
    tot = tot + dm.tAlpha[isub] * pfc[n];
    rhs1[n] = dm.dt * tot;
  }
}

// ---------------------------------------------------------------------------
// Poisson: direct real DFT sums (RFFTF / RFFTB definitions)
// ---------------------------------------------------------------------------
struct RealDft {
  int n;
  std::vector<double> c, s;  // cos/sin(2 pi m / n)
  explicit RealDft(int n_) : n(n_), c(n_), s(n_) {
    for (int m = 0; m < n; ++m) { c[m] = std::cos(2.0 * PI * m / n); s[m] = std::sin(2.0 * PI * m / n); }
  }
  void forward(double* r) const {  // RFFTF
    std::vector<double> out(n);
    double s0 = 0.0;
    for (int i = 0; i < n; ++i) s0 += r[i];
    out[0] = s0;
    int L = (n % 2 == 0) ? n / 2 : (n + 1) / 2;
    for (int K = 2; K <= L; ++K) {
      double a = 0.0, b = 0.0;
      for (int i = 0; i < n; ++i) {
        int m = (int)(((long)(K - 1) * i) % n);
        a += r[i] * c[m];
        b += -r[i] * s[m];
      }
      out[2 * K - 3] = a;
      out[2 * K - 2] = b;
    }
    if (n % 2 == 0) {
      double a = 0.0;
      for (int i = 0; i < n; ++i) a += (i % 2 == 0 ? 1.0 : -1.0) * r[i];
      out[n - 1] = a;
    }
    std::memcpy(r, out.data(), sizeof(double) * n);
  }
  void backward(double* r) const {  // RFFTB
    std::vector<double> out(n);
    int L = (n % 2 == 0) ? n / 2 : (n + 1) / 2;
    for (int i = 0; i < n; ++i) {
      double v = r[0];
      if (n % 2 == 0) v += (i % 2 == 0 ? 1.0 : -1.0) * r[n - 1];
      for (int K = 2; K <= L; ++K) {
        int m = (int)(((long)(K - 1) * i) % n);
        v += 2.0 * r[2 * K - 3] * c[m] - 2.0 * r[2 * K - 2] * s[m];
      }
      out[i] = v;
    }
    std::memcpy(r, out.data(), sizeof(double) * n);
  }
};

// fishpack_root_1D for LP = 1 (poisson_fishpack.f90:60-110)
static void fishpack_root(int L, double c1, std::vector<double>& xrt, double& scal) {
  const double pi = 2.0 * std::asin(1.0);
  xrt.assign(L, 0.0);
  scal = double(L);
  const double dx = pi / (2.0 * scal);
  xrt[0] = 0.0;
  xrt[L - 1] = -4.0 * c1;
  for (int I = 3; I <= L; I += 2) {
    double s = std::sin(double(I - 1) * dx);
    xrt[I - 2] = -4.0 * c1 * s * s;
    xrt[I - 1] = xrt[I - 2];
  }
}

static void fishpack_init(Domain& dm) {
  double sx, sz;
  fishpack_root(dm.nc[0], dm.h2r[0], dm.xrt, sx);
  fishpack_root(dm.nc[2], dm.h2r[2], dm.zrt, sz);
  const int ny = dm.nc[1];
  dm.pa.assign(ny, 0.0); dm.pb.assign(ny, 0.0); dm.pc.assign(ny, 0.0);
  for (int j = 1; j <= ny; ++j) {  // poisson_fishpack.f90:312-323 (Cartesian: rp = rc = 1)
    dm.pa[j - 1] = dm.h2r[1] * dm.mpcc[j - 1] * dm.mppt[j - 1] * 1.0 * 1.0;
    dm.pc[j - 1] = dm.h2r[1] * dm.mpcc[j - 1] * dm.mppt[j] * 1.0 * 1.0;
  }
  for (int j = 0; j < ny; ++j) dm.pb[j] = -(dm.pa[j] + dm.pc[j]);
  if (!dm.periodic[1]) {
    dm.pb[0] = dm.pb[0] + dm.pa[0];
    dm.pa[0] = 0.0;
    dm.pb[ny - 1] = dm.pb[ny - 1] + dm.pc[ny - 1];
    dm.pc[ny - 1] = 0.0;
  }
}

// TRID0 (poisson_fishpack.f90:20-57)
static void trid0(int NG, double* T, const double* A, const double* BB, const double* C) {
  std::vector<double> D(NG);
  const int NR = NG, MM1 = NR - 1;
  double Z = 1.0 / BB[0];
  D[0] = C[0] * Z;
  T[0] = T[0] * Z;
  for (int I = 2; I <= MM1; ++I) {
    Z = 1.0 / (BB[I - 1] - A[I - 1] * D[I - 2]);
    D[I - 1] = C[I - 1] * Z;
    T[I - 1] = (T[I - 1] - A[I - 1] * T[I - 2]) * Z;
  }
  Z = BB[NR - 1] - A[NR - 1] * D[MM1 - 1];
  if (std::fabs(Z) > 1.0e-10) T[NR - 1] = (T[NR - 1] - A[NR - 1] * T[MM1 - 1]) / Z;
  else T[NR - 1] = 0.0;
  for (int IP = 1; IP <= MM1; ++IP) {
    int I = NR - IP;
    T[I - 1] = T[I - 1] - D[I - 1] * T[I];
  }
}

// fishpack_fft_simple (poisson_fishpack.f90:354-490)
static void poisson_fishpack(const Domain& dm, std::vector<double>& rhs) {
  const int nx = dm.nc[0], ny = dm.nc[1], nz = dm.nc[2];
  RealDft fx(nx), fz(nz);
  auto at = [&](int i, int j, int k) -> double& { return rhs[((size_t)k * ny + j) * nx + i]; };
#pragma omp parallel for collapse(2)
  for (int j = 0; j < ny; ++j)
    for (int k = 0; k < nz; ++k) {
      std::vector<double> t(nx);
      for (int i = 0; i < nx; ++i) t[i] = at(i, j, k);
      fx.forward(t.data());
      for (int i = 0; i < nx; ++i) at(i, j, k) = t[i];
    }
#pragma omp parallel for collapse(2)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      std::vector<double> t(nz);
      for (int k = 0; k < nz; ++k) t[k] = at(i, j, k);
      fz.forward(t.data());
      for (int k = 0; k < nz; ++k) at(i, j, k) = t[k];
    }
#pragma omp parallel for collapse(2)
  for (int i = 0; i < nx; ++i)
    for (int k = 0; k < nz; ++k) {
      std::vector<double> bb(ny), ty(ny);
      for (int j = 0; j < ny; ++j) {
        bb[j] = dm.pb[j] + dm.xrt[i] / (1.0 * 1.0) + dm.zrt[k];
        ty[j] = at(i, j, k);
      }
      trid0(ny, ty.data(), dm.pa.data(), bb.data(), dm.pc.data());
      for (int j = 0; j < ny; ++j) at(i, j, k) = ty[j];
    }
#pragma omp parallel for collapse(2)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j) {
      std::vector<double> t(nz);
      for (int k = 0; k < nz; ++k) t[k] = at(i, j, k);
      fz.backward(t.data());
      for (int k = 0; k < nz; ++k) at(i, j, k) = t[k];
    }
#pragma omp parallel for collapse(2)
  for (int j = 0; j < ny; ++j)
    for (int k = 0; k < nz; ++k) {
      std::vector<double> t(nx);
      for (int i = 0; i < nx; ++i) t[i] = at(i, j, k);
      fx.backward(t.data());
      for (int i = 0; i < nx; ++i) at(i, j, k) = t[i];
    }
  const double sx = double(nx), sz = double(nz);
  for (auto& v : rhs) v = v / sx / sz;
}

// waves(): modified wavenumber squared of the periodic C2P derivative (poisson_1stderivcomp.f90:2448-2470)
static std::vector<double> mod_k2(const Domain& dm, int d, int n, double len, double dh) {
  const Family& c2p = dm.T.fam[FAM_D1C2P];
  const int m = dm.iacc - 1;
  const double alc = c2p.f[2][0][BC_PERIODIC][m];
  const double ac = c2p.r[2][0][BC_PERIODIC][m] / dh;
  const double bc = c2p.r[2][1][BC_PERIODIC][m] / dh;
  std::vector<double> k2(n, 0.0);
  for (int i = 1; i <= n / 2 + 1; ++i) {
    double w = 2.0 * PI * double(i - 1) / double(n);
    double wp = ac * 2.0 * dh * std::sin(w * 0.5) + bc * 2.0 * dh * std::sin(3.0 * 0.5 * w);
    wp = wp / (1.0 + 2.0 * alc * std::cos(w));
    double v = double(n) * wp / len;
    k2[i - 1] = v * v;
  }
  for (int i = n / 2 + 2; i <= n; ++i) k2[i - 1] = k2[n - i + 1];
  (void)d;
  return k2;
}

// complex DFT along one axis of a (nx, ny, nz) complex array
static void cdft_axis(std::vector<std::complex<double>>& a, const int n3[3], int ax, int sign) {
  const int n = n3[ax];
  std::vector<std::complex<double>> w(n);
  for (int m = 0; m < n; ++m) w[m] = std::complex<double>(std::cos(2.0 * PI * m / n), sign * std::sin(2.0 * PI * m / n));
  const size_t st[3] = {1, (size_t)n3[0], (size_t)n3[0] * n3[1]};
  const int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
#pragma omp parallel for collapse(2)
  for (int b = 0; b < n3[o2]; ++b)
    for (int c = 0; c < n3[o1]; ++c) {
      std::vector<std::complex<double>> t(n), o(n);
      size_t base = b * st[o2] + c * st[o1];
      for (int i = 0; i < n; ++i) t[i] = a[base + i * st[ax]];
      for (int k = 0; k < n; ++k) {
        std::complex<double> s(0.0, 0.0);
        for (int i = 0; i < n; ++i) s += t[i] * w[(size_t)k * i % n];
        o[k] = s;
      }
      for (int i = 0; i < n; ++i) a[base + i * st[ax]] = o[i];
    }
}

// poisson_000 (poisson_1stderivcomp.f90:1016-1195).  The forward and backward half-cell
// phase shifts of the reference multiply each mode by e^{-i theta} and then e^{+i theta};
// they cancel, so the mode update reduces to the division by -(kx'^2 + ky'^2 + kz'^2).
static void poisson_3dfft(const Domain& dm, std::vector<double>& rhs) {
  const int nx = dm.nc[0], ny = dm.nc[1], nz = dm.nc[2];
  const int n3[3] = {nx, ny, nz};
  std::vector<std::complex<double>> a(rhs.size());
  for (size_t n = 0; n < rhs.size(); ++n) a[n] = rhs[n];
  for (int ax = 0; ax < 3; ++ax) cdft_axis(a, n3, ax, -1);
  auto kx = mod_k2(dm, 0, nx, dm.lxx, dm.h[0]);
  auto ky = mod_k2(dm, 1, ny, dm.lyt - dm.lyb, dm.h[1]);
  auto kz = mod_k2(dm, 2, nz, dm.lzz, dm.h[2]);
  const double norm = double(nx) * double(ny) * double(nz);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        std::complex<double>& v = a[((size_t)k * ny + j) * nx + i];
        v = v / double(nx) / double(ny) / double(nz);
        double kk = kx[i] + ky[j] + kz[k];
        if (kk < 1.0e-16) v = 0.0;
        else v = std::complex<double>(v.real() / (-kk), v.imag() / (-kk));
      }
  (void)norm;
  for (int ax = 0; ax < 3; ++ax) cdft_axis(a, n3, ax, +1);
  for (size_t n = 0; n < rhs.size(); ++n) rhs[n] = a[n].real();
}

// ---------------------------------------------------------------------------
// poisson_010: x and z periodic, y non-periodic (poisson_1stderivcomp.f90:1457-1816)
// ---------------------------------------------------------------------------
// waves() for bcy = 1 (poisson_1stderivcomp.f90:2484-2501): yky = nym*wp (stretched, in eta) and
// yk2 = (nym*wp/yly)^2 at w = pi*(j-1)/nym, j = 1..ny
static void waves_y_neumann(const Domain& dm, std::vector<double>& yky, std::vector<double>& yk2) {
  const Family& c2p = dm.T.fam[FAM_D1C2P];
  const int m = dm.iacc - 1;
  const int ny = dm.nc[1], nym = dm.nc[1];
  const double dy = dm.h[1], yly = dm.lyt - dm.lyb;
  const double alc = c2p.f[2][0][BC_PERIODIC][m];
  const double ac = c2p.r[2][0][BC_PERIODIC][m] / dy;
  const double bc = c2p.r[2][1][BC_PERIODIC][m] / dy;
  yky.assign(ny, 0.0);
  yk2.assign(ny, 0.0);
  for (int j = 1; j <= ny; ++j) {
    const double w = 2.0 * PI * 0.5 * double(j - 1) / double(nym);
    double wp = ac * 2.0 * dy * std::sin(w * 0.5) + (bc * 2.0 * dy) * std::sin(3.0 * 0.5 * w);
    wp = wp / (1.0 + 2.0 * alc * std::cos(w));
    yky[j - 1] = dm.stretch_y ? double(nym) * wp : double(nym) * wp / yly;
    const double q = double(nym) * wp / yly;
    yk2[j - 1] = q * q;
  }
  yky[0] = 0.0;
  yk2[0] = 0.0;
}

// The pentadiagonal systems of matrice_refinement (poisson_1stderivcomp.f90:2718-3039, istret 1
// or 2, with the compact-interpolation transfer factors switched off (ftr = .false.) so they are
// 1): for the odd (sys 0, a) and even (sys 1, a2) cosine modes, row r = 0..ny/2-1, the five
// diagonals c[0..4] = a(.,.,.,1..5) at the main-diagonal shift s = xk2 + zk2.
struct Penta {
  int h;
  double xa0, xa1;
  std::vector<double> c[2];  // cw22 = yky(2j-1) and cw2 = yky(2j), j = 1..h
  void init(const Domain& dm, const std::vector<double>& yky) {
    h = dm.nc[1] / 2;
    const double beta = dm.rstret;
    const double alpha = (-1.0 + std::sqrt(1.0 + 4.0 * PI * PI * beta * beta)) / beta * 0.5;
    xa0 = alpha / PI + 0.5 / beta / PI;
    xa1 = dm.istret == 1 ? +1.0 / 4.0 / beta / PI : -1.0 / 4.0 / beta / PI;
    const double yly = dm.lyt - dm.lyb;
    xa0 = xa0 / yly;
    xa1 = xa1 / yly;
    for (int s = 0; s < 2; ++s) {
      c[s].assign(h + 1, 0.0);  // 1-based
      for (int j = 1; j <= h; ++j) c[s][j] = yky[2 * j - 2 + s];
    }
  }
  // row j (1-based) of system s into d[1..5]
  void row(int s, int j, double sxz, bool pin, double d[6]) const {
    const std::vector<double>& w = c[s];
    const double xa0_2 = xa0 * xa0, xa1_2 = xa1 * xa1, xa01 = xa0 * xa1, xa0p1_2 = (xa0 + xa1) * (xa0 + xa1);
    for (int q = 0; q < 6; ++q) d[q] = 0.0;
    // main diagonal (:2846-2926)
    if (j >= 2 && j <= h - 1) d[3] = -(sxz + xa0_2 * (w[j] * w[j]) + xa1_2 * w[j] * (w[j - 1] + w[j + 1]));
    else if (j == 1) {
      if (s == 0) d[3] = -(sxz + xa0_2 * (w[1] * w[1]) + xa1_2 * w[1] * w[2]);
      else d[3] = -(sxz + (xa0_2 - xa1_2) * (w[1] * w[1]) + xa1_2 * w[1] * w[2]);
    } else {
      if (s == 0) d[3] = -(sxz + xa0_2 * (w[h] * w[h]) + xa1_2 * w[h] * w[h - 1]);
      else d[3] = -(sxz + xa0p1_2 * (w[h] * w[h]) + xa1_2 * w[h] * w[h - 1]);
    }
    // super-diagonal +1 (:2930-2975)
    if (j >= 2 && j <= h - 1) d[4] = xa01 * (w[j + 1] * (w[j] + w[j + 1]));
    if (j == 1) {
      if (s == 0) d[4] = 2.0 * xa01 * (w[1] * w[2] + w[2] * w[2]);
      else d[4] = (xa0 - xa1) * xa1 * (w[1] * w[2]) + xa0 * xa1 * (w[2] * w[2]);
    }
    if (s == 1 && j == h - 1) d[4] = xa0 * xa1 * w[h - 1] * w[h] + (xa0 + xa1) * xa1 * (w[h] * w[h]);
    if (s == 1 && j == h) d[4] = 0.0;
    // super-diagonal +2 (:2977-2997)
    if (j <= h - 2) d[5] = xa1_2 * (-(w[j + 1] * w[j + 2]));
    if (s == 0 && j == 1) d[5] = 2.0 * d[5];
    // sub-diagonal -1 (:2999-3023)
    if (j >= 2) d[2] = xa01 * (w[j - 1] * (w[j] + w[j - 1]));
    if (s == 1 && j == 2) d[2] = xa0 * xa1 * (w[2] * w[1]) + (xa0 + xa1) * xa1 * (w[1] * w[1]);
    if (s == 1 && j == h) d[2] = (xa0 + xa1) * xa1 * (w[h] * w[h - 1]) + xa0 * xa1 * (w[h - 1] * w[h - 1]);
    // sub-diagonal -2 (:3025-3036)
    if (j >= 3) d[1] = xa1_2 * (-(w[j - 1] * w[j - 2]));
    // the zero mode is pinned (:3038-3046)
    if (pin && s == 0 && j == 1) { d[3] = 1.0; d[4] = 0.0; d[5] = 0.0; }
  }
};

// inversion5_v1 (poisson_1stderivcomp.f90:420-561) for one real system (rows 1..h, diagonals
// a[j][1..5]) and right-hand side e[1..h]; eps = 1e-16 (DOUBLE_PREC).  The real and imaginary
// parts of the reference share the same real matrix, so one call handles one part.
static void inversion5(std::vector<std::array<double, 6>> a, std::vector<double>& e, int h) {
  const double eps = 1.0e-16;
  double tmp = 0.0;  // a zero pivot keeps the previous multiplier, as the reference does
  for (int m = 1; m <= h - 2; ++m) {
    for (int i = 1; i <= 2; ++i) {
      const int mi = m + i;
      if (a[m][3] != 0.0) tmp = a[mi][3 - i] / a[m][3];
      e[mi] = e[mi] - tmp * e[m];
      for (int jc = 4 - i; jc <= 5 - i; ++jc) a[mi][jc] = a[mi][jc] - tmp * a[m][jc + i];
    }
  }
  double t1 = std::fabs(a[h - 1][3]) > eps ? a[h][2] / a[h - 1][3] : 0.0;
  const double sr = t1;
  double b1 = a[h][3] - t1 * a[h - 1][4];
  double t3;
  if (std::fabs(b1) > eps) {
    t1 = sr / b1;
    t3 = e[h] / b1 - t1 * e[h - 1];
  } else {
    t1 = 0.0;
    t3 = 0.0;
  }
  e[h] = t3;
  b1 = std::fabs(a[h - 1][3]) > eps ? 1.0 / a[h - 1][3] : 0.0;
  double a1 = a[h - 1][4] * b1;
  e[h - 1] = e[h - 1] * b1 - a1 * e[h];
  for (int i = h - 2; i >= 1; --i) {
    const double s = std::fabs(a[i][3]) > eps ? 1.0 / a[i][3] : 0.0;
    a1 = a[i][4] * s;
    const double bb = a[i][5] * s;
    e[i] = e[i] * s - a1 * e[i + 1] - bb * e[i + 2];
  }
}

// poisson_010.  The reference's real-to-complex 3D FFT (z halved) is taken here as the full
// complex DFT of the real data; the forward and backward x and z half-cell phase factors
// (:1527-1553, :1740-1767) multiply each (kx, kz) column by e^{-i theta} and e^{+i theta} around
// a y stage that applies one real operator to both real and imaginary parts, so they cancel and
// are left out, as in poisson_000 above.
static void poisson_010(const Domain& dm, std::vector<double>& rhs) {
  const int nx = dm.nc[0], ny = dm.nc[1], nz = dm.nc[2];
  if (ny % 2 || ny < 8) throw std::runtime_error("poisson_010 needs an even ny >= 8");
  if (dm.stretch_y && dm.istret != 1 && dm.istret != 2) throw std::runtime_error("poisson_010: istret 1 or 2");
  const int n3[3] = {nx, ny, nz};
  auto at = [&](int i, int j, int k) { return ((size_t)k * ny + j) * nx + i; };
  // even/odd reordering in y (:1491-1501)
  std::vector<std::complex<double>> a(rhs.size());
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i) {
      for (int j = 1; j <= ny / 2; ++j) a[at(i, j - 1, k)] = rhs[at(i, 2 * (j - 1), k)];
      for (int j = ny / 2 + 1; j <= ny; ++j) a[at(i, j - 1, k)] = rhs[at(i, 2 * ny - 2 * j + 1, k)];
    }
  for (int ax = 0; ax < 3; ++ax) cdft_axis(a, n3, ax, -1);
  for (auto& v : a) v = v / double(nx) / double(ny) / double(nz);
  std::vector<double> ay(ny), by(ny);  // abxyz, bcy = 1 (:2376-2382)
  for (int j = 1; j <= ny; ++j) {
    ay[j - 1] = std::sin(double(j - 1) * PI * 0.5 / double(ny));
    by[j - 1] = std::cos(double(j - 1) * PI * 0.5 / double(ny));
  }
  auto kx = mod_k2(dm, 0, nx, dm.lxx, dm.h[0]);
  auto kz = mod_k2(dm, 2, nz, dm.lzz, dm.h[2]);
  std::vector<double> yky, yk2;
  waves_y_neumann(dm, yky, yk2);
  Penta P;
  if (dm.stretch_y) P.init(dm, yky);
  const int h = ny / 2;
#pragma omp parallel for collapse(2)
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i) {
      std::vector<std::complex<double>> c(ny), b(ny);
      for (int j = 0; j < ny; ++j) c[j] = a[at(i, j, k)];
      // forward post-processing in y (:1557-1575)
      b[0] = c[0];
      for (int j = 2; j <= ny; ++j) {
        const double t1 = c[j - 1].real(), t2 = c[j - 1].imag();
        const double t3 = c[ny - j + 1].real(), t4 = c[ny - j + 1].imag();
        const double yb = by[j - 1], ya = ay[j - 1];
        const double xx1 = t1 * yb, xx2 = t1 * ya, xx3 = t2 * yb, xx4 = t2 * ya;
        const double xx5 = t3 * yb, xx6 = t3 * ya, xx7 = t4 * yb, xx8 = t4 * ya;
        b[j - 1] = 0.5 * std::complex<double>(xx1 + xx4 + xx5 - xx8, -xx2 + xx3 + xx6 + xx7);
      }
      if (!dm.stretch_y) {
        // wavenumber division (:1591-1613), kxyz = xk2 + yk2 + zk2 with equal parts
        for (int j = 0; j < ny; ++j) {
          const double kk = kx[i] + yk2[j] + kz[k];
          if (std::fabs(kk) < 1.0e-16) b[j] = 0.0;
          else b[j] = std::complex<double>(b[j].real() / (-kk), b[j].imag() / (-kk));
        }
      } else {
        // odd and even modes (:1650-1675), inversion5_v1 on each
        const bool pin = kx[i] == 0.0 && kz[k] == 0.0;
        const double sxz = kx[i] + kz[k];
        for (int s = 0; s < 2; ++s) {
          std::vector<std::array<double, 6>> mat(h + 1);
          std::vector<double> er(h + 1), ei(h + 1);
          for (int j = 1; j <= h; ++j) {
            double d[6];
            P.row(s, j, sxz, pin, d);
            for (int q = 0; q < 6; ++q) mat[j][q] = d[q];
            er[j] = b[2 * j - 2 + s].real();
            ei[j] = b[2 * j - 2 + s].imag();
          }
          inversion5(mat, er, h);
          inversion5(mat, ei, h);
          for (int j = 1; j <= h; ++j) b[2 * j - 2 + s] = std::complex<double>(er[j], ei[j]);
        }
      }
      // backward post-processing in y (:1717-1735)
      c[0] = b[0];
      for (int j = 2; j <= ny; ++j) {
        const double t1 = b[j - 1].real(), t2 = b[j - 1].imag();
        const double t3 = b[ny - j + 1].real(), t4 = b[ny - j + 1].imag();
        const double yb = by[j - 1], ya = ay[j - 1];
        const double xx1 = t1 * yb, xx2 = t1 * ya, xx3 = t2 * yb, xx4 = t2 * ya;
        const double xx5 = t3 * yb, xx6 = t3 * ya, xx7 = t4 * yb, xx8 = t4 * ya;
        c[j - 1] = std::complex<double>(xx1 - xx4 + xx6 + xx7, -(-xx2 - xx3 + xx5 - xx8));
      }
      for (int j = 0; j < ny; ++j) a[at(i, j, k)] = c[j];
    }
  for (int ax = 0; ax < 3; ++ax) cdft_axis(a, n3, ax, +1);
  // undo the reordering (:1772-1782)
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i) {
      for (int j = 1; j <= ny / 2; ++j) rhs[at(i, 2 * j - 2, k)] = a[at(i, j - 1, k)].real();
      for (int j = 1; j <= ny / 2; ++j) rhs[at(i, 2 * j - 1, k)] = a[at(i, ny - j, k)].real();
    }
}

static void poisson_dispatch(const Domain& dm, std::vector<double>& rhs) {
  // solve_fft_poisson (poisson_interface.f90:119-149) and the poisson_000 / poisson_010 choice of
  // decomp_2d_poisson_init (poisson_1stderivcomp.f90:794-820)
  if (dm.ifft == 2) poisson_fishpack(dm, rhs);
  else if (dm.periodic[1]) poisson_3dfft(dm, rhs);
  else poisson_010(dm, rhs);
}

// Get_divergence_flow (eq_continuity.f90:91-161)
static Arr divergence(const Domain& dm, const std::vector<double>& ux, const std::vector<double>& uy,
                      const std::vector<double>& uz) {
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2];
  Arr qx(dm.np[0], nc1, nc2), qy(nc0, dm.np[1], nc2), qz(nc0, nc1, dm.np[2]);
  qx.v = ux; qy.v = uy; qz.v = uz;
  std::vector<double> fbcx_any((size_t)4 * nc1 * nc2, MAXP);
  Arr a = op(dm, 0, FAM_D1P2C, dm.ibcx[V_QX], &fbcx_any, qx);
  Arr b = op(dm, 1, FAM_D1P2C, dm.ibcy[V_QY], nullptr, qy);
  Arr c = op(dm, 2, FAM_D1P2C, dm.ibcz[V_QZ], nullptr, qz);
  Arr div(nc0, nc1, nc2);
  for (size_t n = 0; n < div.size(); ++n) div.v[n] = ((0.0 + a.v[n]) + b.v[n]) + c.v[n];
  return div;
}
static Arr divergence(const Domain& dm, const Flow& fl) {
  return fl.thermo ? divergence(dm, fl.th.gx, fl.th.gy, fl.th.gz) : divergence(dm, fl.qx, fl.qy, fl.qz);
}

static void enforce_velo(const Domain& dm, Flow& fl) {
  // enforce_velo_from_fbc (bc_dirichlet.f90:461-516); x/z periodic so only the y walls act
  const int nc0 = dm.nc[0], np1 = dm.np[1], nc2 = dm.nc[2];
  for (int side = 0; side < 2; ++side) {
    if (dm.ibcy[V_QY][side] != BC_DIRICHLET) continue;
    int j = side == 0 ? 0 : np1 - 1;
    for (int k = 0; k < nc2; ++k)
      for (int i = 0; i < nc0; ++i) {
        const size_t c = ((size_t)k * np1 + j) * nc0 + i;
        if (fl.thermo) fl.th.gy[c] = dm.fbcy_const[V_QY][side] * fl.th.fbcy_ftp[((size_t)k * 4 + side) * nc0 + i].d;
        else fl.qy[c] = dm.fbcy_const[V_QY][side];
      }
  }
}

void convert_q_g(const Domain& dm, Flow& fl, bool to_q);

// Solve_momentum_eq (eq_momentum2.f90:1799-1932), flow-only Cartesian
void momentum_substep(Domain& dm, Flow& fl, int isub, double* bulk_out) {
  Rhs3 r;
  momentum_rhs(dm, fl, r);
  fractional_step(dm, isub, fl.mx_rhs0, r.mx.v, r.px.v);
  fractional_step(dm, isub, fl.my_rhs0, r.my.v, r.py.v);
  fractional_step(dm, isub, fl.mz_rhs0, r.mz.v, r.pz.v);
  double bulk = 0.0;
  if (dm.idriven == 1) {
    bulk = vol_average(dm, r.mx);
    for (auto& v : r.mx.v) v = v - bulk;
  }
  if (bulk_out) *bulk_out = bulk;
  // the advanced variable: momentum g for variable properties, velocity q otherwise
  std::vector<double>& ux = fl.thermo ? fl.th.gx : fl.qx;
  std::vector<double>& uy = fl.thermo ? fl.th.gy : fl.qy;
  std::vector<double>& uz = fl.thermo ? fl.th.gz : fl.qz;
  for (size_t n = 0; n < ux.size(); ++n) ux[n] = ux[n] + r.mx.v[n];
  for (size_t n = 0; n < uy.size(); ++n) uy[n] = uy[n] + r.my.v[n];
  for (size_t n = 0; n < uz.size(); ++n) uz[n] = uz[n] + r.mz.v[n];
  enforce_velo(dm, fl);
  // solve_poisson (eq_momentum2.f90:1663-1718)
  Arr div = divergence(dm, fl);
  std::vector<double> pcor(div.size(), 0.0);
  for (size_t n = 0; n < pcor.size(); ++n) pcor[n] = pcor[n] + div.v[n];
  const double coeff = 1.0 / (dm.tAlpha[isub] * dm.sigma2p * dm.dt);
  for (auto& v : pcor) v = v * coeff;
  poisson_dispatch(dm, pcor);
  for (size_t n = 0; n < fl.pres.size(); ++n) fl.pres[n] = fl.pres[n] + pcor[n];
  fl.pcor = pcor;
  // Correct_massflux (eq_momentum2.f90:1577-1660)
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2];
  Arr phi(nc0, nc1, nc2);
  phi.v = pcor;
  std::vector<double> fbcx_any((size_t)4 * nc1 * nc2, MAXP), fbcz_any((size_t)nc0 * nc1 * 4, MAXP);
  const auto fbcy_pr = fbcy_const_plane(nc0, nc2, dm.fbcy_const[V_PR][0], dm.fbcy_const[V_PR][1]);
  Arr dpx = op(dm, 0, FAM_D1C2P, dm.ibcx[V_PR], &fbcx_any, phi);
  Arr dpy = op(dm, 1, FAM_D1C2P, dm.ibcy[V_PR], &fbcy_pr, phi);
  Arr dpz = op(dm, 2, FAM_D1C2P, dm.ibcz[V_PR], &fbcz_any, phi);
  const double f = dm.dt * dm.tAlpha[isub] * dm.sigma2p;
  for (size_t n = 0; n < ux.size(); ++n) ux[n] = ux[n] - f * dpx.v[n];
  for (size_t n = 0; n < uy.size(); ++n) uy[n] = uy[n] - f * dpy.v[n];
  for (size_t n = 0; n < uz.size(); ++n) uz[n] = uz[n] - f * dpz.v[n];
  enforce_velo(dm, fl);
  // Calculate_drhodt (src/eq_continuity.f90:26-78) adds (rho - rho_m1)/dt to the Poisson RHS,
  // but Update_thermal_properties has already set rho_m1 = rho, so that term is zero and is
  // left out here.
  if (fl.thermo) convert_q_g(dm, fl, true);
}

// ---------------------------------------------------------------------------
// Thermal property lookup (src/input_thermo.f90:345-446)
// ---------------------------------------------------------------------------
static const double MINP = 1.0e-20;  // src/modules.f90:141

// bisection on a monotonic table column (the sign test of the reference: i1 moves while
// (col[i1]-x)*(col[im]-x) > MINP), then linear weights
static void bracket(const std::vector<double>& col, double x, int& i1, int& i2, double& w1) {
  i1 = 0;
  i2 = (int)col.size() - 1;
  while (i2 - i1 > 1) {
    const int im = i1 + (i2 - i1) / 2;
    const double d1 = col[i1] - x, dmid = col[im] - x;
    if (d1 * dmid > MINP) i1 = im;
    else i2 = im;
  }
  w1 = (col[i2] - x) / (col[i2] - col[i1]);
}

void ftp_from_h(const ThermoTable& tb, Ftp& f) {
  int i1, i2;
  double w1;
  bracket(tb.h, f.h, i1, i2, w1);
  const double w2 = 1.0 - w1;
  f.d = w1 * tb.d[i1] + w2 * tb.d[i2];
  f.m = w1 * tb.m[i1] + w2 * tb.m[i2];
  f.k = w1 * tb.k[i1] + w2 * tb.k[i2];
  f.t = w1 * tb.t[i1] + w2 * tb.t[i2];
  f.b = w1 * tb.b[i1] + w2 * tb.b[i2];
  f.cp = w1 * tb.cp[i1] + w2 * tb.cp[i2];
}

void ftp_from_dh(const ThermoTable& tb, Ftp& f) {
  if (f.rhoh < tb.dhmin) f.rhoh = tb.dhmin;
  else if (f.rhoh > tb.dhmax) f.rhoh = tb.dhmax;
  int i1, i2;
  double w1;
  bracket(tb.rhoh, f.rhoh, i1, i2, w1);
  const double w2 = 1.0 - w1;
  f.h = w1 * tb.h[i1] + w2 * tb.h[i2];
  ftp_from_h(tb, f);
  f.h = f.rhoh / f.d;
  ftp_from_h(tb, f);
}

// ftp_refresh_thermal_properties_from_T_undim (src/input_thermo.f90:272-307): T -> all
void ftp_from_t(const ThermoTable& tb, Ftp& f) {
  int i1, i2;
  double w1;
  bracket(tb.t, f.t, i1, i2, w1);
  const double w2 = 1.0 - w1;
  f.d = w1 * tb.d[i1] + w2 * tb.d[i2];
  f.m = w1 * tb.m[i1] + w2 * tb.m[i2];
  f.k = w1 * tb.k[i1] + w2 * tb.k[i2];
  f.h = w1 * tb.h[i1] + w2 * tb.h[i2];
  f.b = w1 * tb.b[i1] + w2 * tb.b[i2];
  f.cp = w1 * tb.cp[i1] + w2 * tb.cp[i2];
  f.rhoh = f.d * f.h;
}

// Update_thermal_properties (src/eq_energy.f90:14-146), y walls only (x and z are periodic).
// The top wall takes row np(2) of the interpolated rho*h (the reference indexes np(1) there).
static void update_thermal_properties(const Domain& dm, Thermo& th) {
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2], np1 = dm.np[1];
  const size_t n = (size_t)nc0 * nc1 * nc2;
#pragma omp parallel for schedule(static)
  for (long long c = 0; c < (long long)n; ++c) {
    Ftp f{};
    f.rhoh = th.rhoh[c];
    ftp_from_dh(th.tab, f);
    th.hEnth[c] = f.h;
    th.tTemp[c] = f.t;
    th.kCond[c] = f.k;
    th.dDens[c] = f.d;
    th.mVisc[c] = f.m;
  }
  if (dm.ibcy[V_TM][0] == BC_NEUMANN || dm.ibcy[V_TM][1] == BC_NEUMANN) {
    Arr dh(nc0, nc1, nc2);
    dh.v = th.rhoh;
    Arr dh_cpc = op(dm, 1, FAM_M1C2P, dm.ibcy_ftp, nullptr, dh);
    for (int side = 0; side < 2; ++side) {
      if (dm.ibcy[V_TM][side] != BC_NEUMANN) continue;
      const int j = side == 0 ? 0 : np1 - 1;
      for (int k = 0; k < nc2; ++k)
        for (int i = 0; i < nc0; ++i) {
          Ftp f{};
          f.rhoh = dh_cpc.at(i, j, k);
          ftp_from_dh(th.tab, f);
          th.fbcy_ftp[((size_t)k * 4 + side) * nc0 + i] = f;
          th.fbcy_ftp[((size_t)k * 4 + side + 2) * nc0 + i] = f;
        }
    }
  }
}

static std::vector<double> fbcy_prop(const Thermo& th, double Ftp::*field) {
  std::vector<double> v(th.fbcy_ftp.size());
  for (size_t n = 0; n < v.size(); ++n) v[n] = th.fbcy_ftp[n].*field;
  return v;
}

// Compute_energy_rhs + Calculate_energy_fractional_step (src/eq_energy.f90:148-401).  The y
// diffusion boundary value is taken from the wall rows of kappa*dT/dy (the reference tests the
// x-velocity flag there and passes MAXP for an x-periodic channel).
static void energy_rhs(const Domain& dm, Flow& fl, int isub, std::vector<double>& rhs) {
  Thermo& th = fl.th;
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2];
  const int np0 = dm.np[0], np1 = dm.np[1], np2 = dm.np[2];
  int ftpx[2] = {BC_PERIODIC, BC_PERIODIC}, ftpz[2] = {BC_PERIODIC, BC_PERIODIC};
  int ebcx_conv[2], ebcy_conv[2], ebcz_conv[2], ebcx_difu[2], ebcy_difu[2], ebcz_difu[2];
  prod_of(dm.ibcx[V_QX], ftpx, ebcx_conv);
  prod_of(dm.ibcy[V_QY], dm.ibcy_ftp, ebcy_conv);
  prod_of(dm.ibcz[V_QZ], ftpz, ebcz_conv);
  tau_of(dm.ibcx[V_TM], ftpx, ebcx_difu);
  tau_of(dm.ibcy[V_TM], dm.ibcy_ftp, ebcy_difu);
  tau_of(dm.ibcz[V_TM], ftpz, ebcz_difu);
  Arr h(nc0, nc1, nc2), kc(nc0, nc1, nc2), T(nc0, nc1, nc2);
  h.v = th.hEnth; kc.v = th.kCond; T.v = th.tTemp;
  Arr gx(np0, nc1, nc2), gy(nc0, np1, nc2), gz(nc0, nc1, np2);
  gx.v = th.gx; gy.v = th.gy; gz.v = th.gz;
  std::vector<double> fbcx_any((size_t)4 * nc1 * nc2, MAXP), fbcz_any((size_t)nc0 * nc1 * 4, MAXP);
  const auto fh = fbcy_prop(th, &Ftp::h), fk = fbcy_prop(th, &Ftp::k);
  Arr h_pcc = op(dm, 0, FAM_M1C2P, ftpx, &fbcx_any, h);
  Arr h_cpc = op(dm, 1, FAM_M1C2P, dm.ibcy_ftp, &fh, h);
  Arr h_ccp = op(dm, 2, FAM_M1C2P, ftpz, &fbcz_any, h);
  Arr k_pcc = op(dm, 0, FAM_M1C2P, ftpx, &fbcx_any, kc);
  Arr k_cpc = op(dm, 1, FAM_M1C2P, dm.ibcy_ftp, &fk, kc);
  Arr k_ccp = op(dm, 2, FAM_M1C2P, ftpz, &fbcz_any, kc);
  const size_t n = (size_t)nc0 * nc1 * nc2;
  std::vector<double> ex(n, 0.0), ey(n, 0.0), ez(n, 0.0);
  {  // conv-x
    Arr a(np0, nc1, nc2);
    for (size_t m = 0; m < a.size(); ++m) a.v[m] = -gx.v[m] * h_pcc.v[m];
    Arr r = op(dm, 0, FAM_D1P2C, ebcx_conv, nullptr, a);
    for (size_t m = 0; m < n; ++m) ex[m] = ex[m] + r.v[m];
  }
  {  // conv-y
    Arr a(nc0, np1, nc2);
    for (size_t m = 0; m < a.size(); ++m) a.v[m] = -gy.v[m] * h_cpc.v[m];
    Arr r = op(dm, 1, FAM_D1P2C, ebcy_conv, nullptr, a);
    for (size_t m = 0; m < n; ++m) ey[m] = ey[m] + r.v[m];
  }
  {  // conv-z
    Arr a(nc0, nc1, np2);
    for (size_t m = 0; m < a.size(); ++m) a.v[m] = -gz.v[m] * h_ccp.v[m];
    Arr r = op(dm, 2, FAM_D1P2C, ebcz_conv, nullptr, a);
    for (size_t m = 0; m < n; ++m) ez[m] = ez[m] + r.v[m];
  }
  const double rpr = th.rPrRen;
  {  // diff-x (get_fbcx_iTh gives zeros for periodic x; no velocity walls in x: MAXP)
    std::vector<double> f0((size_t)4 * nc1 * nc2, 0.0);
    Arr d = op(dm, 0, FAM_D1C2P, dm.ibcx[V_TM], &f0, T);
    for (size_t m = 0; m < d.size(); ++m) d.v[m] = d.v[m] * k_pcc.v[m];
    Arr r = op(dm, 0, FAM_D1P2C, ebcx_difu, &fbcx_any, d);
    for (size_t m = 0; m < n; ++m) ex[m] = ex[m] + r.v[m] * rpr;
  }
  {  // diff-y: get_fbcy_iTh: planes 1, 2 = q_w for Neumann sides (T values for Dirichlet), 3, 4 = 0
    std::vector<double> f((size_t)nc0 * 4 * nc2, 0.0);
    for (int k = 0; k < nc2; ++k)
      for (int side = 0; side < 2; ++side)
        for (int i = 0; i < nc0; ++i) {
          double v = 0.0;
          if (dm.ibcy[V_TM][side] == BC_NEUMANN) v = th.qw[side];
          else if (dm.ibcy[V_TM][side] == BC_DIRICHLET) v = th.fbcy_ftp[((size_t)k * 4 + side) * nc0 + i].t;
          f[((size_t)k * 4 + side) * nc0 + i] = v;
        }
    Arr d = op(dm, 1, FAM_D1C2P, dm.ibcy[V_TM], &f, T);
    for (size_t m = 0; m < d.size(); ++m) d.v[m] = d.v[m] * k_cpc.v[m];
    const auto fw = extract_fbcy(d);
    Arr r = op(dm, 1, FAM_D1P2C, ebcy_difu, &fw, d);
    for (size_t m = 0; m < n; ++m) ey[m] = ey[m] + r.v[m] * rpr;
  }
  {  // diff-z
    std::vector<double> f0((size_t)nc0 * nc1 * 4, 0.0);
    Arr d = op(dm, 2, FAM_D1C2P, dm.ibcz[V_TM], &f0, T);
    for (size_t m = 0; m < d.size(); ++m) d.v[m] = d.v[m] * k_ccp.v[m];
    Arr r = op(dm, 2, FAM_D1P2C, ebcz_difu, nullptr, d);
    for (size_t m = 0; m < n; ++m) ez[m] = ez[m] + r.v[m] * rpr;
  }
  rhs.assign(n, 0.0);
  for (size_t m = 0; m < n; ++m) rhs[m] = ex[m] + (ey[m] + ez[m]);
  // Calculate_energy_fractional_step (:148-177)
  for (size_t m = 0; m < n; ++m) {
    const double cur = rhs[m], last = th.ene_rhs0[m];
    const double tot = dm.tGamma[isub] * cur + dm.tZeta[isub] * last;
    th.ene_rhs0[m] = cur;
    rhs[m] = dm.dt * tot;
  }
}

// Solve_energy_eq (src/eq_energy.f90:405-458)
void energy_substep(Domain& dm, Flow& fl, int isub) {
  std::vector<double> rhs;
  energy_rhs(dm, fl, isub, rhs);
  for (size_t m = 0; m < rhs.size(); ++m) fl.th.rhoh[m] = fl.th.rhoh[m] + rhs[m];
  update_thermal_properties(dm, fl.th);
}

// convert_primary_conservative (src/para_conversion.f90:5-227): q = g / rho_face (g2q) or
// g = q * rho_face (q2g); the wall values of g and q are zero for the no-slip channel
void convert_q_g(const Domain& dm, Flow& fl, bool to_q) {
  Thermo& th = fl.th;
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2];
  Arr d(nc0, nc1, nc2);
  d.v = th.dDens;
  std::vector<double> fbcx_any((size_t)4 * nc1 * nc2, MAXP), fbcz_any((size_t)nc0 * nc1 * 4, MAXP);
  const int per[2] = {BC_PERIODIC, BC_PERIODIC};
  const auto fd = fbcy_prop(th, &Ftp::d);
  Arr dx = op(dm, 0, FAM_M1C2P, per, &fbcx_any, d);
  Arr dy = op(dm, 1, FAM_M1C2P, dm.ibcy_ftp, &fd, d);
  Arr dz = op(dm, 2, FAM_M1C2P, per, &fbcz_any, d);
  if (to_q) {
    for (size_t m = 0; m < fl.qx.size(); ++m) fl.qx[m] = th.gx[m] / dx.v[m];
    for (size_t m = 0; m < fl.qy.size(); ++m) fl.qy[m] = th.gy[m] / dy.v[m];
    for (size_t m = 0; m < fl.qz.size(); ++m) fl.qz[m] = th.gz[m] / dz.v[m];
  } else {
    for (size_t m = 0; m < fl.qx.size(); ++m) th.gx[m] = fl.qx[m] * dx.v[m];
    for (size_t m = 0; m < fl.qy.size(); ++m) th.gy[m] = fl.qy[m] * dy.v[m];
    for (size_t m = 0; m < fl.qz.size(); ++m) th.gz[m] = fl.qz[m] * dz.v[m];
  }
}

// bulk kinetic energy (io_monitor.f90:209-241)
double bulk_ke(const Domain& dm, const Flow& fl) {
  const int nc0 = dm.nc[0], nc1 = dm.nc[1], nc2 = dm.nc[2];
  Arr qx(dm.np[0], nc1, nc2), qy(nc0, dm.np[1], nc2), qz(nc0, nc1, dm.np[2]);
  qx.v = fl.qx; qy.v = fl.qy; qz.v = fl.qz;
  std::vector<double> fbcx_any((size_t)4 * nc1 * nc2, MAXP), fbcz_any((size_t)nc0 * nc1 * 4, MAXP);
  const auto fbcy_qy = fbcy_const_plane(nc0, nc2, dm.fbcy_const[V_QY][0], dm.fbcy_const[V_QY][1]);
  Arr u = op(dm, 0, FAM_M1P2C, dm.ibcx[V_QX], &fbcx_any, qx);
  Arr v = op(dm, 1, FAM_M1P2C, dm.ibcy[V_QY], &fbcy_qy, qy);
  Arr w = op(dm, 2, FAM_M1P2C, dm.ibcz[V_QZ], &fbcz_any, qz);
  Arr e(nc0, nc1, nc2);
  for (size_t n = 0; n < e.size(); ++n) e.v[n] = 0.5 * (u.v[n] * u.v[n] + v.v[n] * v.v[n] + w.v[n] * w.v[n]);
  return vol_average(dm, e);
}

}  // namespace orc

// ===========================================================================
// C API used by tests through ctypes
// ===========================================================================
using namespace orc;

struct OrcHandle {
  Domain dm;
  Flow fl;
};

extern "C" {

// TDMA known-answer entry (restates Test_TDMA_noncyclic / Test_TDMA_cyclic): r in, x out
int orc_tdma(int cyclic, const double* a, const double* b, const double* c_in, double* r, int n) {
  std::vector<double> c(c_in, c_in + n), d(n, 0.0);
  if (cyclic) tdma_preprocess(a, b, c.data(), d.data(), n - 1);
  else tdma_preprocess(a, b, c.data(), d.data(), n);
  tdma_solve(cyclic != 0, r, a, b, c.data(), d.data(), n);
  return 0;
}

// params: ints[16] = {nc0,nc1,nc2, iacc, istret, idriven, ifft, periodic_y}
//         dbl[16]  = {lxx, lyt, lyb, lzz, rstret, dt, ren}
//         nominal bc codes nom[3][5][2] (x,y,z; qx,qy,qz,pr,Tm; side), fbcy const [5][2]
void* orc_create(const int* ints, const double* dbl, const int* nom, const double* fbcy_const) {
  try {
    OrcHandle* h = new OrcHandle();
    Domain& dm = h->dm;
    dm.nc[0] = ints[0]; dm.nc[1] = ints[1]; dm.nc[2] = ints[2];
    dm.iacc = ints[3];
    dm.istret = ints[4];
    dm.idriven = ints[5];
    dm.ifft = ints[6];
    dm.periodic[0] = true;
    dm.periodic[1] = ints[7] != 0;
    dm.periodic[2] = true;
    dm.stretch_y = dm.istret != 0;
    dm.lxx = dbl[0]; dm.lyt = dbl[1]; dm.lyb = dbl[2]; dm.lzz = dbl[3];
    dm.rstret = dbl[4]; dm.dt = dbl[5];
    dm.rre = 1.0 / dbl[6];
    int nm[3][5][2];
    std::memcpy(nm, nom, sizeof(nm));
    for (int v = 0; v < 5; ++v)
      for (int s = 0; s < 2; ++s) dm.fbcy_const[v][s] = fbcy_const[v * 2 + s];
    build_tables(dm.T);
    build_geometry(dm);
    configure_bcs(dm, nm);
    dm.sigma2p = 1.0;
    dm.tGamma[0] = 1.0; dm.tGamma[1] = 8.0 / 15.0; dm.tGamma[2] = 5.0 / 12.0; dm.tGamma[3] = 3.0 * 0.25;
    dm.tZeta[0] = 0.0; dm.tZeta[1] = 0.0; dm.tZeta[2] = -17.0 / 60.0; dm.tZeta[3] = -5.0 / 12.0;
    for (int i = 0; i < 4; ++i) dm.tAlpha[i] = dm.tGamma[i] + dm.tZeta[i];
    if (dm.ifft == 2) fishpack_init(dm);
    Flow& fl = h->fl;
    const size_t npcc = (size_t)dm.np[0] * dm.nc[1] * dm.nc[2];
    const size_t ncpc = (size_t)dm.nc[0] * dm.np[1] * dm.nc[2];
    const size_t nccp = (size_t)dm.nc[0] * dm.nc[1] * dm.np[2];
    const size_t nccc = (size_t)dm.nc[0] * dm.nc[1] * dm.nc[2];
    fl.qx.assign(npcc, 0.0); fl.qy.assign(ncpc, 0.0); fl.qz.assign(nccp, 0.0);
    fl.pres.assign(nccc, 0.0); fl.pcor.assign(nccc, 0.0);
    fl.mx_rhs0.assign(npcc, 0.0); fl.my_rhs0.assign(ncpc, 0.0); fl.mz_rhs0.assign(nccp, 0.0);
    return h;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_create: %s\n", e.what());
    return nullptr;
  }
}

void orc_destroy(void* p) { delete static_cast<OrcHandle*>(p); }

// geometry out: yp(np_geo), yc(nc), mppt(np_geo), mpcc(nc); ints: np[3]; dbl: h[3]
void orc_geometry(void* p, double* yp, double* yc, double* mppt, double* mpcc, int* np, double* h) {
  auto* H = static_cast<OrcHandle*>(p);
  const Domain& dm = H->dm;
  std::memcpy(yp, dm.yp.data(), sizeof(double) * dm.yp.size());
  std::memcpy(yc, dm.yc.data(), sizeof(double) * dm.yc.size());
  std::memcpy(mppt, dm.mppt.data(), sizeof(double) * dm.mppt.size());
  std::memcpy(mpcc, dm.mpcc.data(), sizeof(double) * dm.mpcc.size());
  for (int d = 0; d < 3; ++d) { np[d] = dm.np[d]; h[d] = dm.h[d]; }
}

// calculated bcs out: ibc[3][5][2], mbc[18][2] in the order cov1 x,y,z, tau1 x,y,z, cov2..., tau3
void orc_bcs(void* p, int* ibc, int* mbc) {
  auto* H = static_cast<OrcHandle*>(p);
  const Domain& dm = H->dm;
  std::memcpy(ibc, dm.ibcx, sizeof(dm.ibcx));
  std::memcpy(ibc + 10, dm.ibcy, sizeof(dm.ibcy));
  std::memcpy(ibc + 20, dm.ibcz, sizeof(dm.ibcz));
  const int* all[18] = {dm.mbcx_cov1, dm.mbcy_cov1, dm.mbcz_cov1, dm.mbcx_tau1, dm.mbcy_tau1, dm.mbcz_tau1,
                        dm.mbcx_cov2, dm.mbcy_cov2, dm.mbcz_cov2, dm.mbcx_tau2, dm.mbcy_tau2, dm.mbcz_tau2,
                        dm.mbcx_cov3, dm.mbcy_cov3, dm.mbcz_cov3, dm.mbcx_tau3, dm.mbcy_tau3, dm.mbcz_tau3};
  for (int i = 0; i < 18; ++i) { mbc[2 * i] = all[i][0]; mbc[2 * i + 1] = all[i][1]; }
}

// one compact operator on a 3D array (x-fastest); fbc2d may be null
int orc_op3d(void* p, int dir, int fam, int ibc1, int ibc2, const double* fbc2d, const double* fi,
             const int* nin3, double* fo) {
  try {
    auto* H = static_cast<OrcHandle*>(p);
    int ibc[2] = {ibc1, ibc2};
    op3d(H->dm, dir, fam, ibc, fbc2d, fi, nin3, fo);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_op3d: %s\n", e.what());
    return 1;
  }
}

// one compact operator on a single line (for the analytic operator tests); fbc may be null
int orc_op1d(void* p, int dir, int fam, int ibc1, int ibc2, const double* fbc, const double* fi, double* fo) {
  auto* H = static_cast<OrcHandle*>(p);
  int ibc[2] = {ibc1, ibc2};
  op1d(H->dm, dir, fam, ibc, fbc, fi, fo);
  return 0;
}

void orc_set_fields(void* p, const double* qx, const double* qy, const double* qz, const double* pr) {
  auto* H = static_cast<OrcHandle*>(p);
  Flow& fl = H->fl;
  std::memcpy(fl.qx.data(), qx, sizeof(double) * fl.qx.size());
  std::memcpy(fl.qy.data(), qy, sizeof(double) * fl.qy.size());
  std::memcpy(fl.qz.data(), qz, sizeof(double) * fl.qz.size());
  std::memcpy(fl.pres.data(), pr, sizeof(double) * fl.pres.size());
}

void orc_get_fields(void* p, double* qx, double* qy, double* qz, double* pr, double* pcor) {
  auto* H = static_cast<OrcHandle*>(p);
  const Flow& fl = H->fl;
  if (qx) std::memcpy(qx, fl.qx.data(), sizeof(double) * fl.qx.size());
  if (qy) std::memcpy(qy, fl.qy.data(), sizeof(double) * fl.qy.size());
  if (qz) std::memcpy(qz, fl.qz.data(), sizeof(double) * fl.qz.size());
  if (pr) std::memcpy(pr, fl.pres.data(), sizeof(double) * fl.pres.size());
  if (pcor) std::memcpy(pcor, fl.pcor.data(), sizeof(double) * fl.pcor.size());
}

void orc_get_rhs0(void* p, double* mx, double* my, double* mz) {
  auto* H = static_cast<OrcHandle*>(p);
  const Flow& fl = H->fl;
  std::memcpy(mx, fl.mx_rhs0.data(), sizeof(double) * fl.mx_rhs0.size());
  std::memcpy(my, fl.my_rhs0.data(), sizeof(double) * fl.my_rhs0.size());
  std::memcpy(mz, fl.mz_rhs0.data(), sizeof(double) * fl.mz_rhs0.size());
}

// momentum RHS before the fractional step: conv+visc (mx,my,mz) and pressure gradients (px,py,pz)
int orc_momentum_rhs(void* p, double* mx, double* my, double* mz, double* px, double* py, double* pz) {
  try {
    auto* H = static_cast<OrcHandle*>(p);
    Rhs3 r;
    momentum_rhs(H->dm, H->fl, r);
    std::memcpy(mx, r.mx.v.data(), sizeof(double) * r.mx.size());
    std::memcpy(my, r.my.v.data(), sizeof(double) * r.my.size());
    std::memcpy(mz, r.mz.v.data(), sizeof(double) * r.mz.size());
    std::memcpy(px, r.px.v.data(), sizeof(double) * r.px.size());
    std::memcpy(py, r.py.v.data(), sizeof(double) * r.py.size());
    std::memcpy(pz, r.pz.v.data(), sizeof(double) * r.pz.size());
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_momentum_rhs: %s\n", e.what());
    return 1;
  }
}

int orc_momentum_substep(void* p, int isub, double* bulk) {
  try {
    auto* H = static_cast<OrcHandle*>(p);
    momentum_substep(H->dm, H->fl, isub, bulk);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_momentum_substep: %s\n", e.what());
    return 1;
  }
}

// Variable-property run: nondimensional table (sorted by T), 1/(Re Pr), wall heat fluxes and
// the initial temperature (initialise_thermal_properties, src/input_thermo.f90:1070-1103; the
// momentum g = rho q of the initial velocity, src/initialisation.f90:389).  Call after the
// velocity has been set.
int orc_thermo_init(void* p, int n, const double* t, const double* h, const double* d, const double* m,
                    const double* k, const double* cp, const double* b, double rPrRen, const double* qw,
                    double t_ini) {
  try {
    auto* H = static_cast<OrcHandle*>(p);
    Domain& dm = H->dm;
    Flow& fl = H->fl;
    Thermo& th = fl.th;
    ThermoTable& tb = th.tab;
    tb.t.assign(t, t + n); tb.h.assign(h, h + n); tb.d.assign(d, d + n); tb.m.assign(m, m + n);
    tb.k.assign(k, k + n); tb.cp.assign(cp, cp + n); tb.b.assign(b, b + n);
    tb.rhoh.resize(n);
    for (int i = 0; i < n; ++i) tb.rhoh[i] = tb.d[i] * tb.h[i];
    tb.dhmin = *std::min_element(tb.rhoh.begin(), tb.rhoh.end());
    tb.dhmax = *std::max_element(tb.rhoh.begin(), tb.rhoh.end());
    th.rPrRen = rPrRen;
    th.qw[0] = qw[0]; th.qw[1] = qw[1];
    Ftp f0{};
    f0.t = t_ini;
    ftp_from_t(tb, f0);
    const size_t nccc = (size_t)dm.nc[0] * dm.nc[1] * dm.nc[2];
    th.rhoh.assign(nccc, f0.rhoh); th.hEnth.assign(nccc, f0.h); th.tTemp.assign(nccc, f0.t);
    th.kCond.assign(nccc, f0.k); th.dDens.assign(nccc, f0.d); th.mVisc.assign(nccc, f0.m);
    th.ene_rhs0.assign(nccc, 0.0);
    th.fbcy_ftp.assign((size_t)dm.nc[0] * 4 * dm.nc[2], f0);
    th.gx.assign(fl.qx.size(), 0.0); th.gy.assign(fl.qy.size(), 0.0); th.gz.assign(fl.qz.size(), 0.0);
    fl.thermo = true;
    convert_q_g(dm, fl, false);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_thermo_init: %s\n", e.what());
    return 1;
  }
}

// One substep of the time loop (src/chapsim.f90:292-309): energy (variable-property runs, isub
// >= 1) then momentum.  isub = 0 is the initial momentum-only step (src/chapsim.f90:135).
int orc_substep(void* p, int isub, double* bulk) {
  try {
    auto* H = static_cast<OrcHandle*>(p);
    if (H->fl.thermo && isub >= 1) energy_substep(H->dm, H->fl, isub);
    momentum_substep(H->dm, H->fl, isub, bulk);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "orc_substep: %s\n", e.what());
    return 1;
  }
}

// thermal fields out (ccc): rho*h, h, T, kappa, rho, mu; momentum gx, gy, gz
void orc_get_thermo(void* p, double* rhoh, double* h, double* T, double* k, double* d, double* m, double* gx,
                    double* gy, double* gz) {
  auto* H = static_cast<OrcHandle*>(p);
  const Thermo& th = H->fl.th;
  std::memcpy(rhoh, th.rhoh.data(), th.rhoh.size() * sizeof(double));
  std::memcpy(h, th.hEnth.data(), th.hEnth.size() * sizeof(double));
  std::memcpy(T, th.tTemp.data(), th.tTemp.size() * sizeof(double));
  std::memcpy(k, th.kCond.data(), th.kCond.size() * sizeof(double));
  std::memcpy(d, th.dDens.data(), th.dDens.size() * sizeof(double));
  std::memcpy(m, th.mVisc.data(), th.mVisc.size() * sizeof(double));
  std::memcpy(gx, th.gx.data(), th.gx.size() * sizeof(double));
  std::memcpy(gy, th.gy.data(), th.gy.size() * sizeof(double));
  std::memcpy(gz, th.gz.data(), th.gz.size() * sizeof(double));
}

// per-value property lookup from rho*h with the handle's table: out[6][n] = h, T, rho, mu, kappa, cp
void orc_ftp_from_dh(void* p, int n, const double* rhoh, double* out) {
  auto* H = static_cast<OrcHandle*>(p);
  for (int i = 0; i < n; ++i) {
    Ftp f{};
    f.rhoh = rhoh[i];
    ftp_from_dh(H->fl.th.tab, f);
    out[i] = f.h; out[n + i] = f.t; out[2 * n + i] = f.d; out[3 * n + i] = f.m; out[4 * n + i] = f.k;
    out[5 * n + i] = f.cp;
  }
}

// Poisson solve in place on a (nc0, nc1, nc2) array, dispatching like solve_fft_poisson
int orc_poisson(void* p, double* rhs) {
  auto* H = static_cast<OrcHandle*>(p);
  const Domain& dm = H->dm;
  std::vector<double> r(rhs, rhs + (size_t)dm.nc[0] * dm.nc[1] * dm.nc[2]);
  poisson_dispatch(dm, r);
  std::memcpy(rhs, r.data(), sizeof(double) * r.size());
  return 0;
}

void orc_divergence(void* p, double* div) {
  auto* H = static_cast<OrcHandle*>(p);
  Arr d = divergence(H->dm, H->fl);
  std::memcpy(div, d.v.data(), sizeof(double) * d.size());
}

double orc_bulk_ke(void* p) {
  auto* H = static_cast<OrcHandle*>(p);
  return bulk_ke(H->dm, H->fl);
}

double orc_vol_average_pcc(void* p, const double* a) {
  auto* H = static_cast<OrcHandle*>(p);
  Arr x(H->dm.np[0], H->dm.nc[1], H->dm.nc[2]);
  std::memcpy(x.v.data(), a, sizeof(double) * x.size());
  return vol_average(H->dm, x);
}

}  // extern "C"
