// ORACLE (test infrastructure only; never linked into the product library).
// Domain, flow state and entry points of the CPU FP64 restatement.
#pragma once
#include <map>
#include <tuple>
#include <vector>

#include "orc.h"

namespace orc {

// variable slots of the nominal boundary-condition table (src/modules.f90 ibc*_nominal(2,5))
enum { V_QX = 0, V_QY = 1, V_QZ = 2, V_PR = 3, V_TM = 4 };

struct Domain {
  // grid (src/geometry.f90:410-530)
  int nc[3], np[3], np_geo[3];
  bool periodic[3];
  bool stretch_y;
  int istret;
  double rstret;
  double lxx, lyt, lyb, lzz;
  double h[3], h1r[3], h2r[3];
  std::vector<double> yp, yc, mppt, mpcc;  // yp(np_geo), yc(nc), yMappingpt(:,1), yMappingcc(:,1)
  int iacc;
  Tables T;
  mutable std::map<std::tuple<int, int, int, int>, Lhs> lhs_cache;
  const Lhs& lhs(int fam, int n, int bc1, int bc2) const;

  // calculated boundary conditions (src/bc_general.f90:137-248), [var][side]
  int ibcx[5][2], ibcy[5][2], ibcz[5][2];
  int ibcy_ftp[2];
  double fbcy_const[5][2];
  // operation boundary conditions (src/bc_general.f90:512-760)
  int mbcx_cov1[2], mbcy_cov1[2], mbcz_cov1[2], mbcx_tau1[2], mbcy_tau1[2], mbcz_tau1[2];
  int mbcx_cov2[2], mbcy_cov2[2], mbcz_cov2[2], mbcx_tau2[2], mbcy_tau2[2], mbcz_tau2[2];
  int mbcx_cov3[2], mbcy_cov3[2], mbcz_cov3[2], mbcx_tau3[2], mbcy_tau3[2], mbcz_tau3[2];
  bool fbcy_velo_required;

  // time stepping (src/input_general.f90:851-886)
  double dt, tGamma[4], tZeta[4], tAlpha[4], sigma2p;
  double rre;
  int idriven;
  int ifft;  // 2 = FISHPACK (x/z FFT + y TDMA), 3 = 3D FFT with modified wavenumbers

  // Poisson tables
  std::vector<double> xrt, zrt, pa, pb, pc;  // FISHPACK roots and y coefficients
};

// One thermal state (t_fluidThermoProperty, src/modules.f90): nondimensional values.
struct Ftp {
  double rhoh, h, t, d, m, k, cp, b;
};

// Property table sorted by T (ftplist, src/input_thermo.f90:512-556), nondimensional, with the
// rho*h range used for clamping (:683-688).
struct ThermoTable {
  std::vector<double> t, h, d, m, k, cp, b, rhoh;
  double dhmin = 0.0, dhmax = 0.0;
  int n() const { return (int)t.size(); }
};

// Thermal state of a variable-property run (t_thermo plus the flow's density, viscosity and
// momentum, src/modules.f90:412-681).  Ordering of ccc arrays: x fastest.
struct Thermo {
  ThermoTable tab;
  double rPrRen = 0.0;
  double qw[2] = {0.0, 0.0};  // wall heat flux (Neumann T) at y walls, fbcy_qw
  std::vector<double> rhoh, hEnth, tTemp, kCond, dDens, mVisc, ene_rhs0;  // ccc
  std::vector<double> gx, gy, gz;                                          // pcc, cpc, ccp
  std::vector<Ftp> fbcy_ftp;  // wall states, reference layout (nc0, 4, nc2)
};

struct Flow {
  std::vector<double> qx, qy, qz, pres, pcor;
  std::vector<double> mx_rhs0, my_rhs0, mz_rhs0;
  bool thermo = false;
  Thermo th;
};

// ftp_refresh_thermal_properties_from_H / _from_DH (src/input_thermo.f90:345-446)
void ftp_from_h(const ThermoTable& tb, Ftp& f);
void ftp_from_dh(const ThermoTable& tb, Ftp& f);
void ftp_from_t(const ThermoTable& tb, Ftp& f);

int op_out_len(const Domain& dm, int dir, int fam);
int op_in_len(const Domain& dm, int dir, int fam);
void reduce_bc(int fam, const int ibc0[2], bool has_fbc, int ibc[2]);
void op1d(const Domain& dm, int dir, int fam, const int ibc0[2], const double* fbc, const double* fi, double* fo);
void op3d(const Domain& dm, int dir, int fam, const int ibc[2], const double* fbc2d, const double* fi3d,
          const int nin3[3], double* fo3d);

}  // namespace orc
