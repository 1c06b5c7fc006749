// ORACLE (test infrastructure only; never linked into the product library).
//
// Ghost cells, RHS builders and the 1D/3D operator wrappers of CHAPSim2's
// compact finite-difference module, restated line by line from
// src/basics_operations2.f90 (ghost cells :1803-1968, RHS builders
// :1980-2738, 1D wrappers :2739-3950, 3D wrappers :3952-4800).
#include "orc_domain.h"

#include <cmath>
#include <map>
#include <stdexcept>
#include <tuple>

namespace orc {

// bc_ghost_cd = .true., bc_intp_upw = .false. (basics_operations2.f90:33-34)

// buildup_ghost_cells_C (basics_operations2.f90:1805-1880); fc[0..3] <-> fc(-1:2)
static void ghost_C(const double* fi, int nc, const int ibc[2], double fc_[4], const double* fbc,
                    const double dp[4]) {
  double* fc = fc_ + 1;  // fc[-1..2]
#define FI(i) fi[(i)-1]
#define FBC(i) fbc[(i)-1]
#define DP(i) dp[(i)-1]
  switch (ibc[0]) {
    case BC_INTERIOR: fc[0] = FBC(1); fc[-1] = FBC(3); break;
    case BC_PERIODIC: fc[0] = FI(nc); fc[-1] = FI(nc - 1); break;
    case BC_SYMMETRIC: fc[0] = FI(1); fc[-1] = FI(2); break;
    case BC_ASYMMETRIC: fc[0] = -FI(1); fc[-1] = -FI(2); break;
    case BC_DIRICHLET: fc[0] = 2.0 * FBC(1) - FI(1); fc[-1] = 2.0 * FBC(1) - FI(2); break;
    case BC_NEUMANN: fc[0] = FI(1) - FBC(1) * DP(1); fc[-1] = FI(2) - FBC(1) * DP(3); break;
    default: fc[0] = MAXP; fc[-1] = MAXP;
  }
  switch (ibc[1]) {
    case BC_INTERIOR: fc[1] = FBC(2); fc[2] = FBC(4); break;
    case BC_PERIODIC: fc[1] = FI(1); fc[2] = FI(2); break;
    case BC_SYMMETRIC: fc[1] = FI(nc); fc[2] = FI(nc - 1); break;
    case BC_ASYMMETRIC: fc[1] = -FI(nc); fc[2] = -FI(nc - 1); break;
    case BC_DIRICHLET: fc[1] = 2.0 * FBC(2) - FI(nc); fc[2] = 2.0 * FBC(2) - FI(nc - 1); break;
    case BC_NEUMANN: fc[1] = FI(nc) + FBC(2) * DP(2); fc[2] = FI(nc - 1) + FBC(2) * DP(4); break;
    default: fc[1] = MAXP; fc[2] = MAXP;
  }
}

// buildup_ghost_cells_P (basics_operations2.f90:1883-1966); fp[0..3] <-> fp(-1:2)
static void ghost_P(const double* fi, int np, const int ibc[2], double fp_[4], const double* fbc,
                    const double dp[4]) {
  double* fp = fp_ + 1;
  switch (ibc[0]) {
    case BC_INTERIOR: fp[0] = FBC(1); fp[-1] = FBC(3); break;
    case BC_PERIODIC: fp[0] = FI(np); fp[-1] = FI(np - 1); break;
    case BC_SYMMETRIC: fp[0] = FI(2); fp[-1] = FI(3); break;
    case BC_ASYMMETRIC: fp[0] = -FI(2); fp[-1] = -FI(3); break;
    case BC_DIRICHLET:
      if (fbc) { fp[0] = 2.0 * FBC(1) - FI(2); fp[-1] = 2.0 * FBC(1) - FI(3); }
      else { fp[0] = 2.0 * FI(1) - FI(2); fp[-1] = 2.0 * FI(1) - FI(3); }
      break;
    case BC_NEUMANN: fp[0] = FI(2) - FBC(1) * DP(1); fp[-1] = FI(3) - FBC(1) * DP(3); break;
    default: fp[0] = MAXP; fp[-1] = MAXP;
  }
  switch (ibc[1]) {
    case BC_INTERIOR: fp[1] = FBC(2); fp[2] = FBC(4); break;
    case BC_PERIODIC: fp[1] = FI(1); fp[2] = FI(2); break;
    case BC_SYMMETRIC: fp[1] = FI(np - 1); fp[2] = FI(np - 2); break;
    case BC_ASYMMETRIC: fp[1] = -FI(np - 1); fp[2] = -FI(np - 2); break;
    case BC_NEUMANN: fp[1] = FI(np - 1) + FBC(2) * DP(2); fp[2] = FI(np - 2) + FBC(2) * DP(4); break;
    case BC_DIRICHLET:
      if (fbc) { fp[1] = 2.0 * FBC(2) - FI(np - 1); fp[2] = 2.0 * FBC(2) - FI(np - 2); }
      else { fp[1] = 2.0 * FI(np) - FI(np - 1); fp[2] = 2.0 * FI(np) - FI(np - 2); }
      break;
    default: fp[1] = MAXP; fp[2] = MAXP;
  }
}

// coefficient accessor: r(l, s, bc) for a fixed accuracy
struct RC {
  const Family* fam;
  int m;
  double operator()(int l, int s, int bc) const { return fam->r[l - 1][s - 1][bc][m]; }
};

static inline bool in(int v, std::initializer_list<int> set) {
  for (int s : set) if (v == s) return true;
  return false;
}

// Prepare_TDMA_interp_P2C_RHS_array (basics_operations2.f90:1980-2074)
static void rhs_interp_P2C(const double* fi, int nin, double* fo, int nc, const RC& r, const int ibc[2],
                           const double* fbc, const double dp[4]) {
#define FO(i) fo[(i)-1]
  for (int i = 1; i <= nc; ++i) FO(i) = 0.0;
  for (int i = 2; i <= nc - 2; ++i)
    FO(i) = r(3, 1, BC_PERIODIC) * (FI(i) + FI(i + 1)) + r(3, 2, BC_PERIODIC) * (FI(i - 1) + FI(i + 2));
  double fpa[4];
  ghost_P(fi, nin, ibc, fpa, fbc, dp);
  const double* fp = fpa + 1;
  bool bc1 = in(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
  bool bc5 = in(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
  int i = 1;
  if (bc1) FO(i) = r(1, 1, ibc[0]) * (FI(i) + FI(i + 1)) + r(1, 2, ibc[0]) * (fp[0] + FI(i + 2));
  else
    FO(i) = r(1, 1, BC_INTRPL) * FI(i) + r(1, 2, BC_INTRPL) * FI(i + 1) + r(1, 3, BC_INTRPL) * FI(i + 2) +
            r(1, 4, BC_INTRPL) * FI(i + 3) + r(1, 5, BC_INTRPL) * FI(i + 4) + r(1, 6, BC_INTRPL) * FI(i + 5);
  i = nc;
  if (bc5) FO(i) = r(5, 1, ibc[1]) * (FI(i) + FI(i + 1)) + r(5, 2, ibc[1]) * (FI(i - 1) + fp[1]);
  else if (ibc[1] == BC_PERIODIC)
    FO(i) = r(5, 1, BC_PERIODIC) * (FI(i) + fp[1]) + r(5, 2, BC_PERIODIC) * (FI(i - 1) + fp[2]);
  else
    FO(nc) = r(5, 1, BC_INTRPL) * FI(i + 1) + r(5, 2, BC_INTRPL) * FI(i) + r(5, 3, BC_INTRPL) * FI(i - 1) +
             r(5, 4, BC_INTRPL) * FI(i - 2) + r(5, 5, BC_INTRPL) * FI(i - 3) + r(5, 6, BC_INTRPL) * FI(i - 4);
  i = nc - 1;
  if (ibc[1] == BC_PERIODIC)
    FO(i) = r(4, 1, BC_PERIODIC) * (FI(i) + FI(i + 1)) + r(4, 2, BC_PERIODIC) * (FI(i - 1) + fp[1]);
  else FO(i) = r(4, 1, ibc[1]) * (FI(i) + FI(i + 1)) + r(4, 2, ibc[1]) * (FI(i - 1) + FI(i + 2));
}

// Prepare_TDMA_interp_C2P_RHS_array (basics_operations2.f90:2087-2208)
static void rhs_interp_C2P(const double* fi, int nin, double* fo, int np, const RC& r, const int ibc[2],
                           const double* fbc, const double dp[4]) {
  for (int i = 1; i <= np; ++i) FO(i) = 0.0;
  for (int i = 3; i <= np - 2; ++i)
    FO(i) = r(3, 1, BC_PERIODIC) * (FI(i) + FI(i - 1)) + r(3, 2, BC_PERIODIC) * (FI(i + 1) + FI(i - 2));
  double fca[4];
  ghost_C(fi, nin, ibc, fca, fbc, dp);
  const double* fc = fca + 1;
  bool bc1 = in(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_NEUMANN});
  bool bc5 = in(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_NEUMANN});
  bool bc2 = bc1 || ibc[0] == BC_DIRICHLET;
  bool bc4 = bc5 || ibc[1] == BC_DIRICHLET;
  int i = 1;
  if (bc1) FO(i) = r(1, 1, ibc[0]) * (FI(i) + fc[0]) + r(1, 2, ibc[0]) * (FI(i + 1) + fc[-1]);
  else if (ibc[0] == BC_DIRICHLET) FO(i) = FBC(1);
  else
    FO(i) = r(1, 1, BC_INTRPL) * FI(i) + r(1, 2, BC_INTRPL) * FI(i + 1) + r(1, 3, BC_INTRPL) * FI(i + 2) +
            r(1, 4, BC_INTRPL) * FI(i + 3) + r(1, 5, BC_INTRPL) * FI(i + 4) + r(1, 6, BC_INTRPL) * FI(i + 5);
  i = 2;
  if (bc2) FO(i) = r(2, 1, ibc[0]) * (FI(i) + FI(i - 1)) + r(2, 2, ibc[0]) * (FI(i + 1) + fc[0]);
  else
    FO(i) = r(2, 1, BC_INTRPL) * FI(i - 1) + r(2, 2, BC_INTRPL) * FI(i) + r(2, 3, BC_INTRPL) * FI(i + 1) +
            r(2, 4, BC_INTRPL) * FI(i + 2) + r(2, 5, BC_INTRPL) * FI(i + 3) + r(2, 6, BC_INTRPL) * FI(i + 4);
  i = np;
  if (bc5) FO(i) = r(5, 1, ibc[1]) * (fc[1] + FI(i - 1)) + r(5, 2, ibc[1]) * (fc[2] + FI(i - 2));
  else if (ibc[1] == BC_PERIODIC)
    FO(i) = r(5, 1, BC_PERIODIC) * (FI(i) + FI(i - 1)) + r(5, 2, BC_PERIODIC) * (fc[1] + FI(i - 2));
  else if (ibc[1] == BC_DIRICHLET) FO(i) = FBC(2);
  else
    FO(i) = r(5, 1, BC_INTRPL) * FI(i - 1) + r(5, 2, BC_INTRPL) * FI(i - 2) + r(5, 3, BC_INTRPL) * FI(i - 3) +
            r(5, 4, BC_INTRPL) * FI(i - 4) + r(5, 5, BC_INTRPL) * FI(i - 5) + r(5, 6, BC_INTRPL) * FI(i - 6);
  i = np - 1;
  if (bc4) FO(i) = r(4, 1, ibc[1]) * (FI(i) + FI(i - 1)) + r(4, 2, ibc[1]) * (fc[1] + FI(i - 2));
  else if (ibc[1] == BC_PERIODIC)
    FO(i) = r(4, 1, BC_PERIODIC) * (FI(i) + FI(i - 1)) + r(4, 2, BC_PERIODIC) * (FI(i + 1) + FI(i - 2));
  else
    FO(i) = r(4, 1, BC_INTRPL) * FI(i) + r(4, 2, BC_INTRPL) * FI(i - 1) + r(4, 3, BC_INTRPL) * FI(i - 2) +
            r(4, 4, BC_INTRPL) * FI(i - 3) + r(4, 5, BC_INTRPL) * FI(i - 4) + r(4, 6, BC_INTRPL) * FI(i - 5);
}

// Prepare_TDMA_1deri_C2C_RHS_array (basics_operations2.f90:2230-2333)
static void rhs_d1_C2C(const double* fi, int nin, double* fo, int nc, const RC& r, double dd, const int ibc[2],
                       const double* fbc, const double dp[4]) {
  for (int i = 1; i <= nc; ++i) FO(i) = 0.0;
  for (int i = 3; i <= nc - 2; ++i)
    FO(i) = r(3, 1, BC_PERIODIC) * (FI(i + 1) - FI(i - 1)) + r(3, 2, BC_PERIODIC) * (FI(i + 2) - FI(i - 2));
  double fca[4];
  ghost_C(fi, nin, ibc, fca, fbc, dp);
  const double* fc = fca + 1;
  bool isbc[2];
  for (int k = 0; k < 2; ++k)
    isbc[k] = in(ibc[k], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
  int i = 1;
  if (isbc[0]) FO(i) = r(1, 1, ibc[0]) * (FI(i + 1) - fc[0]) + r(1, 2, ibc[0]) * (FI(i + 2) - fc[-1]);
  else
    FO(i) = r(1, 1, BC_INTRPL) * FI(i) + r(1, 2, BC_INTRPL) * FI(i + 1) + r(1, 3, BC_INTRPL) * FI(i + 2) +
            r(1, 4, BC_INTRPL) * FI(i + 3) + r(1, 5, BC_INTRPL) * FI(i + 4) + r(1, 6, BC_INTRPL) * FI(i + 5);
  i = 2;
  if (isbc[0]) FO(i) = r(2, 1, ibc[0]) * (FI(i + 1) - FI(i - 1)) + r(2, 2, ibc[0]) * (FI(i + 2) - fc[0]);
  else
    FO(i) = r(2, 1, BC_INTRPL) * FI(i - 1) + r(2, 2, BC_INTRPL) * FI(i) + r(2, 3, BC_INTRPL) * FI(i + 1) +
            r(2, 4, BC_INTRPL) * FI(i + 2) + r(2, 5, BC_INTRPL) * FI(i + 3) + r(2, 6, BC_INTRPL) * FI(i + 4);
  i = nc;
  if (isbc[1]) FO(i) = r(5, 1, ibc[1]) * (fc[1] - FI(i - 1)) + r(5, 2, ibc[1]) * (fc[2] - FI(i - 2));
  else
    FO(i) = r(5, 1, BC_INTRPL) * FI(i) + r(5, 2, BC_INTRPL) * FI(i - 1) + r(5, 3, BC_INTRPL) * FI(i - 2) +
            r(5, 4, BC_INTRPL) * FI(i - 3) + r(5, 5, BC_INTRPL) * FI(i - 4) + r(5, 6, BC_INTRPL) * FI(i - 5);
  i = nc - 1;
  if (isbc[1]) FO(i) = r(4, 1, ibc[1]) * (FI(i + 1) - FI(i - 1)) + r(4, 2, ibc[1]) * (fc[1] - FI(i - 2));
  else
    FO(i) = r(4, 1, BC_INTRPL) * FI(i + 1) + r(4, 2, BC_INTRPL) * FI(i) + r(4, 3, BC_INTRPL) * FI(i - 1) +
            r(4, 4, BC_INTRPL) * FI(i - 2) + r(4, 5, BC_INTRPL) * FI(i - 3) + r(4, 6, BC_INTRPL) * FI(i - 4);
  for (int k = 1; k <= nc; ++k) FO(k) = FO(k) * dd;
}

// Prepare_TDMA_1deri_P2P_RHS_array (basics_operations2.f90:2352-2463)
static void rhs_d1_P2P(const double* fi, int nin, double* fo, int np, const RC& r, double dd, const int ibc[2],
                       const double* fbc, const double dp[4]) {
  for (int i = 1; i <= np; ++i) FO(i) = 0.0;
  for (int i = 3; i <= np - 2; ++i)
    FO(i) = r(3, 1, BC_PERIODIC) * (FI(i + 1) - FI(i - 1)) + r(3, 2, BC_PERIODIC) * (FI(i + 2) - FI(i - 2));
  double fpa[4];
  ghost_P(fi, nin, ibc, fpa, fbc, dp);
  const double* fp = fpa + 1;
  bool b1[2], b2[2];
  for (int k = 0; k < 2; ++k) {
    b1[k] = in(ibc[k], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET});
    b2[k] = b1[k] || ibc[k] == BC_DIRICHLET || ibc[k] == BC_NEUMANN;
  }
  int i = 1;
  if (b1[0]) FO(i) = r(1, 1, ibc[0]) * (FI(i + 1) - fp[0]) + r(1, 2, ibc[0]) * (FI(i + 2) - fp[-1]);
  else if (ibc[0] == BC_NEUMANN) FO(i) = FBC(1) / dd;
  else
    FO(i) = r(1, 1, BC_INTRPL) * FI(i) + r(1, 2, BC_INTRPL) * FI(i + 1) + r(1, 3, BC_INTRPL) * FI(i + 2) +
            r(1, 4, BC_INTRPL) * FI(i + 3) + r(1, 5, BC_INTRPL) * FI(i + 4) + r(1, 6, BC_INTRPL) * FI(i + 5);
  i = 2;
  if (b2[0]) FO(i) = r(2, 1, ibc[0]) * (FI(i + 1) - FI(i - 1)) + r(2, 2, ibc[0]) * (FI(i + 2) - fp[0]);
  else
    FO(i) = r(2, 1, BC_INTRPL) * FI(i - 1) + r(2, 2, BC_INTRPL) * FI(i) + r(2, 3, BC_INTRPL) * FI(i + 1) +
            r(2, 4, BC_INTRPL) * FI(i + 2) + r(2, 5, BC_INTRPL) * FI(i + 3) + r(2, 6, BC_INTRPL) * FI(i + 4);
  i = np;
  if (b1[1]) FO(i) = r(5, 1, ibc[1]) * (fp[1] - FI(i - 1)) + r(5, 2, ibc[1]) * (fp[2] - FI(i - 2));
  else if (ibc[1] == BC_NEUMANN) FO(i) = FBC(2) / dd;
  else
    FO(i) = r(5, 1, BC_INTRPL) * FI(i) + r(5, 2, BC_INTRPL) * FI(i - 1) + r(5, 3, BC_INTRPL) * FI(i - 2) +
            r(5, 4, BC_INTRPL) * FI(i - 3) + r(5, 5, BC_INTRPL) * FI(i - 4) + r(5, 6, BC_INTRPL) * FI(i - 5);
  i = np - 1;
  if (b2[1]) FO(i) = r(4, 1, ibc[1]) * (FI(i + 1) - FI(i - 1)) + r(4, 2, ibc[1]) * (fp[1] - FI(i - 2));
  else
    FO(i) = r(4, 1, BC_INTRPL) * FI(i + 1) + r(4, 2, BC_INTRPL) * FI(i) + r(4, 3, BC_INTRPL) * FI(i - 1) +
            r(4, 4, BC_INTRPL) * FI(i - 2) + r(4, 5, BC_INTRPL) * FI(i - 3) + r(4, 6, BC_INTRPL) * FI(i - 4);
  for (int k = 1; k <= np; ++k) FO(k) = FO(k) * dd;
}

// Prepare_TDMA_1deri_C2P_RHS_array (basics_operations2.f90:2482-2604).  The is_bc4 test reads
// ibc(1) where ibc(2) is meant (basics_operations2.f90:2540-2544); restated as written.
static void rhs_d1_C2P(const double* fi, int nin, double* fo, int np, const RC& r, double dd, const int ibc[2],
                       const double* fbc, const double dp[4]) {
  for (int i = 1; i <= np; ++i) FO(i) = 0.0;
  for (int i = 3; i <= np - 2; ++i)
    FO(i) = r(3, 1, BC_PERIODIC) * (FI(i) - FI(i - 1)) + r(3, 2, BC_PERIODIC) * (FI(i + 1) - FI(i - 2));
  double fca[4];
  ghost_C(fi, nin, ibc, fca, fbc, dp);
  const double* fc = fca + 1;
  bool bc1 = in(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET});
  bool bc2 = bc1 || ibc[0] == BC_DIRICHLET || ibc[0] == BC_NEUMANN;
  bool bc5 = in(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET});
  bool bc4 = bc5 || ibc[0] == BC_DIRICHLET || ibc[0] == BC_NEUMANN;
  int i = 1;
  if (bc1) FO(i) = r(1, 1, ibc[0]) * (FI(i) - fc[0]) + r(1, 2, ibc[0]) * (FI(i + 1) - fc[-1]);
  else if (ibc[0] == BC_NEUMANN) FO(i) = FBC(1) / dd;
  else
    FO(i) = r(1, 1, BC_INTRPL) * FI(i) + r(1, 2, BC_INTRPL) * FI(i + 1) + r(1, 3, BC_INTRPL) * FI(i + 2) +
            r(1, 4, BC_INTRPL) * FI(i + 3) + r(1, 5, BC_INTRPL) * FI(i + 4) + r(1, 6, BC_INTRPL) * FI(i + 5);
  i = 2;
  if (bc2) FO(i) = r(2, 1, ibc[0]) * (FI(i) - FI(i - 1)) + r(2, 2, ibc[0]) * (FI(i + 1) - fc[0]);
  else
    FO(i) = r(2, 1, BC_INTRPL) * FI(i - 1) + r(2, 2, BC_INTRPL) * FI(i) + r(2, 3, BC_INTRPL) * FI(i + 1) +
            r(2, 4, BC_INTRPL) * FI(i + 2) + r(2, 5, BC_INTRPL) * FI(i + 3) + r(2, 6, BC_INTRPL) * FI(i + 4);
  i = np;
  if (bc5) FO(i) = r(5, 1, ibc[1]) * (fc[1] - FI(i - 1)) + r(5, 2, ibc[1]) * (fc[2] - FI(i - 2));
  else if (ibc[1] == BC_PERIODIC)
    FO(i) = r(5, 1, BC_PERIODIC) * (FI(i) - FI(i - 1)) + r(5, 2, BC_PERIODIC) * (fc[1] - FI(i - 2));
  else if (ibc[1] == BC_NEUMANN) FO(i) = FBC(2) / dd;
  else
    FO(i) = r(5, 1, BC_INTRPL) * FI(i - 1) + r(5, 2, BC_INTRPL) * FI(i - 2) + r(5, 3, BC_INTRPL) * FI(i - 3) +
            r(5, 4, BC_INTRPL) * FI(i - 4) + r(5, 5, BC_INTRPL) * FI(i - 5) + r(5, 6, BC_INTRPL) * FI(i - 6);
  i = np - 1;
  if (bc4) FO(i) = r(4, 1, ibc[1]) * (FI(i) - FI(i - 1)) + r(4, 2, ibc[1]) * (fc[1] - FI(i - 2));
  else if (ibc[1] == BC_PERIODIC)
    FO(i) = r(4, 1, BC_PERIODIC) * (FI(i) - FI(i - 1)) + r(4, 2, BC_PERIODIC) * (FI(i + 1) - FI(i - 2));
  else
    FO(i) = r(4, 1, BC_INTRPL) * FI(i) + r(4, 2, BC_INTRPL) * FI(i - 1) + r(4, 3, BC_INTRPL) * FI(i - 2) +
            r(4, 4, BC_INTRPL) * FI(i - 3) + r(4, 5, BC_INTRPL) * FI(i - 4) + r(4, 6, BC_INTRPL) * FI(i - 5);
  for (int k = 1; k <= np; ++k) FO(k) = FO(k) * dd;
}

// Prepare_TDMA_1deri_P2C_RHS_array (basics_operations2.f90:2617-2705)
static void rhs_d1_P2C(const double* fi, int nin, double* fo, int nc, const RC& r, double dd, const int ibc[2],
                       const double* fbc, const double dp[4]) {
  for (int i = 1; i <= nc; ++i) FO(i) = 0.0;
  for (int i = 2; i <= nc - 2; ++i)
    FO(i) = r(3, 1, BC_PERIODIC) * (FI(i + 1) - FI(i)) + r(3, 2, BC_PERIODIC) * (FI(i + 2) - FI(i - 1));
  double fpa[4];
  ghost_P(fi, nin, ibc, fpa, fbc, dp);
  const double* fp = fpa + 1;
  bool bc1 = in(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
  bool bc5 = in(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
  int i = 1;
  if (bc1) FO(i) = r(1, 1, ibc[0]) * (FI(i + 1) - FI(i)) + r(1, 2, ibc[0]) * (FI(i + 2) - fp[0]);
  else
    FO(i) = r(1, 1, BC_INTRPL) * FI(i) + r(1, 2, BC_INTRPL) * FI(i + 1) + r(1, 3, BC_INTRPL) * FI(i + 2) +
            r(1, 4, BC_INTRPL) * FI(i + 3) + r(1, 5, BC_INTRPL) * FI(i + 4) + r(1, 6, BC_INTRPL) * FI(i + 5);
  i = nc;
  if (bc5) FO(i) = r(5, 1, ibc[1]) * (FI(i + 1) - FI(i)) + r(5, 2, ibc[1]) * (fp[1] - FI(i - 1));
  else if (ibc[1] == BC_PERIODIC)
    FO(i) = r(5, 1, BC_PERIODIC) * (fp[1] - FI(i)) + r(5, 2, BC_PERIODIC) * (fp[2] - FI(i - 1));
  else
    FO(i) = r(5, 1, BC_INTRPL) * FI(i + 1) + r(5, 2, BC_INTRPL) * FI(i) + r(5, 3, BC_INTRPL) * FI(i - 1) +
            r(5, 4, BC_INTRPL) * FI(i - 2) + r(5, 5, BC_INTRPL) * FI(i - 3) + r(5, 6, BC_INTRPL) * FI(i - 4);
  i = nc - 1;
  if (ibc[1] == BC_PERIODIC)
    FO(i) = r(4, 1, BC_PERIODIC) * (FI(i + 1) - FI(i)) + r(4, 2, BC_PERIODIC) * (fp[1] - FI(i - 1));
  else FO(i) = r(4, 1, BC_PERIODIC) * (FI(i + 1) - FI(i)) + r(4, 2, BC_PERIODIC) * (FI(i + 2) - FI(i - 1));
  for (int k = 1; k <= nc; ++k) FO(k) = FO(k) * dd;
}
#undef FI
#undef FO
#undef FBC
#undef DP

// ---------------------------------------------------------------------------
// LHS cache and the 1D operator wrapper (Get_{x,y,z}_{midp,1der}_*_1D,
// basics_operations2.f90:2739-3950)
// ---------------------------------------------------------------------------
const Lhs& Domain::lhs(int fam, int n, int bc1, int bc2) const {
  auto key = std::make_tuple(fam, n, bc1, bc2);
  auto it = lhs_cache.find(key);
  if (it != lhs_cache.end()) return it->second;
  Lhs L;
  build_lhs(T.fam[fam], n, bc1, bc2, iacc, L);
  return lhs_cache.emplace(key, std::move(L)).first->second;
}

static bool is_c_input(int fam) { return fam == FAM_D1C2C || fam == FAM_D1C2P || fam == FAM_M1C2P; }
static bool is_deriv(int fam) { return fam <= FAM_D1P2C; }

int op_out_len(const Domain& dm, int dir, int fam) {
  bool to_p = (fam == FAM_D1P2P || fam == FAM_D1C2P || fam == FAM_M1C2P);
  return to_p ? dm.np[dir] : dm.nc[dir];
}
int op_in_len(const Domain& dm, int dir, int fam) {
  bool from_p = (fam == FAM_D1P2P || fam == FAM_D1P2C || fam == FAM_M1P2C);
  return from_p ? dm.np[dir] : dm.nc[dir];
}

// reduce_bc_to_interp (basics_operations2.f90:339-354) as applied by each 1D wrapper when no
// boundary values are supplied: C-input operators reduce interior/Dirichlet/Neumann ends,
// P-input operators reduce interior/Neumann ends.
void reduce_bc(int fam, const int ibc0[2], bool has_fbc, int ibc[2]) {
  for (int k = 0; k < 2; ++k) {
    ibc[k] = ibc0[k];
    if (has_fbc) continue;
    if (ibc[k] == BC_INTERIOR || ibc[k] == BC_NEUMANN) ibc[k] = BC_INTRPL;
    if (ibc[k] == BC_DIRICHLET && is_c_input(fam)) ibc[k] = BC_INTRPL;
  }
}

void op1d(const Domain& dm, int dir, int fam, const int ibc0[2], const double* fbc, const double* fi, double* fo) {
  const int nin = op_in_len(dm, dir, fam), nout = op_out_len(dm, dir, fam);
  int ibc[2];
  reduce_bc(fam, ibc0, fbc != nullptr, ibc);
  double dp[4];
  if (dir != 1) {
    double h = dm.h[dir];
    if (is_c_input(fam)) { dp[0] = h; dp[2] = h * 2.0; dp[1] = h; dp[3] = h * 2.0; }
    else { dp[0] = h * 2.0; dp[2] = h * 4.0; dp[1] = h * 2.0; dp[3] = h * 4.0; }
  } else {
    const int np2 = dm.np[1], nc2 = dm.nc[1];
    const auto& yp = dm.yp;
    const auto& yc = dm.yc;
    if (is_c_input(fam)) {
      dp[0] = (yc[0] - yp[0]) * 2.0;
      dp[2] = (yc[1] - yp[0]) * 2.0;
      dp[1] = (yp[np2 - 1] - yc[nc2 - 1]) * 2.0;
      dp[3] = (yp[np2 - 1] - yc[nc2 - 2]) * 2.0;
    } else {
      dp[0] = (yp[1] - yp[0]) * 2.0;
      dp[2] = (yp[2] - yp[0]) * 2.0;
      dp[1] = (yp[np2 - 1] - yp[np2 - 2]) * 2.0;
      dp[3] = (yp[np2 - 1] - yp[np2 - 3]) * 2.0;
    }
  }
  RC r{&dm.T.fam[fam], dm.iacc - 1};
  const double dd = dm.h1r[dir];
  switch (fam) {
    case FAM_M1P2C: rhs_interp_P2C(fi, nin, fo, nout, r, ibc, fbc, dp); break;
    case FAM_M1C2P: rhs_interp_C2P(fi, nin, fo, nout, r, ibc, fbc, dp); break;
    case FAM_D1C2C: rhs_d1_C2C(fi, nin, fo, nout, r, dd, ibc, fbc, dp); break;
    case FAM_D1P2P: rhs_d1_P2P(fi, nin, fo, nout, r, dd, ibc, fbc, dp); break;
    case FAM_D1C2P: rhs_d1_C2P(fi, nin, fo, nout, r, dd, ibc, fbc, dp); break;
    case FAM_D1P2C: rhs_d1_P2C(fi, nin, fo, nout, r, dd, ibc, fbc, dp); break;
  }
  if (dm.iacc == ACC_CP4 || dm.iacc == ACC_CP6) {
    const Lhs& L = dm.lhs(fam, nout, ibc[0], ibc[1]);
    tdma_solve(ibc[0] == BC_PERIODIC, fo, L.a.data(), L.b.data(), L.c.data(), L.d.data(), nout);
  }
  if (dir == 1 && is_deriv(fam)) {
    if (dm.stretch_y) {
      const bool at_cc = (fam == FAM_D1C2C || fam == FAM_D1P2C);
      const auto& mp = at_cc ? dm.mpcc : dm.mppt;
      for (int i = 0; i < nout; ++i) fo[i] = fo[i] * mp[i];
    }
    if (fam == FAM_D1P2P || fam == FAM_D1C2P) {
      if (ibc[0] == BC_NEUMANN && fbc) fo[0] = fbc[0];
      if (ibc[1] == BC_NEUMANN && fbc) fo[nout - 1] = fbc[1];
    }
  }
}

// 3D wrapper: loops over lines of an x-fastest (Fortran order) array.  fbc2d, when given,
// holds 4 planes laid out like the reference's fbcx(4,n2,n3) / fbcy(n1,4,n3) / fbcz(n1,n2,4).
void op3d(const Domain& dm, int dir, int fam, const int ibc[2], const double* fbc2d, const double* fi3d,
          const int nin3[3], double* fo3d) {
  const int nin = op_in_len(dm, dir, fam), nout = op_out_len(dm, dir, fam);
  if (nin3[dir] != nin) throw std::runtime_error("op3d: input extent mismatch");
  int nout3[3] = {nin3[0], nin3[1], nin3[2]};
  nout3[dir] = nout;
  const int n1 = nin3[0], n2 = nin3[1], n3 = nin3[2];
  const int o1 = nout3[0], o2 = nout3[1];
  std::vector<double> fi(nin), fo(nout);
  double fbc[4];
  if (dm.iacc == ACC_CP4 || dm.iacc == ACC_CP6) {  // build the LHS before the threaded loop
    int rb[2];
    reduce_bc(fam, ibc, fbc2d != nullptr, rb);
    dm.lhs(fam, nout, rb[0], rb[1]);
  }
  if (dir == 0) {
#pragma omp parallel for collapse(2) firstprivate(fi, fo, fbc)
    for (int k = 0; k < n3; ++k)
      for (int j = 0; j < n2; ++j) {
        for (int i = 0; i < nin; ++i) fi[i] = fi3d[(size_t)(k * n2 + j) * n1 + i];
        if (fbc2d) for (int u = 0; u < 4; ++u) fbc[u] = fbc2d[(size_t)(k * n2 + j) * 4 + u];
        op1d(dm, dir, fam, ibc, fbc2d ? fbc : nullptr, fi.data(), fo.data());
        for (int i = 0; i < nout; ++i) fo3d[(size_t)(k * o2 + j) * o1 + i] = fo[i];
      }
  } else if (dir == 1) {
#pragma omp parallel for collapse(2) firstprivate(fi, fo, fbc)
    for (int k = 0; k < n3; ++k)
      for (int i = 0; i < n1; ++i) {
        for (int j = 0; j < nin; ++j) fi[j] = fi3d[(size_t)(k * n2 + j) * n1 + i];
        if (fbc2d) for (int u = 0; u < 4; ++u) fbc[u] = fbc2d[(size_t)(k * 4 + u) * n1 + i];
        op1d(dm, dir, fam, ibc, fbc2d ? fbc : nullptr, fi.data(), fo.data());
        for (int j = 0; j < nout; ++j) fo3d[(size_t)(k * o2 + j) * o1 + i] = fo[j];
      }
  } else {
#pragma omp parallel for collapse(2) firstprivate(fi, fo, fbc)
    for (int j = 0; j < n2; ++j)
      for (int i = 0; i < n1; ++i) {
        for (int k = 0; k < nin; ++k) fi[k] = fi3d[(size_t)(k * n2 + j) * n1 + i];
        if (fbc2d) for (int u = 0; u < 4; ++u) fbc[u] = fbc2d[(size_t)(u * n2 + j) * n1 + i];
        op1d(dm, dir, fam, ibc, fbc2d ? fbc : nullptr, fi.data(), fo.data());
        for (int k = 0; k < nout; ++k) fo3d[(size_t)(k * o2 + j) * o1 + i] = fo[k];
      }
  }
}

}  // namespace orc
