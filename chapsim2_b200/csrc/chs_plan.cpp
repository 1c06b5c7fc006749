// Compact-scheme coefficient sets and operator plans (host side).
//
// Coefficients: Prepare_compact_coefficients, src/basics_operations2.f90:361-1528
// (Gaitonde & Visbal 1998 tables 2.1-2.13).  Boundary rows: the RHS builders
// src/basics_operations2.f90:1980-2738 with the ghost cells of :1803-1968,
// evaluated symbolically as linear forms.  LHS: Buildup_TDMA_LHS_array and
// Preprocess_TDMA_coeffs (src/basics_operations2.f90:1529-1588,
// src/basics_algorithms.f90:14-34).
#include "chs_plan.h"

#include <cmath>
#include <cstring>
#include <stdexcept>

namespace chs {

// ---------------------------------------------------------------------------
// coefficient sets
// ---------------------------------------------------------------------------
namespace {

struct Closure {        // one boundary row of the extrapolation (IBC_INTRPL) closure
  double alpha;
  double c[6];
};

// Per-family description: bulk scheme, extrapolation closures and the rules for
// the symmetric/antisymmetric first row.  Index [acc-1].
struct FamilyDesc {
  double alpha[4], ra[4], rb[4];  // bulk LHS alpha and the two RHS coefficients
  bool rb_zero_col3;              // third RHS column of the periodic row is 0 (staggered schemes)
  Closure row1[4];
  bool has_row2;                  // extrapolation row 2 given (else rows 2:4 are periodic)
  Closure row2[4];
  double mirror;                  // sign of the row-5/row-4 RHS mirror
  // first-row LHS for symmetric / antisymmetric ends: (b, c) = (bs + ks*alpha, cs*alpha)
  double sym_b_k, sym_c_k, asym_b_k, asym_c_k;
  // which ends keep explicit identity rows (rows 1 and 5): Neumann (P2P, C2P), Dirichlet (C2P interp)
  bool neumann_identity, dirichlet_identity;
  // Dirichlet/Neumann fallbacks: rows taken from the interior set
  bool dir_all_interior, neu_all_interior;
};

inline Closure cl(double al, double a, double b, double c = 0, double d = 0, double e = 0, double f = 0) {
  return Closure{al, {a, b, c, d, e, f}};
}

FamilyDesc desc_d1c2c() {
  FamilyDesc D{};
  const double al[4] = {0.0, 0.0, 0.25, 1.0 / 3.0};
  const double a[4] = {1.0, 4.0 / 3.0, 1.5, 14.0 / 9.0};
  const double b[4] = {0.0, -1.0 / 3.0, 0.0, 1.0 / 9.0};
  for (int n = 0; n < 4; ++n) { D.alpha[n] = al[n]; D.ra[n] = a[n] * 0.5; D.rb[n] = b[n] * 0.25; }
  D.rb_zero_col3 = false;
  D.row1[0] = cl(0.0, -1.5, 2.0, -0.5);
  D.row1[1] = cl(0.0, -25.0 / 12.0, 4.0, -3.0, 4.0 / 3.0, -0.25);
  D.row1[2] = cl(3.0, -17.0 / 6.0, 1.5, 1.5, -1.0 / 6.0);
  D.row1[3] = cl(5.0, -197.0 / 60.0, -5.0 / 12.0, 5.0, -5.0 / 3.0, 5.0 / 12.0, -1.0 / 20.0);
  D.has_row2 = true;
  D.row2[0] = cl(0.0, -0.5, 0.0, 0.5);
  D.row2[1] = cl(0.0, -0.25, -5.0 / 6.0, 1.5, -0.5, 1.0 / 12.0);
  D.row2[2] = cl(0.25, -0.75, 0.0, 0.75);
  D.row2[3] = cl(2.0 / 11.0, -20.0 / 33.0, -35.0 / 132.0, 34.0 / 33.0, -7.0 / 33.0, 2.0 / 33.0, -1.0 / 132.0);
  D.mirror = -1.0;
  D.sym_b_k = -1.0; D.sym_c_k = 1.0; D.asym_b_k = 1.0; D.asym_c_k = 1.0;
  D.neumann_identity = false; D.dirichlet_identity = false;
  D.dir_all_interior = true; D.neu_all_interior = true;
  return D;
}

FamilyDesc desc_d1c2p() {
  FamilyDesc D{};
  const double al[4] = {0.0, 0.0, 1.0 / 22.0, 9.0 / 62.0};
  for (int n = 0; n < 4; ++n) D.alpha[n] = al[n];
  double a[4], b[4];
  a[0] = 1.0; b[0] = 0.0;
  for (int n : {1, 2}) { a[n] = (9.0 - 6.0 * al[n]) / 8.0; b[n] = (-1.0 + 22.0 * al[n]) / 8.0; }
  a[3] = 63.0 / 62.0; b[3] = 17.0 / 62.0;
  for (int n = 0; n < 4; ++n) { D.ra[n] = a[n]; D.rb[n] = b[n] * (1.0 / 3.0); }
  D.rb_zero_col3 = true;
  D.row1[0] = cl(0.0, -2.0, 3.0, -1.0);
  for (int n : {1, 2}) {
    const double q = 0.0;
    D.row1[n] = cl(q, (-93.0 - 22.0 * q) / 24.0, (229.0 + 17.0 * q) / 24.0, (-75.0 + 3.0 * q) / 8.0,
                   (111.0 - 5.0 * q) / 24.0, (-22.0 + q) / 24.0);
  }
  {
    const double q = 1689.0 / 71.0;
    D.row1[3] = cl(q, (-3043.0 - 563.0 * q) / 640.0, (5353.0 + 201.0 * q) / 384.0, (-3489.0 + 143.0 * q) / 192.0,
                   (859.0 - 37.0 * q) / 64.0, (-2041.0 + 87.0 * q) / 384.0, (1689.0 - 71.0 * q) / 1920.0);
  }
  D.has_row2 = true;
  D.row2[0] = cl(0.0, -1.0, 1.0);
  for (int n : {1, 2}) {
    const double q = (n == 1) ? 0.0 : 1.0 / 22.0;
    D.row2[n] = cl(q, (-11.0 - 46.0 * q) / 12.0, (17.0 + 202.0 * q) / 24.0, (3.0 - 66.0 * q) / 8.0,
                   (-5.0 + 110.0 * q) / 24.0, (1.0 - 22.0 * q) / 24.0);
  }
  D.row2[3] = cl(31.0 / 818.0, -5195.0 / 4908.0, 4957.0 / 4908.0, 119.0 / 1227.0, -85.0 / 1227.0,
                 119.0 / 4908.0, -17.0 / 4908.0);
  D.mirror = -1.0;
  D.sym_b_k = 0.0; D.sym_c_k = 0.0; D.asym_b_k = 0.0; D.asym_c_k = 2.0;
  D.neumann_identity = true; D.dirichlet_identity = false;
  D.dir_all_interior = true; D.neu_all_interior = false;
  return D;
}

FamilyDesc desc_m1c2p() {
  FamilyDesc D{};
  const double al[4] = {0.0, 0.0, 1.0 / 6.0, 0.3};
  for (int n = 0; n < 4; ++n) D.alpha[n] = al[n];
  double a[4], b[4];
  a[0] = 1.0; b[0] = 0.0;
  for (int n : {1, 2}) { a[n] = 9.0 / 8.0 + 5.0 / 4.0 * al[n]; b[n] = -1.0 / 8.0 + 3.0 / 4.0 * al[n]; }
  a[3] = 5.0 * (15.0 + 14.0 * al[3]) / 64.0;
  b[3] = (-25.0 + 126.0 * al[3]) / 128.0;
  for (int n = 0; n < 4; ++n) { D.ra[n] = a[n] * 0.5; D.rb[n] = b[n] * 0.5; }
  D.rb_zero_col3 = true;
  D.row1[0] = cl(0.0, 1.5, -0.5);
  for (int n : {1, 2}) {
    const double q = (n == 1) ? 0.0 : 5.0;
    D.row1[n] = cl(q, (35.0 + 5.0 * q) / 16.0, (-35.0 + 15.0 * q) / 16.0, (21.0 - 5.0 * q) / 16.0, (-5.0 + q) / 16.0);
  }
  {
    const double q = 9.0;
    D.row1[3] = cl(q, (693.0 + 63.0 * q) / 256.0, (-1155.0 + 315.0 * q) / 256.0, (693.0 - 105.0 * q) / 128.0,
                   (-495.0 + 63.0 * q) / 128.0, (385.0 - 45.0 * q) / 256.0, (-63.0 + 7.0 * q) / 256.0);
  }
  D.has_row2 = true;
  D.row2[0] = cl(0.0, 0.5, 0.5);
  for (int n : {1, 2}) {
    const double q = (n == 1) ? 0.0 : 1.0 / 6.0;
    D.row2[n] = cl(q, (5.0 + 34.0 * q) / 16.0, (15.0 - 26.0 * q) / 16.0, (-5.0 + 30.0 * q) / 16.0,
                   (1.0 - 6.0 * q) / 16.0);
  }
  {
    const double q = 9.0;
    D.row2[3] = cl(q, (63.0 + 686.0 * q) / 256.0, (315.0 - 1050.0 * q) / 256.0, (-105.0 + 798.0 * q) / 128.0,
                   (63.0 - 530.0 * q) / 128.0, (-45.0 + 406.0 * q) / 256.0, (7.0 - 66.0 * q) / 256.0);
  }
  D.mirror = 1.0;
  D.sym_b_k = 0.0; D.sym_c_k = 2.0; D.asym_b_k = 0.0; D.asym_c_k = 0.0;
  D.neumann_identity = false; D.dirichlet_identity = true;
  D.dir_all_interior = false; D.neu_all_interior = true;
  return D;
}

FamilyDesc desc_d1p2c() {
  FamilyDesc D = desc_d1c2p();
  D.row1[0] = cl(0.0, -1.0, 1.0);
  for (int n : {1, 2}) {
    const double q = 0.0;
    D.row1[n] = cl(q, (-22.0 + q) / 24.0, (17.0 - 27.0 * q) / 24.0, (3.0 + 9.0 * q) / 8.0, (-5.0 - q) / 24.0,
                   1.0 / 24.0);
  }
  {
    const double q = 71.0 / 9.0;
    D.row1[3] = cl(q, (-1689.0 + 71.0 * q) / 1920.0, (67.0 - 141.0 * q) / 128.0, (143.0 + 207.0 * q) / 192.0,
                   (-111.0 + q) / 192.0, (29.0 - 3.0 * q) / 128.0, (-71.0 + 9.0 * q) / 1920.0);
  }
  D.has_row2 = false;
  D.sym_b_k = -1.0; D.sym_c_k = 1.0; D.asym_b_k = 1.0; D.asym_c_k = 1.0;
  D.neumann_identity = false; D.dirichlet_identity = false;
  D.dir_all_interior = true; D.neu_all_interior = true;
  return D;
}

FamilyDesc desc_m1p2c() {
  FamilyDesc D = desc_m1c2p();
  D.row1[0] = cl(0.0, 0.5, 0.5, 0.0);
  for (int n : {1, 2}) {
    const double q = (n == 1) ? 0.0 : 1.0;
    D.row1[n] = cl(q, (5.0 - q) / 16.0, (15.0 + 9.0 * q) / 16.0, (-5.0 + 9.0 * q) / 16.0, (1.0 - q) / 16.0);
  }
  {
    const double q = 7.0 / 3.0;
    D.row1[3] = cl(q, (63.0 - 7.0 * q) / 256.0, (315.0 + 105.0 * q) / 256.0, (-7.0 + 7.0 * q) * 15.0 / 128.0,
                   (63.0 - 35.0 * q) / 128.0, (-15.0 + 7.0 * q) * 3.0 / 256.0, (7.0 - 3.0 * q) / 256.0);
  }
  D.has_row2 = false;
  D.sym_b_k = 1.0; D.sym_c_k = 1.0; D.asym_b_k = -1.0; D.asym_c_k = 1.0;
  D.neumann_identity = false; D.dirichlet_identity = false;
  D.dir_all_interior = true; D.neu_all_interior = true;
  return D;
}

FamilyDesc desc_d1p2p() {
  FamilyDesc D = desc_d1c2c();
  D.sym_b_k = 0.0; D.sym_c_k = 0.0; D.asym_b_k = 0.0; D.asym_c_k = 2.0;
  D.neumann_identity = true;
  D.neu_all_interior = false;
  return D;
}

void set_row(CoefSet& s, int row, int bc, double a, double b, double c) {
  s.lhs[row][0][bc] = a; s.lhs[row][1][bc] = b; s.lhs[row][2][bc] = c;
}
void copy_row(CoefSet& dst, int row, int bcd, const CoefSet& src, int bcs, bool l, bool r) {
  if (l) for (int k = 0; k < 3; ++k) dst.lhs[row][k][bcd] = src.lhs[row][k][bcs];
  if (r) for (int k = 0; k < 6; ++k) dst.rhs[row][k][bcd] = src.rhs[row][k][bcs];
}

// assemble the table of one family at accuracy index m (0..3); cd4 is the same family at CD4
CoefSet assemble(const FamilyDesc& D, int m, bool p2c_interior_rows_only_periodic) {
  (void)p2c_interior_rows_only_periodic;
  CoefSet s;
  for (int r = 0; r < 5; ++r)
    for (int bc = 0; bc < 7; ++bc) {
      for (int k = 0; k < 3; ++k) s.lhs[r][k][bc] = kMaxp;
      for (int k = 0; k < 6; ++k) s.rhs[r][k][bc] = kMaxp;
    }
  auto periodic_rows = [&](CoefSet& t, int mm) {
    for (int r = 0; r < 5; ++r) {
      set_row(t, r, BC_PERIODIC, D.alpha[mm], 1.0, D.alpha[mm]);
      t.rhs[r][0][BC_PERIODIC] = D.ra[mm];
      t.rhs[r][1][BC_PERIODIC] = D.rb[mm];
      if (D.rb_zero_col3) t.rhs[r][2][BC_PERIODIC] = 0.0;
    }
  };
  periodic_rows(s, m);
  CoefSet cd4 = s;
  periodic_rows(cd4, ACC_CD4 - 1);
  const double al = D.alpha[m];
  // symmetric / antisymmetric ends: rows 1 and 5 modified, rows 2-4 and all RHS periodic
  for (int bc : {BC_SYMMETRIC, BC_ASYMMETRIC}) {
    for (int r = 0; r < 5; ++r) copy_row(s, r, bc, s, BC_PERIODIC, r >= 1 && r <= 3, true);
    double b1 = (bc == BC_SYMMETRIC) ? 1.0 + D.sym_b_k * al : 1.0 + D.asym_b_k * al;
    double c1 = (bc == BC_SYMMETRIC) ? D.sym_c_k * al : D.asym_c_k * al;
    set_row(s, 0, bc, 0.0, b1, c1);
    set_row(s, 4, bc, c1, b1, 0.0);
  }
  // interior: periodic rows, CD4 end rows for the compact schemes
  for (int r = 0; r < 5; ++r) copy_row(s, r, BC_INTERIOR, s, BC_PERIODIC, true, true);
  if (m == ACC_CP4 - 1 || m == ACC_CP6 - 1) {
    copy_row(s, 0, BC_INTERIOR, cd4, BC_PERIODIC, true, true);
    copy_row(s, 4, BC_INTERIOR, cd4, BC_PERIODIC, true, true);
  }
  // extrapolation closure
  {
    const Closure& c1 = D.row1[m];
    set_row(s, 0, BC_INTRPL, 0.0, 1.0, c1.alpha);
    set_row(s, 4, BC_INTRPL, c1.alpha, 1.0, 0.0);
    for (int k = 0; k < 6; ++k) { s.rhs[0][k][BC_INTRPL] = c1.c[k]; s.rhs[4][k][BC_INTRPL] = D.mirror * c1.c[k]; }
    if (D.has_row2) {
      const Closure& c2 = D.row2[m];
      set_row(s, 1, BC_INTRPL, c2.alpha, 1.0, c2.alpha);
      set_row(s, 3, BC_INTRPL, c2.alpha, 1.0, c2.alpha);
      for (int k = 0; k < 6; ++k) { s.rhs[1][k][BC_INTRPL] = c2.c[k]; s.rhs[3][k][BC_INTRPL] = D.mirror * c2.c[k]; }
      copy_row(s, 2, BC_INTRPL, s, BC_PERIODIC, true, true);
    } else {
      for (int r = 1; r <= 3; ++r) copy_row(s, r, BC_INTRPL, s, BC_PERIODIC, true, true);
    }
  }
  // Dirichlet / Neumann (ghost-cell treatment): interior rows, with identity end rows where the
  // boundary value itself is the result
  for (int r = 0; r < 5; ++r) {
    copy_row(s, r, BC_DIRICHLET, s, BC_INTERIOR, true, true);
    copy_row(s, r, BC_NEUMANN, s, BC_INTERIOR, true, true);
  }
  if (D.neumann_identity) {
    for (int r : {0, 4}) {
      set_row(s, r, BC_NEUMANN, 0.0, 1.0, 0.0);
      for (int k = 0; k < 6; ++k) s.rhs[r][k][BC_NEUMANN] = 0.0;
    }
  }
  if (D.dirichlet_identity) {
    for (int r : {0, 4}) {
      set_row(s, r, BC_DIRICHLET, 0.0, 1.0, 0.0);
      for (int k = 0; k < 6; ++k) s.rhs[r][k][BC_DIRICHLET] = 0.0;
    }
  }
  return s;
}

struct AllSets {
  CoefSet s[6][4];
  AllSets() {
    FamilyDesc d[6] = {desc_d1c2c(), desc_d1p2p(), desc_d1c2p(), desc_d1p2c(), desc_m1c2p(), desc_m1p2c()};
    for (int f = 0; f < 6; ++f)
      for (int m = 0; m < 4; ++m) s[f][m] = assemble(d[f], m, false);
  }
};

}  // namespace

const CoefSet& coef(int fam, int acc) {
  static const AllSets all;
  return all.s[fam][acc - 1];
}

// ---------------------------------------------------------------------------
// linear forms over the input line and the boundary values
// ---------------------------------------------------------------------------
namespace {

struct Lin {
  int n = 0;
  int idx[16];
  double w[16];
  double b[4] = {0, 0, 0, 0};
  bool valid = true;  // false for a ghost value the reference sets to MAXP
  void addf(int i, double c) {
    for (int t = 0; t < n; ++t)
      if (idx[t] == i) { w[t] += c; return; }
    if (n >= 16) throw std::runtime_error("linear form overflow");
    idx[n] = i; w[n] = c; ++n;
  }
  static Lin F(int i) { Lin l; l.addf(i, 1.0); return l; }
  static Lin B(int u) { Lin l; l.b[u] = 1.0; return l; }
  static Lin bad() { Lin l; l.valid = false; return l; }
};
Lin operator+(const Lin& x, const Lin& y) {
  Lin r = x;
  for (int t = 0; t < y.n; ++t) r.addf(y.idx[t], y.w[t]);
  for (int u = 0; u < 4; ++u) r.b[u] += y.b[u];
  r.valid = x.valid && y.valid;
  return r;
}
Lin operator*(double c, const Lin& x) {
  Lin r = x;
  for (int t = 0; t < r.n; ++t) r.w[t] *= c;
  for (int u = 0; u < 4; ++u) r.b[u] *= c;
  return r;
}
Lin operator-(const Lin& x, const Lin& y) { return x + (-1.0) * y; }
Lin operator-(const Lin& x) { return (-1.0) * x; }

// ghost values at the low end (g0 = cell/point 0, gm1 = -1) and high end (g1, g2)
struct Ghost { Lin lo0, lom1, hi1, hi2; };

// cell-centred input (buildup_ghost_cells_C, src/basics_operations2.f90:1805-1880); 1-based indices
Ghost ghost_c(int nc, const int ibc[2], const double dp[4]) {
  Ghost g;
  switch (ibc[0]) {
    case BC_INTERIOR: g.lo0 = Lin::B(0); g.lom1 = Lin::B(2); break;
    case BC_PERIODIC: g.lo0 = Lin::F(nc); g.lom1 = Lin::F(nc - 1); break;
    case BC_SYMMETRIC: g.lo0 = Lin::F(1); g.lom1 = Lin::F(2); break;
    case BC_ASYMMETRIC: g.lo0 = -Lin::F(1); g.lom1 = -Lin::F(2); break;
    case BC_DIRICHLET: g.lo0 = 2.0 * Lin::B(0) - Lin::F(1); g.lom1 = 2.0 * Lin::B(0) - Lin::F(2); break;
    case BC_NEUMANN: g.lo0 = Lin::F(1) - dp[0] * Lin::B(0); g.lom1 = Lin::F(2) - dp[2] * Lin::B(0); break;
    default: g.lo0 = Lin::bad(); g.lom1 = Lin::bad();
  }
  switch (ibc[1]) {
    case BC_INTERIOR: g.hi1 = Lin::B(1); g.hi2 = Lin::B(3); break;
    case BC_PERIODIC: g.hi1 = Lin::F(1); g.hi2 = Lin::F(2); break;
    case BC_SYMMETRIC: g.hi1 = Lin::F(nc); g.hi2 = Lin::F(nc - 1); break;
    case BC_ASYMMETRIC: g.hi1 = -Lin::F(nc); g.hi2 = -Lin::F(nc - 1); break;
    case BC_DIRICHLET: g.hi1 = 2.0 * Lin::B(1) - Lin::F(nc); g.hi2 = 2.0 * Lin::B(1) - Lin::F(nc - 1); break;
    case BC_NEUMANN: g.hi1 = Lin::F(nc) + dp[1] * Lin::B(1); g.hi2 = Lin::F(nc - 1) + dp[3] * Lin::B(1); break;
    default: g.hi1 = Lin::bad(); g.hi2 = Lin::bad();
  }
  return g;
}

// node input (buildup_ghost_cells_P, src/basics_operations2.f90:1883-1966)
Ghost ghost_p(int np, const int ibc[2], const double dp[4], bool has_fbc) {
  Ghost g;
  switch (ibc[0]) {
    case BC_INTERIOR: g.lo0 = Lin::B(0); g.lom1 = Lin::B(2); break;
    case BC_PERIODIC: g.lo0 = Lin::F(np); g.lom1 = Lin::F(np - 1); break;
    case BC_SYMMETRIC: g.lo0 = Lin::F(2); g.lom1 = Lin::F(3); break;
    case BC_ASYMMETRIC: g.lo0 = -Lin::F(2); g.lom1 = -Lin::F(3); break;
    case BC_DIRICHLET:
      if (has_fbc) { g.lo0 = 2.0 * Lin::B(0) - Lin::F(2); g.lom1 = 2.0 * Lin::B(0) - Lin::F(3); }
      else { g.lo0 = 2.0 * Lin::F(1) - Lin::F(2); g.lom1 = 2.0 * Lin::F(1) - Lin::F(3); }
      break;
    case BC_NEUMANN: g.lo0 = Lin::F(2) - dp[0] * Lin::B(0); g.lom1 = Lin::F(3) - dp[2] * Lin::B(0); break;
    default: g.lo0 = Lin::bad(); g.lom1 = Lin::bad();
  }
  switch (ibc[1]) {
    case BC_INTERIOR: g.hi1 = Lin::B(1); g.hi2 = Lin::B(3); break;
    case BC_PERIODIC: g.hi1 = Lin::F(1); g.hi2 = Lin::F(2); break;
    case BC_SYMMETRIC: g.hi1 = Lin::F(np - 1); g.hi2 = Lin::F(np - 2); break;
    case BC_ASYMMETRIC: g.hi1 = -Lin::F(np - 1); g.hi2 = -Lin::F(np - 2); break;
    case BC_NEUMANN: g.hi1 = Lin::F(np - 1) + dp[1] * Lin::B(1); g.hi2 = Lin::F(np - 2) + dp[3] * Lin::B(1); break;
    case BC_DIRICHLET:
      if (has_fbc) { g.hi1 = 2.0 * Lin::B(1) - Lin::F(np - 1); g.hi2 = 2.0 * Lin::B(1) - Lin::F(np - 2); }
      else { g.hi1 = 2.0 * Lin::F(np) - Lin::F(np - 1); g.hi2 = 2.0 * Lin::F(np) - Lin::F(np - 2); }
      break;
    default: g.hi1 = Lin::bad(); g.hi2 = Lin::bad();
  }
  return g;
}

inline bool one_of(int v, std::initializer_list<int> s) {
  for (int x : s) if (x == v) return true;
  return false;
}

// Sum_k r(row, k) * F(start + step*k), k = 0..5 (the extrapolation rows)
Lin extrap(const CoefSet& c, int row, int start, int step) {
  Lin l;
  for (int k = 0; k < 6; ++k) {
    double w = c.rhs[row][k][BC_INTRPL];
    if (w != 0.0) l.addf(start + step * k, w);
  }
  return l;
}

struct RowOut {
  int row;  // 1-based
  Lin lin;
};

// The RHS builders (src/basics_operations2.f90:1980-2705) as linear forms for the special rows.
// Returns the rows in the order the reference assigns them (later entries win).
std::vector<RowOut> special_rows(int fam, const CoefSet& c, int nin, int nout, const int ibc[2], bool has_fbc,
                                 const double dp[4], double dd) {
  std::vector<RowOut> rows;
  auto R = [&](int row, int k, int bc) { return c.rhs[row - 1][k - 1][bc]; };
  const int P = BC_PERIODIC;
  auto F = [](int i) { return Lin::F(i); };
  switch (fam) {
    case M1P2C: {  // Prepare_TDMA_interp_P2C_RHS_array
      const int nc = nout;
      Ghost g = ghost_p(nin, ibc, dp, has_fbc);
      bool bc1 = one_of(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
      bool bc5 = one_of(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
      int i = 1;
      if (bc1) rows.push_back({i, R(1, 1, ibc[0]) * (F(i) + F(i + 1)) + R(1, 2, ibc[0]) * (g.lo0 + F(i + 2))});
      else rows.push_back({i, extrap(c, 0, i, 1)});
      i = nc;
      if (bc5) rows.push_back({i, R(5, 1, ibc[1]) * (F(i) + F(i + 1)) + R(5, 2, ibc[1]) * (F(i - 1) + g.hi1)});
      else if (ibc[1] == P) rows.push_back({i, R(5, 1, P) * (F(i) + g.hi1) + R(5, 2, P) * (F(i - 1) + g.hi2)});
      else rows.push_back({i, extrap(c, 4, i + 1, -1)});
      i = nc - 1;
      if (ibc[1] == P) rows.push_back({i, R(4, 1, P) * (F(i) + F(i + 1)) + R(4, 2, P) * (F(i - 1) + g.hi1)});
      else rows.push_back({i, R(4, 1, ibc[1]) * (F(i) + F(i + 1)) + R(4, 2, ibc[1]) * (F(i - 1) + F(i + 2))});
      break;
    }
    case M1C2P: {  // Prepare_TDMA_interp_C2P_RHS_array
      const int np = nout;
      Ghost g = ghost_c(nin, ibc, dp);
      bool bc1 = one_of(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_NEUMANN});
      bool bc5 = one_of(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_NEUMANN});
      bool bc2 = bc1 || ibc[0] == BC_DIRICHLET;
      bool bc4 = bc5 || ibc[1] == BC_DIRICHLET;
      int i = 1;
      if (bc1) rows.push_back({i, R(1, 1, ibc[0]) * (F(i) + g.lo0) + R(1, 2, ibc[0]) * (F(i + 1) + g.lom1)});
      else if (ibc[0] == BC_DIRICHLET) rows.push_back({i, Lin::B(0)});
      else rows.push_back({i, extrap(c, 0, i, 1)});
      i = 2;
      if (bc2) rows.push_back({i, R(2, 1, ibc[0]) * (F(i) + F(i - 1)) + R(2, 2, ibc[0]) * (F(i + 1) + g.lo0)});
      else rows.push_back({i, extrap(c, 1, i - 1, 1)});
      i = np;
      if (bc5) rows.push_back({i, R(5, 1, ibc[1]) * (g.hi1 + F(i - 1)) + R(5, 2, ibc[1]) * (g.hi2 + F(i - 2))});
      else if (ibc[1] == P) rows.push_back({i, R(5, 1, P) * (F(i) + F(i - 1)) + R(5, 2, P) * (g.hi1 + F(i - 2))});
      else if (ibc[1] == BC_DIRICHLET) rows.push_back({i, Lin::B(1)});
      else rows.push_back({i, extrap(c, 4, i - 1, -1)});
      i = np - 1;
      if (bc4) rows.push_back({i, R(4, 1, ibc[1]) * (F(i) + F(i - 1)) + R(4, 2, ibc[1]) * (g.hi1 + F(i - 2))});
      else if (ibc[1] == P) rows.push_back({i, R(4, 1, P) * (F(i) + F(i - 1)) + R(4, 2, P) * (F(i + 1) + F(i - 2))});
      else rows.push_back({i, extrap(c, 3, i, -1)});
      break;
    }
    case D1C2C: {  // Prepare_TDMA_1deri_C2C_RHS_array
      const int nc = nout;
      Ghost g = ghost_c(nin, ibc, dp);
      bool b[2];
      for (int k = 0; k < 2; ++k)
        b[k] = one_of(ibc[k], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
      int i = 1;
      if (b[0]) rows.push_back({i, R(1, 1, ibc[0]) * (F(i + 1) - g.lo0) + R(1, 2, ibc[0]) * (F(i + 2) - g.lom1)});
      else rows.push_back({i, extrap(c, 0, i, 1)});
      i = 2;
      if (b[0]) rows.push_back({i, R(2, 1, ibc[0]) * (F(i + 1) - F(i - 1)) + R(2, 2, ibc[0]) * (F(i + 2) - g.lo0)});
      else rows.push_back({i, extrap(c, 1, i - 1, 1)});
      i = nc;
      if (b[1]) rows.push_back({i, R(5, 1, ibc[1]) * (g.hi1 - F(i - 1)) + R(5, 2, ibc[1]) * (g.hi2 - F(i - 2))});
      else rows.push_back({i, extrap(c, 4, i, -1)});
      i = nc - 1;
      if (b[1]) rows.push_back({i, R(4, 1, ibc[1]) * (F(i + 1) - F(i - 1)) + R(4, 2, ibc[1]) * (g.hi1 - F(i - 2))});
      else rows.push_back({i, extrap(c, 3, i + 1, -1)});
      break;
    }
    case D1P2P: {  // Prepare_TDMA_1deri_P2P_RHS_array
      const int np = nout;
      Ghost g = ghost_p(nin, ibc, dp, has_fbc);
      bool b1[2], b2[2];
      for (int k = 0; k < 2; ++k) {
        b1[k] = one_of(ibc[k], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET});
        b2[k] = b1[k] || ibc[k] == BC_NEUMANN;
      }
      int i = 1;
      if (b1[0]) rows.push_back({i, R(1, 1, ibc[0]) * (F(i + 1) - g.lo0) + R(1, 2, ibc[0]) * (F(i + 2) - g.lom1)});
      else if (ibc[0] == BC_NEUMANN) rows.push_back({i, (1.0 / dd) * Lin::B(0)});
      else rows.push_back({i, extrap(c, 0, i, 1)});
      i = 2;
      if (b2[0]) rows.push_back({i, R(2, 1, ibc[0]) * (F(i + 1) - F(i - 1)) + R(2, 2, ibc[0]) * (F(i + 2) - g.lo0)});
      else rows.push_back({i, extrap(c, 1, i - 1, 1)});
      i = np;
      if (b1[1]) rows.push_back({i, R(5, 1, ibc[1]) * (g.hi1 - F(i - 1)) + R(5, 2, ibc[1]) * (g.hi2 - F(i - 2))});
      else if (ibc[1] == BC_NEUMANN) rows.push_back({i, (1.0 / dd) * Lin::B(1)});
      else rows.push_back({i, extrap(c, 4, i, -1)});
      i = np - 1;
      if (b2[1]) rows.push_back({i, R(4, 1, ibc[1]) * (F(i + 1) - F(i - 1)) + R(4, 2, ibc[1]) * (g.hi1 - F(i - 2))});
      else rows.push_back({i, extrap(c, 3, i + 1, -1)});
      break;
    }
    case D1C2P: {  // Prepare_TDMA_1deri_C2P_RHS_array (is_bc4 reads ibc(1), as in the reference)
      const int np = nout;
      Ghost g = ghost_c(nin, ibc, dp);
      bool bc1 = one_of(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET});
      bool bc2 = bc1 || ibc[0] == BC_NEUMANN;
      bool bc5 = one_of(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET});
      bool bc4 = bc5 || ibc[0] == BC_DIRICHLET || ibc[0] == BC_NEUMANN;
      int i = 1;
      if (bc1) rows.push_back({i, R(1, 1, ibc[0]) * (F(i) - g.lo0) + R(1, 2, ibc[0]) * (F(i + 1) - g.lom1)});
      else if (ibc[0] == BC_NEUMANN) rows.push_back({i, (1.0 / dd) * Lin::B(0)});
      else rows.push_back({i, extrap(c, 0, i, 1)});
      i = 2;
      if (bc2) rows.push_back({i, R(2, 1, ibc[0]) * (F(i) - F(i - 1)) + R(2, 2, ibc[0]) * (F(i + 1) - g.lo0)});
      else rows.push_back({i, extrap(c, 1, i - 1, 1)});
      i = np;
      if (bc5) rows.push_back({i, R(5, 1, ibc[1]) * (g.hi1 - F(i - 1)) + R(5, 2, ibc[1]) * (g.hi2 - F(i - 2))});
      else if (ibc[1] == P) rows.push_back({i, R(5, 1, P) * (F(i) - F(i - 1)) + R(5, 2, P) * (g.hi1 - F(i - 2))});
      else if (ibc[1] == BC_NEUMANN) rows.push_back({i, (1.0 / dd) * Lin::B(1)});
      else rows.push_back({i, extrap(c, 4, i - 1, -1)});
      i = np - 1;
      if (bc4) rows.push_back({i, R(4, 1, ibc[1]) * (F(i) - F(i - 1)) + R(4, 2, ibc[1]) * (g.hi1 - F(i - 2))});
      else if (ibc[1] == P) rows.push_back({i, R(4, 1, P) * (F(i) - F(i - 1)) + R(4, 2, P) * (F(i + 1) - F(i - 2))});
      else rows.push_back({i, extrap(c, 3, i, -1)});
      break;
    }
    case D1P2C: {  // Prepare_TDMA_1deri_P2C_RHS_array
      const int nc = nout;
      Ghost g = ghost_p(nin, ibc, dp, has_fbc);
      bool bc1 = one_of(ibc[0], {BC_INTERIOR, BC_PERIODIC, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
      bool bc5 = one_of(ibc[1], {BC_INTERIOR, BC_SYMMETRIC, BC_ASYMMETRIC, BC_DIRICHLET, BC_NEUMANN});
      int i = 1;
      if (bc1) rows.push_back({i, R(1, 1, ibc[0]) * (F(i + 1) - F(i)) + R(1, 2, ibc[0]) * (F(i + 2) - g.lo0)});
      else rows.push_back({i, extrap(c, 0, i, 1)});
      i = nc;
      if (bc5) rows.push_back({i, R(5, 1, ibc[1]) * (F(i + 1) - F(i)) + R(5, 2, ibc[1]) * (g.hi1 - F(i - 1))});
      else if (ibc[1] == P) rows.push_back({i, R(5, 1, P) * (g.hi1 - F(i)) + R(5, 2, P) * (g.hi2 - F(i - 1))});
      else rows.push_back({i, extrap(c, 4, i + 1, -1)});
      i = nc - 1;
      if (ibc[1] == P) rows.push_back({i, R(4, 1, P) * (F(i + 1) - F(i)) + R(4, 2, P) * (g.hi1 - F(i - 1))});
      else rows.push_back({i, R(4, 1, P) * (F(i + 1) - F(i)) + R(4, 2, P) * (F(i + 2) - F(i - 1))});
      break;
    }
    default: throw std::runtime_error("unknown operator family");
  }
  return rows;
}

// Thomas pre-factorisation (Preprocess_TDMA_coeffs, src/basics_algorithms.f90:14-34)
void prefactor(const std::vector<double>& a, const std::vector<double>& b, std::vector<double>& c,
               std::vector<double>& d, int n) {
  c[0] = c[0] / b[0];
  for (int i = 1; i < n; ++i) {
    d[i] = 1.0 / (b[i] - a[i] * c[i - 1]);
    if (i < n - 1) c[i] = c[i] * d[i];
  }
}
void thomas(std::vector<double>& x, const std::vector<double>& a, const std::vector<double>& b,
            const std::vector<double>& c, const std::vector<double>& d, int n) {
  x[0] = x[0] / b[0];
  for (int i = 1; i < n; ++i) x[i] = (x[i] - a[i] * x[i - 1]) * d[i];
  for (int i = n - 2; i >= 0; --i) x[i] = x[i] - c[i] * x[i + 1];
}

}  // namespace

void reduce_bc(int fam, const int ibc0[2], bool has_fbc, int ibc[2]) {
  for (int k = 0; k < 2; ++k) {
    ibc[k] = ibc0[k];
    if (has_fbc) continue;
    if (ibc[k] == BC_INTERIOR || ibc[k] == BC_NEUMANN) ibc[k] = BC_INTRPL;
    if (ibc[k] == BC_DIRICHLET && fam_c_input(fam)) ibc[k] = BC_INTRPL;
  }
}

int64_t PlanBook::add_array(const std::vector<double>& v) {
  // keep every array 32-byte aligned inside the table
  while (table.size() % 4) table.push_back(0.0);
  int64_t off = (int64_t)table.size();
  table.insert(table.end(), v.begin(), v.end());
  return off;
}

const PlanBook::LhsKey& PlanBook::lhs(int fam, int n, int bc1, int bc2) {
  for (const auto& k : lhs_)
    if (k.fam == fam && k.n == n && k.b1 == bc1 && k.b2 == bc2) return k;
  const CoefSet& c = coef(fam, iacc);
  std::vector<double> a(n), b(n), cc(n), d(n, 0.0);
  for (int col = 0; col < 3; ++col) {
    std::vector<double>& v = col == 0 ? a : (col == 1 ? b : cc);
    v[0] = c.lhs[0][col][bc1];
    v[1] = c.lhs[1][col][bc1];
    for (int i = 2; i <= n - 3; ++i) v[i] = c.lhs[2][col][BC_PERIODIC];
    v[n - 2] = c.lhs[3][col][bc2];
    v[n - 1] = c.lhs[4][col][bc2];
  }
  LhsKey k{};
  k.fam = fam; k.n = n; k.b1 = bc1; k.b2 = bc2;
  const bool cyc = (bc1 == BC_PERIODIC && bc2 == BC_PERIODIC);
  prefactor(a, b, cc, d, cyc ? n - 1 : n);
  k.b1v = b[0];
  std::vector<double> x1(n, 0.0);
  if (cyc) {
    // cyclic correction vector: solve the (n-1) system for [-a(1), 0, ..., -c(n-1)]
    // (Solve_TDMA_cyclic, src/basics_algorithms.f90:68-90)
    x1[0] = -a[0];
    x1[n - 2] = -cc[n - 2];
    thomas(x1, a, b, cc, d, n - 1);
    k.an = a[n - 1];
    k.cn = cc[n - 1];
    k.inv_den = 1.0 / (b[n - 1] + cc[n - 1] * x1[0] + a[n - 1] * x1[n - 2]);
  }
  k.la = add_array(a);
  k.lc = add_array(cc);
  k.ld = add_array(d);
  k.lx1 = add_array(x1);
  lhs_.push_back(k);
  return lhs_.back();
}

OpPlan PlanBook::make(int d, int fam, const int ibc0[2], bool has_fbc) {
  const DirGeom& G = dir[d];
  OpPlan p;
  std::memset(&p, 0, sizeof(p));
  p.fam = fam;
  p.nin = (fam == D1P2P || fam == D1P2C || fam == M1P2C) ? G.np : G.nc;
  p.nout = fam_p_output(fam) ? G.np : G.nc;
  if (p.nin < 8 || p.nout < 8) throw std::runtime_error("line operators need at least 8 points");
  int ibc[2];
  reduce_bc(fam, ibc0, has_fbc, ibc);
  const CoefSet& c = coef(fam, iacc);
  const double dd = fam_deriv(fam) ? G.dd : 1.0;
  p.dd = dd;
  p.r1 = c.rhs[2][0][BC_PERIODIC];
  p.r2 = c.rhs[2][1][BC_PERIODIC];
  int b_lo1 = 3;  // 1-based first bulk row
  switch (fam) {
    case M1P2C: p.off[0] = 0; p.off[1] = 1; p.off[2] = -1; p.off[3] = 2; p.sgn = 1.0; b_lo1 = 2; break;
    case M1C2P: p.off[0] = 0; p.off[1] = -1; p.off[2] = 1; p.off[3] = -2; p.sgn = 1.0; b_lo1 = 3; break;
    case D1C2C:
    case D1P2P: p.off[0] = 1; p.off[1] = -1; p.off[2] = 2; p.off[3] = -2; p.sgn = -1.0; b_lo1 = 3; break;
    case D1C2P: p.off[0] = 0; p.off[1] = -1; p.off[2] = 1; p.off[3] = -2; p.sgn = -1.0; b_lo1 = 3; break;
    case D1P2C: p.off[0] = 1; p.off[1] = 0; p.off[2] = 2; p.off[3] = -1; p.sgn = -1.0; b_lo1 = 2; break;
  }
  p.b_lo = b_lo1 - 1;
  p.b_hi = p.nout - 3;  // rows up to n-2 (1-based)
  const double* dp = fam_c_input(fam) ? G.dp_c : G.dp_p;
  auto rows = special_rows(fam, c, p.nin, p.nout, ibc, has_fbc, dp, dd);
  // collapse to at most 4 distinct rows, later assignments win
  p.nspec = 0;
  for (const auto& r : rows) {
    if (!r.lin.valid) throw std::runtime_error("boundary row reads an undefined ghost value");
    int slot = -1;
    for (int s = 0; s < p.nspec; ++s)
      if (p.sp[s].row == r.row - 1) slot = s;
    if (slot < 0) {
      if (p.nspec >= 4) throw std::runtime_error("too many boundary rows");
      slot = p.nspec++;
    }
    SpecialRow& S = p.sp[slot];
    S.row = r.row - 1;
    S.nt = 0;
    for (int t = 0; t < r.lin.n; ++t) {
      if (r.lin.w[t] == 0.0) continue;
      int idx = r.lin.idx[t] - 1;
      if (idx < 0 || idx >= p.nin) throw std::runtime_error("boundary row index out of range");
      if (S.nt >= kMaxTerms) throw std::runtime_error("boundary row has too many terms");
      S.idx[S.nt] = idx;
      S.w[S.nt] = r.lin.w[t];
      ++S.nt;
    }
    for (int u = 0; u < 4; ++u) {
      S.wb[u] = r.lin.b[u];
      if (S.wb[u] != 0.0) p.needs_fbc = 1;
    }
  }
  if (p.needs_fbc && !has_fbc) throw std::runtime_error("plan reads boundary values that were not supplied");
  // Thomas solve only for the compact schemes (src/basics_operations2.f90:2780-2792)
  p.tdma = 0;
  p.la = p.lc = p.ld = p.lx1 = -1;
  if (iacc == ACC_CP4 || iacc == ACC_CP6) {
    const LhsKey& k = lhs(fam, p.nout, ibc[0], ibc[1]);
    p.tdma = (ibc[0] == BC_PERIODIC) ? 2 : 1;
    if (p.tdma == 2 && ibc[1] != BC_PERIODIC) throw std::runtime_error("mixed periodic ends are not supported");
    p.b1 = k.b1v; p.an = k.an; p.cn = k.cn; p.inv_den = k.inv_den;
    p.la = k.la; p.lc = k.lc; p.ld = k.ld; p.lx1 = k.lx1;
  }
  // y: stretching metric and Neumann overrides (src/basics_operations2.f90:3474-3704)
  p.lmap = -1;
  p.neu1 = p.neu2 = 0;
  if (d == 1 && fam_deriv(fam)) {
    p.lmap = (fam == D1C2C || fam == D1P2C) ? G.map_cc : G.map_pt;
    if ((fam == D1P2P || fam == D1C2P) && has_fbc) {
      p.neu1 = ibc[0] == BC_NEUMANN;
      p.neu2 = ibc[1] == BC_NEUMANN;
      if (p.neu1 || p.neu2) p.needs_fbc = 1;
    }
  }
  // A periodic explicit line whose boundary rows equal the bulk stencil with wrapped indices runs
  // every row through the bulk formula (no per-row branches in the kernels).  The check compares
  // the assembled boundary rows with the kernels' bulk formula term by term.
  p.wrap = 0;
  if (p.tdma == 0 && ibc[0] == BC_PERIODIC && ibc[1] == BC_PERIODIC && p.nin == p.nout && p.lmap < 0 && !p.neu1 &&
      !p.neu2) {
    int o[4];
    double cf[4];
    const double r1 = p.r1, r2 = p.r2;
    switch (fam) {
      case M1P2C: o[0] = 0; o[1] = 1; o[2] = -1; o[3] = 2; cf[0] = r1; cf[1] = r1; cf[2] = r2; cf[3] = r2; break;
      case M1C2P: o[0] = 0; o[1] = -1; o[2] = 1; o[3] = -2; cf[0] = r1; cf[1] = r1; cf[2] = r2; cf[3] = r2; break;
      case D1C2C:
      case D1P2P: o[0] = 1; o[1] = -1; o[2] = 2; o[3] = -2; cf[0] = r1; cf[1] = -r1; cf[2] = r2; cf[3] = -r2; break;
      case D1C2P: o[0] = 0; o[1] = -1; o[2] = 1; o[3] = -2; cf[0] = r1; cf[1] = -r1; cf[2] = r2; cf[3] = -r2; break;
      default: o[0] = 1; o[1] = 0; o[2] = 2; o[3] = -1; cf[0] = r1; cf[1] = -r1; cf[2] = r2; cf[3] = -r2; break;
    }
    const int n = p.nin;
    const double tol = 1e-13 * (std::fabs(r1) + std::fabs(r2));
    bool ok = true;
    int covered = 0;
    for (int s = 0; s < p.nspec && ok; ++s) {
      const SpecialRow& S = p.sp[s];
      for (int u = 0; u < 4; ++u)
        if (S.wb[u] != 0.0) ok = false;
      std::vector<double> want(n, 0.0), have(n, 0.0);
      for (int k = 0; k < 4; ++k) want[((S.row + o[k]) % n + n) % n] += cf[k];
      for (int t = 0; t < S.nt; ++t) have[S.idx[t]] += S.w[t];
      for (int i = 0; i < n && ok; ++i)
        if (std::fabs(want[i] - have[i]) > tol) ok = false;
      if (S.row < p.b_lo || S.row > p.b_hi) ++covered;
    }
    if (ok && covered == p.b_lo + (p.nout - 1 - p.b_hi)) p.wrap = 1;
  }
  return p;
}

}  // namespace chs
