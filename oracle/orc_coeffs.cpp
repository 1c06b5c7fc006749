// ORACLE (test infrastructure only; never linked into the product library).
//
// CPU FP64 restatement of CHAPSim2's compact finite-difference coefficient
// tables and TDMA routines.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py may load this code, and only as a
// checker or as the timed CPU baseline.
//
// Parity status: pinned by the reference's own known answers -- the TDMA
// vectors of src/basics_algorithms.f90:111-188 and the analytic sin-function
// operator tests of src/basics_operations2.f90:4806-5357 (convergence orders).
// The reference solver itself cannot be built here (it is Fortran + MPI and
// no Fortran compiler exists in this image), so bit-level parity against the
// running reference is not available.
#include "orc.h"

#include <cmath>
#include <cstring>

namespace orc {

// ---------------------------------------------------------------------------
// Coefficient tables, restating Prepare_compact_coefficients
// (src/basics_operations2.f90:361-1528).  Indices follow the Fortran tables:
// row l = 1..5, column s = 1..3 (LHS) or 1..6 (RHS), bc = 0..6, acc = 1..4.
// Entries that the reference leaves at MAXP stay at MAXP.
// ---------------------------------------------------------------------------
static void fill_maxp(Family& t) {
  for (int l = 0; l < NL; ++l)
    for (int bc = 0; bc < NBC; ++bc)
      for (int a = 0; a < NACC; ++a) {
        for (int s = 0; s < 3; ++s) t.f[l][s][bc][a] = MAXP;
        for (int s = 0; s < 6; ++s) t.r[l][s][bc][a] = MAXP;
      }
}

static inline double& F(Family& t, int l, int s, int bc, int n) { return t.f[l - 1][s - 1][bc][n - 1]; }
static inline double& R(Family& t, int l, int s, int bc, int n) { return t.r[l - 1][s - 1][bc][n - 1]; }

// copy rows lo..hi (all columns) of bc `src` (accuracy ns) into bc `dst` (accuracy nd)
static void copy_rows(Family& t, int lo, int hi, int dst, int nd, int src, int ns, bool lhs, bool rhs) {
  for (int l = lo; l <= hi; ++l) {
    if (lhs) for (int s = 1; s <= 3; ++s) F(t, l, s, dst, nd) = F(t, l, s, src, ns);
    if (rhs) for (int s = 1; s <= 6; ++s) R(t, l, s, dst, nd) = R(t, l, s, src, ns);
  }
}

// mirror row 1 into row 5 (LHS only): f5 = (f1_3, f1_2, f1_1)
static void mirror_lhs(Family& t, int bc, int n, int from, int to) {
  double a = F(t, from, 1, bc, n), b = F(t, from, 2, bc, n), c = F(t, from, 3, bc, n);
  F(t, to, 1, bc, n) = c;
  F(t, to, 2, bc, n) = b;
  F(t, to, 3, bc, n) = a;
}

static void set_lhs(Family& t, int l, int bc, int n, double a, double b, double c) {
  F(t, l, 1, bc, n) = a;
  F(t, l, 2, bc, n) = b;
  F(t, l, 3, bc, n) = c;
}

static void set_rhs6(Family& t, int l, int bc, int n, const double v[6]) {
  for (int s = 1; s <= 6; ++s) R(t, l, s, bc, n) = v[s - 1];
}

// interior closure for CP4/CP6: rows 1 and 5 take the CD4 periodic rows
static void interior_from_periodic(Family& t) {
  copy_rows(t, 1, 5, BC_INTERIOR, 1, BC_PERIODIC, 1, true, true);
  for (int n = 1; n <= NACC; ++n) copy_rows(t, 1, 5, BC_INTERIOR, n, BC_PERIODIC, n, true, true);
  for (int n = 1; n <= NACC; ++n) {
    if (n == ACC_CP4 || n == ACC_CP6) {
      copy_rows(t, 1, 1, BC_INTERIOR, n, BC_PERIODIC, ACC_CD4, true, true);
      copy_rows(t, 5, 5, BC_INTERIOR, n, BC_PERIODIC, ACC_CD4, true, true);
    }
  }
}

void build_tables(Tables& T) {
  double alpha[5], a[5], b[5], c[5];
  double al1[5], a1[5], b1[5], c1[5], d1[5], e1[5], f1[5];
  double al2[5], a2[5], b2[5], c2[5], d2[5], e2[5], f2[5];
  auto zero5 = [](double* v) { for (int i = 0; i < 5; ++i) v[i] = 0.0; };

  for (int k = 0; k < NFAM; ++k) fill_maxp(T.fam[k]);
  Family& C2C = T.fam[FAM_D1C2C];
  Family& P2P = T.fam[FAM_D1P2P];
  Family& C2P = T.fam[FAM_D1C2P];
  Family& P2C = T.fam[FAM_D1P2C];
  Family& M2P = T.fam[FAM_M1C2P];
  Family& M2C = T.fam[FAM_M1P2C];

  // ---------------- 1st derivative, C2C (basics_operations2.f90:403-599)
  zero5(alpha); zero5(a); zero5(b); zero5(c);
  alpha[ACC_CD2] = 0.0;        a[ACC_CD2] = 1.0;         b[ACC_CD2] = 0.0;
  alpha[ACC_CD4] = 0.0;        a[ACC_CD4] = 4.0 / 3.0;   b[ACC_CD4] = -1.0 / 3.0;
  alpha[ACC_CP4] = 1.0 / 4.0;  a[ACC_CP4] = 3.0 / 2.0;   b[ACC_CP4] = 0.0;
  alpha[ACC_CP6] = 1.0 / 3.0;  a[ACC_CP6] = 14.0 / 9.0;  b[ACC_CP6] = 1.0 / 9.0;
  for (int n = 1; n <= NACC; ++n)
    for (int l = 1; l <= 5; ++l) {
      set_lhs(C2C, l, BC_PERIODIC, n, alpha[n], 1.0, alpha[n]);
      R(C2C, l, 1, BC_PERIODIC, n) = a[n] * 0.5;
      R(C2C, l, 2, BC_PERIODIC, n) = b[n] * 0.25;
    }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(C2C, 1, BC_SYMMETRIC, n, 0.0, 1.0 - alpha[n], alpha[n]);
    mirror_lhs(C2C, BC_SYMMETRIC, n, 1, 5);
    copy_rows(C2C, 2, 4, BC_SYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(C2C, 1, 5, BC_SYMMETRIC, n, BC_PERIODIC, n, false, true);
    set_lhs(C2C, 1, BC_ASYMMETRIC, n, 0.0, 1.0 + alpha[n], alpha[n]);
    mirror_lhs(C2C, BC_ASYMMETRIC, n, 1, 5);
    copy_rows(C2C, 2, 4, BC_ASYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(C2C, 1, 5, BC_ASYMMETRIC, n, BC_PERIODIC, n, false, true);
  }
  interior_from_periodic(C2C);
  zero5(al1); zero5(a1); zero5(b1); zero5(c1); zero5(d1); zero5(e1); zero5(f1);
  al1[ACC_CD2] = 0.0; a1[ACC_CD2] = -3.0 / 2.0; b1[ACC_CD2] = 2.0; c1[ACC_CD2] = -1.0 / 2.0;
  al1[ACC_CD4] = 0.0; a1[ACC_CD4] = -25.0 / 12.0; b1[ACC_CD4] = 4.0; c1[ACC_CD4] = -3.0;
  d1[ACC_CD4] = 4.0 / 3.0; e1[ACC_CD4] = -1.0 / 4.0;
  al1[ACC_CP4] = 3.0; a1[ACC_CP4] = -17.0 / 6.0; b1[ACC_CP4] = 3.0 / 2.0; c1[ACC_CP4] = 3.0 / 2.0;
  d1[ACC_CP4] = -1.0 / 6.0;
  al1[ACC_CP6] = 5.0; a1[ACC_CP6] = -197.0 / 60.0; b1[ACC_CP6] = -5.0 / 12.0; c1[ACC_CP6] = 5.0;
  d1[ACC_CP6] = -5.0 / 3.0; e1[ACC_CP6] = 5.0 / 12.0; f1[ACC_CP6] = -1.0 / 20.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(C2C, 1, BC_INTRPL, n, 0.0, 1.0, al1[n]);
    double v[6] = {a1[n], b1[n], c1[n], d1[n], e1[n], f1[n]};
    set_rhs6(C2C, 1, BC_INTRPL, n, v);
    mirror_lhs(C2C, BC_INTRPL, n, 1, 5);
    for (int s = 1; s <= 6; ++s) R(C2C, 5, s, BC_INTRPL, n) = -R(C2C, 1, s, BC_INTRPL, n);
  }
  for (int n = 1; n <= NACC; ++n) copy_rows(C2C, 3, 3, BC_INTRPL, n, BC_PERIODIC, n, true, true);
  zero5(al2); zero5(a2); zero5(b2); zero5(c2); zero5(d2); zero5(e2); zero5(f2);
  al2[ACC_CD2] = 0.0; a2[ACC_CD2] = -1.0 / 2.0; b2[ACC_CD2] = 0.0; c2[ACC_CD2] = 1.0 / 2.0;
  al2[ACC_CD4] = 0.0; a2[ACC_CD4] = -1.0 / 4.0; b2[ACC_CD4] = -5.0 / 6.0; c2[ACC_CD4] = 3.0 / 2.0;
  d2[ACC_CD4] = -1.0 / 2.0; e2[ACC_CD4] = 1.0 / 12.0;
  al2[ACC_CP4] = 1.0 / 4.0; a2[ACC_CP4] = -3.0 / 4.0; b2[ACC_CP4] = 0.0; c2[ACC_CP4] = 3.0 / 4.0;
  al2[ACC_CP6] = 2.0 / 11.0; a2[ACC_CP6] = -20.0 / 33.0; b2[ACC_CP6] = -35.0 / 132.0;
  c2[ACC_CP6] = 34.0 / 33.0; d2[ACC_CP6] = -7.0 / 33.0; e2[ACC_CP6] = 2.0 / 33.0;
  f2[ACC_CP6] = -1.0 / 132.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(C2C, 2, BC_INTRPL, n, al2[n], 1.0, al2[n]);
    double v[6] = {a2[n], b2[n], c2[n], d2[n], e2[n], f2[n]};
    set_rhs6(C2C, 2, BC_INTRPL, n, v);
    mirror_lhs(C2C, BC_INTRPL, n, 2, 4);
    for (int s = 1; s <= 6; ++s) R(C2C, 4, s, BC_INTRPL, n) = -R(C2C, 2, s, BC_INTRPL, n);
  }
  // bc_ghost_cd = .true. (basics_operations2.f90:33): Dirichlet/Neumann use the interior rows
  for (int n = 1; n <= NACC; ++n) {
    copy_rows(C2C, 1, 5, BC_DIRICHLET, n, BC_INTERIOR, n, true, true);
    copy_rows(C2C, 1, 5, BC_NEUMANN, n, BC_INTERIOR, n, true, true);
  }

  // ---------------- 1st derivative, P2P (basics_operations2.f90:612-710)
  for (int n = 1; n <= NACC; ++n) copy_rows(P2P, 1, 5, BC_PERIODIC, n, BC_PERIODIC, n, true, true);
  for (int n = 1; n <= NACC; ++n) {
    copy_rows(P2P, 1, 5, BC_PERIODIC, n, BC_PERIODIC, n, false, false);
    for (int l = 1; l <= 5; ++l) {
      for (int s = 1; s <= 3; ++s) F(P2P, l, s, BC_PERIODIC, n) = F(C2C, l, s, BC_PERIODIC, n);
      for (int s = 1; s <= 6; ++s) R(P2P, l, s, BC_PERIODIC, n) = R(C2C, l, s, BC_PERIODIC, n);
    }
  }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(P2P, 1, BC_SYMMETRIC, n, 0.0, 1.0, 0.0);
    mirror_lhs(P2P, BC_SYMMETRIC, n, 1, 5);
    copy_rows(P2P, 2, 4, BC_SYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(P2P, 1, 5, BC_SYMMETRIC, n, BC_PERIODIC, n, false, true);
    set_lhs(P2P, 1, BC_ASYMMETRIC, n, 0.0, 1.0, 2.0 * alpha[n]);
    mirror_lhs(P2P, BC_ASYMMETRIC, n, 1, 5);
    copy_rows(P2P, 2, 4, BC_ASYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(P2P, 1, 5, BC_ASYMMETRIC, n, BC_PERIODIC, n, false, true);
  }
  interior_from_periodic(P2P);
  for (int n = 1; n <= NACC; ++n) copy_rows(P2P, 1, 5, BC_INTRPL, n, BC_INTRPL, n, false, false);
  for (int n = 1; n <= NACC; ++n)
    for (int l = 1; l <= 5; ++l) {
      for (int s = 1; s <= 3; ++s) F(P2P, l, s, BC_INTRPL, n) = F(C2C, l, s, BC_INTRPL, n);
      for (int s = 1; s <= 6; ++s) R(P2P, l, s, BC_INTRPL, n) = R(C2C, l, s, BC_INTRPL, n);
    }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(P2P, 1, BC_NEUMANN, n, 0.0, 1.0, 0.0);
    for (int s = 1; s <= 6; ++s) R(P2P, 1, s, BC_NEUMANN, n) = 0.0;
    set_lhs(P2P, 5, BC_NEUMANN, n, 0.0, 1.0, 0.0);
    for (int s = 1; s <= 6; ++s) R(P2P, 5, s, BC_NEUMANN, n) = 0.0;
  }
  for (int n = 1; n <= NACC; ++n) {
    copy_rows(P2P, 1, 5, BC_DIRICHLET, n, BC_INTERIOR, n, true, true);
    copy_rows(P2P, 2, 4, BC_NEUMANN, n, BC_INTERIOR, n, true, true);
  }

  // ---------------- 1st derivative, C2P (basics_operations2.f90:722-945)
  zero5(alpha); zero5(a); zero5(b); zero5(c);
  alpha[ACC_CD2] = 0.0; a[ACC_CD2] = 1.0; b[ACC_CD2] = 0.0;
  alpha[ACC_CD4] = 0.0;
  a[ACC_CD4] = (9.0 - 6.0 * alpha[ACC_CD4]) / 8.0;
  b[ACC_CD4] = (-1.0 + 22.0 * alpha[ACC_CD4]) / 8.0;
  alpha[ACC_CP4] = 1.0 / 22.0;
  a[ACC_CP4] = (9.0 - 6.0 * alpha[ACC_CP4]) / 8.0;
  b[ACC_CP4] = (-1.0 + 22.0 * alpha[ACC_CP4]) / 8.0;
  alpha[ACC_CP6] = 9.0 / 62.0; a[ACC_CP6] = 63.0 / 62.0; b[ACC_CP6] = 17.0 / 62.0;
  for (int n = 1; n <= NACC; ++n)
    for (int l = 1; l <= 5; ++l) {
      set_lhs(C2P, l, BC_PERIODIC, n, alpha[n], 1.0, alpha[n]);
      R(C2P, l, 1, BC_PERIODIC, n) = a[n];
      R(C2P, l, 2, BC_PERIODIC, n) = b[n] * (1.0 / 3.0);
      R(C2P, l, 3, BC_PERIODIC, n) = 0.0;
    }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(C2P, 1, BC_SYMMETRIC, n, 0.0, 1.0, 0.0);
    mirror_lhs(C2P, BC_SYMMETRIC, n, 1, 5);
    copy_rows(C2P, 2, 4, BC_SYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(C2P, 1, 5, BC_SYMMETRIC, n, BC_PERIODIC, n, false, true);
    set_lhs(C2P, 1, BC_ASYMMETRIC, n, 0.0, 1.0, 2.0 * alpha[n]);
    mirror_lhs(C2P, BC_ASYMMETRIC, n, 1, 5);
    copy_rows(C2P, 2, 4, BC_ASYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(C2P, 1, 5, BC_ASYMMETRIC, n, BC_PERIODIC, n, false, true);
  }
  interior_from_periodic(C2P);
  zero5(al1); zero5(a1); zero5(b1); zero5(c1); zero5(d1); zero5(e1); zero5(f1);
  al1[ACC_CD2] = 0.0; a1[ACC_CD2] = -2.0 - al1[ACC_CD2]; b1[ACC_CD2] = 3.0 + al1[ACC_CD2];
  c1[ACC_CD2] = -1.0;
  for (int n : {ACC_CD4, ACC_CP4}) {
    al1[n] = 0.0;
    a1[n] = (-93.0 - 22.0 * al1[n]) / 24.0;
    b1[n] = (229.0 + 17.0 * al1[n]) / 24.0;
    c1[n] = (-75.0 + 3.0 * al1[n]) / 8.0;
    d1[n] = (111.0 - 5.0 * al1[n]) / 24.0;
    e1[n] = (-22.0 + 1.0 * al1[n]) / 24.0;
  }
  al1[ACC_CP6] = 1689.0 / 71.0;
  a1[ACC_CP6] = (-3043.0 - 563.0 * al1[ACC_CP6]) / 640.0;
  b1[ACC_CP6] = (5353.0 + 201.0 * al1[ACC_CP6]) / 384.0;
  c1[ACC_CP6] = (-3489.0 + 143.0 * al1[ACC_CP6]) / 192.0;
  d1[ACC_CP6] = (859.0 - 37.0 * al1[ACC_CP6]) / 64.0;
  e1[ACC_CP6] = (-2041.0 + 87.0 * al1[ACC_CP6]) / 384.0;
  f1[ACC_CP6] = (1689.0 - 71.0 * al1[ACC_CP6]) / 1920.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(C2P, 1, BC_INTRPL, n, 0.0, 1.0, al1[n]);
    double v[6] = {a1[n], b1[n], c1[n], d1[n], e1[n], f1[n]};
    set_rhs6(C2P, 1, BC_INTRPL, n, v);
    mirror_lhs(C2P, BC_INTRPL, n, 1, 5);
    for (int s = 1; s <= 6; ++s) R(C2P, 5, s, BC_INTRPL, n) = -R(C2P, 1, s, BC_INTRPL, n);
  }
  for (int n = 1; n <= NACC; ++n) copy_rows(C2P, 3, 3, BC_INTRPL, n, BC_PERIODIC, n, true, true);
  zero5(al2); zero5(a2); zero5(b2); zero5(c2); zero5(d2); zero5(e2); zero5(f2);
  al2[ACC_CD2] = 0.0; a2[ACC_CD2] = -1.0; b2[ACC_CD2] = 1.0;
  for (int n : {ACC_CD4, ACC_CP4}) {
    al2[n] = (n == ACC_CD4) ? 0.0 : 1.0 / 22.0;
    a2[n] = (-11.0 - 46.0 * al2[n]) / 12.0;
    b2[n] = (17.0 + 202.0 * al2[n]) / 24.0;
    c2[n] = (3.0 - 66.0 * al2[n]) / 8.0;
    d2[n] = (-5.0 + 110.0 * al2[n]) / 24.0;
    e2[n] = (1.0 - 22.0 * al2[n]) / 24.0;
  }
  al2[ACC_CP6] = 31.0 / 818.0; a2[ACC_CP6] = -5195.0 / 4908.0; b2[ACC_CP6] = 4957.0 / 4908.0;
  c2[ACC_CP6] = 119.0 / 1227.0; d2[ACC_CP6] = -85.0 / 1227.0; e2[ACC_CP6] = 119.0 / 4908.0;
  f2[ACC_CP6] = -17.0 / 4908.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(C2P, 2, BC_INTRPL, n, al2[n], 1.0, al2[n]);
    double v[6] = {a2[n], b2[n], c2[n], d2[n], e2[n], f2[n]};
    set_rhs6(C2P, 2, BC_INTRPL, n, v);
    mirror_lhs(C2P, BC_INTRPL, n, 2, 4);
    for (int s = 1; s <= 6; ++s) R(C2P, 4, s, BC_INTRPL, n) = -R(C2P, 2, s, BC_INTRPL, n);
  }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(C2P, 1, BC_NEUMANN, n, 0.0, 1.0, 0.0);
    for (int s = 1; s <= 6; ++s) R(C2P, 1, s, BC_NEUMANN, n) = 0.0;
    set_lhs(C2P, 5, BC_NEUMANN, n, 0.0, 1.0, 0.0);
    for (int s = 1; s <= 6; ++s) R(C2P, 5, s, BC_NEUMANN, n) = 0.0;
  }
  for (int n = 1; n <= NACC; ++n) {
    copy_rows(C2P, 1, 5, BC_DIRICHLET, n, BC_INTERIOR, n, true, true);
    copy_rows(C2P, 2, 4, BC_NEUMANN, n, BC_INTERIOR, n, true, true);
  }

  // ---------------- 1st derivative, P2C (basics_operations2.f90:946-1078); alpha/a/b: C2P values
  for (int n = 1; n <= NACC; ++n)
    for (int l = 1; l <= 5; ++l) {
      for (int s = 1; s <= 3; ++s) F(P2C, l, s, BC_PERIODIC, n) = F(C2P, l, s, BC_PERIODIC, n);
      for (int s = 1; s <= 6; ++s) R(P2C, l, s, BC_PERIODIC, n) = R(C2P, l, s, BC_PERIODIC, n);
    }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(P2C, 1, BC_SYMMETRIC, n, 0.0, 1.0 - alpha[n], alpha[n]);
    mirror_lhs(P2C, BC_SYMMETRIC, n, 1, 5);
    copy_rows(P2C, 2, 4, BC_SYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(P2C, 1, 5, BC_SYMMETRIC, n, BC_PERIODIC, n, false, true);
    set_lhs(P2C, 1, BC_ASYMMETRIC, n, 0.0, 1.0 + alpha[n], alpha[n]);
    mirror_lhs(P2C, BC_ASYMMETRIC, n, 1, 5);
    copy_rows(P2C, 2, 4, BC_ASYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(P2C, 1, 5, BC_ASYMMETRIC, n, BC_PERIODIC, n, false, true);
  }
  interior_from_periodic(P2C);
  zero5(al1); zero5(a1); zero5(b1); zero5(c1); zero5(d1); zero5(e1); zero5(f1);
  al1[ACC_CD2] = 0.0; a1[ACC_CD2] = -1.0; b1[ACC_CD2] = 1.0;
  for (int n : {ACC_CD4, ACC_CP4}) {
    al1[n] = 0.0;
    a1[n] = (-22.0 + al1[n]) / 24.0;
    b1[n] = (17.0 - 27.0 * al1[n]) / 24.0;
    c1[n] = (3.0 + 9.0 * al1[n]) / 8.0;
    d1[n] = (-5.0 - al1[n]) / 24.0;
    e1[n] = 1.0 / 24.0;
  }
  al1[ACC_CP6] = 71.0 / 9.0;
  a1[ACC_CP6] = (-1689.0 + 71.0 * al1[ACC_CP6]) / 1920.0;
  b1[ACC_CP6] = (67.0 - 141.0 * al1[ACC_CP6]) / 128.0;
  c1[ACC_CP6] = (143.0 + 207.0 * al1[ACC_CP6]) / 192.0;
  d1[ACC_CP6] = (-111.0 + 1.0 * al1[ACC_CP6]) / 192.0;
  e1[ACC_CP6] = (29.0 - 3.0 * al1[ACC_CP6]) / 128.0;
  f1[ACC_CP6] = (-71.0 + 9.0 * al1[ACC_CP6]) / 1920.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(P2C, 1, BC_INTRPL, n, 0.0, 1.0, al1[n]);
    double v[6] = {a1[n], b1[n], c1[n], d1[n], e1[n], f1[n]};
    set_rhs6(P2C, 1, BC_INTRPL, n, v);
    mirror_lhs(P2C, BC_INTRPL, n, 1, 5);
    for (int s = 1; s <= 6; ++s) R(P2C, 5, s, BC_INTRPL, n) = -R(P2C, 1, s, BC_INTRPL, n);
    copy_rows(P2C, 2, 4, BC_INTRPL, n, BC_PERIODIC, n, true, true);
  }
  for (int n = 1; n <= NACC; ++n) {
    copy_rows(P2C, 1, 5, BC_DIRICHLET, n, BC_INTERIOR, n, true, true);
    copy_rows(P2C, 1, 5, BC_NEUMANN, n, BC_INTERIOR, n, true, true);
  }

  // ---------------- interpolation, C2P (basics_operations2.f90:1079-1355)
  zero5(alpha); zero5(a); zero5(b); zero5(c);
  alpha[ACC_CD2] = 0.0; a[ACC_CD2] = 1.0; b[ACC_CD2] = 0.0;
  for (int n : {ACC_CD4, ACC_CP4}) {
    alpha[n] = (n == ACC_CD4) ? 0.0 : 1.0 / 6.0;
    a[n] = 9.0 / 8.0 + 5.0 / 4.0 * alpha[n];
    b[n] = -1.0 / 8.0 + 3.0 / 4.0 * alpha[n];
  }
  alpha[ACC_CP6] = 3.0 / 10.0;
  a[ACC_CP6] = 5.0 * (15.0 + 14.0 * alpha[ACC_CP6]) / 64.0;
  b[ACC_CP6] = (-25.0 + 126.0 * alpha[ACC_CP6]) / 128.0;
  c[ACC_CP6] = (3.0 - 10.0 * alpha[ACC_CP6]) / 128.0;  // computed but unused by the reference
  for (int n = 1; n <= NACC; ++n)
    for (int l = 1; l <= 5; ++l) {
      set_lhs(M2P, l, BC_PERIODIC, n, alpha[n], 1.0, alpha[n]);
      R(M2P, l, 1, BC_PERIODIC, n) = a[n] * 0.5;
      R(M2P, l, 2, BC_PERIODIC, n) = b[n] * 0.5;
      R(M2P, l, 3, BC_PERIODIC, n) = 0.0;
    }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(M2P, 1, BC_SYMMETRIC, n, 0.0, 1.0, alpha[n] + alpha[n]);
    mirror_lhs(M2P, BC_SYMMETRIC, n, 1, 5);
    copy_rows(M2P, 2, 4, BC_SYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(M2P, 1, 5, BC_SYMMETRIC, n, BC_PERIODIC, n, false, true);
    set_lhs(M2P, 1, BC_ASYMMETRIC, n, 0.0, 1.0, 0.0);
    mirror_lhs(M2P, BC_ASYMMETRIC, n, 1, 5);
    copy_rows(M2P, 2, 4, BC_ASYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(M2P, 1, 5, BC_ASYMMETRIC, n, BC_PERIODIC, n, false, true);
  }
  interior_from_periodic(M2P);
  zero5(al1); zero5(a1); zero5(b1); zero5(c1); zero5(d1); zero5(e1); zero5(f1);
  al1[ACC_CD2] = 0.0; a1[ACC_CD2] = (3.0 + al1[ACC_CD2]) / 2.0; b1[ACC_CD2] = (-1.0 + al1[ACC_CD2]) / 2.0;
  for (int n : {ACC_CD4, ACC_CP4}) {
    al1[n] = (n == ACC_CD4) ? 0.0 : 5.0;
    a1[n] = (35.0 + 5.0 * al1[n]) / 16.0;
    b1[n] = (-35.0 + 15.0 * al1[n]) / 16.0;
    c1[n] = (21.0 - 5.0 * al1[n]) / 16.0;
    d1[n] = (-5.0 + al1[n]) / 16.0;
  }
  al1[ACC_CP6] = 9.0;
  a1[ACC_CP6] = (693.0 + 63.0 * al1[ACC_CP6]) / 256.0;
  b1[ACC_CP6] = (-1155.0 + 315.0 * al1[ACC_CP6]) / 256.0;
  c1[ACC_CP6] = (693.0 - 105.0 * al1[ACC_CP6]) / 128.0;
  d1[ACC_CP6] = (-495.0 + 63.0 * al1[ACC_CP6]) / 128.0;
  e1[ACC_CP6] = (385.0 - 45.0 * al1[ACC_CP6]) / 256.0;
  f1[ACC_CP6] = (-63.0 + 7.0 * al1[ACC_CP6]) / 256.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(M2P, 1, BC_INTRPL, n, 0.0, 1.0, al1[n]);
    double v[6] = {a1[n], b1[n], c1[n], d1[n], e1[n], f1[n]};
    set_rhs6(M2P, 1, BC_INTRPL, n, v);
    mirror_lhs(M2P, BC_INTRPL, n, 1, 5);
    for (int s = 1; s <= 6; ++s) R(M2P, 5, s, BC_INTRPL, n) = R(M2P, 1, s, BC_INTRPL, n);
  }
  for (int n = 1; n <= NACC; ++n) copy_rows(M2P, 3, 3, BC_INTRPL, n, BC_PERIODIC, n, true, true);
  zero5(al2); zero5(a2); zero5(b2); zero5(c2); zero5(d2); zero5(e2); zero5(f2);
  al2[ACC_CD2] = 0.0; a2[ACC_CD2] = (1.0 + 2.0 * al2[ACC_CD2]) / 2.0;
  b2[ACC_CD2] = (1.0 + 2.0 * al2[ACC_CD2]) / 2.0;
  for (int n : {ACC_CD4, ACC_CP4}) {
    al2[n] = (n == ACC_CD4) ? 0.0 : 1.0 / 6.0;
    a2[n] = (5.0 + 34.0 * al2[n]) / 16.0;
    b2[n] = (15.0 - 26.0 * al2[n]) / 16.0;
    c2[n] = (-5.0 + 30.0 * al2[n]) / 16.0;
    d2[n] = (1.0 - 6.0 * al2[n]) / 16.0;
  }
  al2[ACC_CP6] = 9.0;
  a2[ACC_CP6] = (63.0 + 686.0 * al2[ACC_CP6]) / 256.0;
  b2[ACC_CP6] = (315.0 - 1050.0 * al2[ACC_CP6]) / 256.0;
  c2[ACC_CP6] = (-105.0 + 798.0 * al2[ACC_CP6]) / 128.0;
  d2[ACC_CP6] = (63.0 - 530.0 * al2[ACC_CP6]) / 128.0;
  e2[ACC_CP6] = (-45.0 + 406.0 * al2[ACC_CP6]) / 256.0;
  f2[ACC_CP6] = (7.0 - 66.0 * al2[ACC_CP6]) / 256.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(M2P, 2, BC_INTRPL, n, al2[n], 1.0, al2[n]);
    double v[6] = {a2[n], b2[n], c2[n], d2[n], e2[n], f2[n]};
    set_rhs6(M2P, 2, BC_INTRPL, n, v);
    mirror_lhs(M2P, BC_INTRPL, n, 2, 4);
    for (int s = 1; s <= 6; ++s) R(M2P, 4, s, BC_INTRPL, n) = R(M2P, 2, s, BC_INTRPL, n);
  }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(M2P, 1, BC_DIRICHLET, n, 0.0, 1.0, 0.0);
    for (int s = 1; s <= 6; ++s) R(M2P, 1, s, BC_DIRICHLET, n) = 0.0;
    set_lhs(M2P, 5, BC_DIRICHLET, n, 0.0, 1.0, 0.0);
    for (int s = 1; s <= 6; ++s) R(M2P, 5, s, BC_DIRICHLET, n) = 0.0;
  }
  for (int n = 1; n <= NACC; ++n) {
    copy_rows(M2P, 1, 5, BC_NEUMANN, n, BC_INTERIOR, n, true, true);
    copy_rows(M2P, 2, 4, BC_DIRICHLET, n, BC_INTERIOR, n, true, true);
  }

  // ---------------- interpolation, P2C (basics_operations2.f90:1356-1527); alpha: C2P interp values
  for (int n = 1; n <= NACC; ++n)
    for (int l = 1; l <= 5; ++l) {
      for (int s = 1; s <= 3; ++s) F(M2C, l, s, BC_PERIODIC, n) = F(M2P, l, s, BC_PERIODIC, n);
      for (int s = 1; s <= 6; ++s) R(M2C, l, s, BC_PERIODIC, n) = R(M2P, l, s, BC_PERIODIC, n);
    }
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(M2C, 1, BC_SYMMETRIC, n, 0.0, 1.0 + alpha[n], alpha[n]);
    mirror_lhs(M2C, BC_SYMMETRIC, n, 1, 5);
    copy_rows(M2C, 2, 4, BC_SYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(M2C, 1, 5, BC_SYMMETRIC, n, BC_PERIODIC, n, false, true);
    set_lhs(M2C, 1, BC_ASYMMETRIC, n, 0.0, 1.0 - alpha[n], alpha[n]);
    mirror_lhs(M2C, BC_ASYMMETRIC, n, 1, 5);
    copy_rows(M2C, 2, 4, BC_ASYMMETRIC, n, BC_PERIODIC, n, true, false);
    copy_rows(M2C, 1, 5, BC_ASYMMETRIC, n, BC_PERIODIC, n, false, true);
  }
  interior_from_periodic(M2C);
  zero5(al1); zero5(a1); zero5(b1); zero5(c1); zero5(d1); zero5(e1); zero5(f1);
  al1[ACC_CD2] = 0.0; a1[ACC_CD2] = 0.5; b1[ACC_CD2] = 0.5; c1[ACC_CD2] = 0.0;
  for (int n : {ACC_CD4, ACC_CP4}) {
    al1[n] = (n == ACC_CD4) ? 0.0 : 1.0;
    a1[n] = (5.0 - al1[n]) / 16.0;
    b1[n] = (15.0 + 9.0 * al1[n]) / 16.0;
    c1[n] = (-5.0 + 9.0 * al1[n]) / 16.0;
    d1[n] = (1.0 - al1[n]) / 16.0;
  }
  al1[ACC_CP6] = 7.0 / 3.0;
  a1[ACC_CP6] = (63.0 - 7.0 * al1[ACC_CP6]) / 256.0;
  b1[ACC_CP6] = (315.0 + 105.0 * al1[ACC_CP6]) / 256.0;
  c1[ACC_CP6] = (-7.0 + 7.0 * al1[ACC_CP6]) * 15.0 / 128.0;
  d1[ACC_CP6] = (63.0 - 35.0 * al1[ACC_CP6]) / 128.0;
  e1[ACC_CP6] = (-15.0 + 7.0 * al1[ACC_CP6]) * 3.0 / 256.0;
  f1[ACC_CP6] = (7.0 - 3.0 * al1[ACC_CP6]) / 256.0;
  for (int n = 1; n <= NACC; ++n) {
    set_lhs(M2C, 1, BC_INTRPL, n, 0.0, 1.0, al1[n]);
    double v[6] = {a1[n], b1[n], c1[n], d1[n], e1[n], f1[n]};
    set_rhs6(M2C, 1, BC_INTRPL, n, v);
    mirror_lhs(M2C, BC_INTRPL, n, 1, 5);
    for (int s = 1; s <= 6; ++s) R(M2C, 5, s, BC_INTRPL, n) = R(M2C, 1, s, BC_INTRPL, n);
    copy_rows(M2C, 2, 4, BC_INTRPL, n, BC_PERIODIC, n, true, true);
  }
  for (int n = 1; n <= NACC; ++n) {
    copy_rows(M2C, 1, 5, BC_NEUMANN, n, BC_INTERIOR, n, true, true);
    copy_rows(M2C, 1, 5, BC_DIRICHLET, n, BC_INTERIOR, n, true, true);
  }
}

// ---------------------------------------------------------------------------
// TDMA, restating src/basics_algorithms.f90:14-109
// ---------------------------------------------------------------------------
void tdma_preprocess(const double* a, const double* b, double* c, double* d, int n) {
  c[0] = c[0] / b[0];
  for (int i = 2; i <= n; ++i) {
    d[i - 1] = 1.0 / (b[i - 1] - a[i - 1] * c[i - 2]);
    if (i < n) c[i - 1] = c[i - 1] * d[i - 1];
  }
}

void tdma_basic(double* x, const double* a, const double* b, const double* c, const double* d, int n) {
  x[0] = x[0] / b[0];
  for (int i = 2; i <= n; ++i) x[i - 1] = (x[i - 1] - a[i - 1] * x[i - 2]) * d[i - 1];
  for (int i = n - 1; i >= 1; --i) x[i - 1] = x[i - 1] - c[i - 1] * x[i];
}

void tdma_cyclic(double* x, const double* a, const double* b, const double* c, const double* d, int n) {
  tdma_basic(x, a, b, c, d, n - 1);
  std::vector<double> x1(n, 0.0);
  x1[0] = -a[0];
  x1[n - 2] = -c[n - 2];
  tdma_basic(x1.data(), a, b, c, d, n - 1);
  x[n - 1] = (x[n - 1] - c[n - 1] * x[0] - a[n - 1] * x[n - 2]) /
             (b[n - 1] + c[n - 1] * x1[0] + a[n - 1] * x1[n - 2]);
  for (int i = 0; i < n - 1; ++i) x[i] = x[i] + x1[i] * x[n - 1];
}

void tdma_solve(bool peri, double* x, const double* a, const double* b, const double* c, const double* d,
                int n) {
  if (peri) tdma_cyclic(x, a, b, c, d, n);
  else tdma_basic(x, a, b, c, d, n);
}

// Buildup_TDMA_LHS_array (basics_operations2.f90:1529-1588) for one (bc1, bc2, acc)
void build_lhs(const Family& fam, int n, int bc1, int bc2, int acc, Lhs& out) {
  out.n = n;
  out.a.assign(n, 0.0); out.b.assign(n, 0.0); out.c.assign(n, 0.0); out.d.assign(n, 0.0);
  const int k = BC_PERIODIC, m = acc - 1;
  for (int col = 1; col <= 3; ++col) {
    std::vector<double>& v = (col == 1) ? out.a : (col == 2) ? out.b : out.c;
    v[0] = fam.f[0][col - 1][bc1][m];
    v[1] = fam.f[1][col - 1][bc1][m];
    for (int i = 3; i <= n - 2; ++i) v[i - 1] = fam.f[2][col - 1][k][m];
    v[n - 2] = fam.f[3][col - 1][bc2][m];
    v[n - 1] = fam.f[4][col - 1][bc2][m];
  }
  if (bc1 == k && bc2 == k) tdma_preprocess(out.a.data(), out.b.data(), out.c.data(), out.d.data(), n - 1);
  else tdma_preprocess(out.a.data(), out.b.data(), out.c.data(), out.d.data(), n);
}

}  // namespace orc
