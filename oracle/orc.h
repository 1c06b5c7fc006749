// ORACLE (test infrastructure only; never linked into the product library).
// Shared declarations of the CPU FP64 restatement of CHAPSim2's flow path.
#pragma once
#include <vector>

namespace orc {

constexpr double MAXP = 1.0e20;  // src/modules.f90:142
constexpr int NL = 5, NBC = 7, NACC = 4;

// src/modules.f90:223-229
enum { BC_INTERIOR = 0, BC_PERIODIC = 1, BC_SYMMETRIC = 2, BC_ASYMMETRIC = 3, BC_DIRICHLET = 4,
       BC_NEUMANN = 5, BC_INTRPL = 6 };
// src/modules.f90:248-251
enum { ACC_CD2 = 1, ACC_CD4 = 2, ACC_CP4 = 3, ACC_CP6 = 4 };

// operator families: d1fC2C/d1rC2C ... m1fP2C/m1rP2C (src/basics_operations2.f90:115-143)
enum { FAM_D1C2C = 0, FAM_D1P2P = 1, FAM_D1C2P = 2, FAM_D1P2C = 3, FAM_M1C2P = 4, FAM_M1P2C = 5, NFAM = 6 };

struct Family {
  double f[NL][3][NBC][NACC];  // LHS (alpha, 1, alpha)
  double r[NL][6][NBC][NACC];  // RHS
};
struct Tables {
  Family fam[NFAM];
};

struct Lhs {
  int n = 0;
  std::vector<double> a, b, c, d;
};

void build_tables(Tables& T);
void tdma_preprocess(const double* a, const double* b, double* c, double* d, int n);
void tdma_basic(double* x, const double* a, const double* b, const double* c, const double* d, int n);
void tdma_cyclic(double* x, const double* a, const double* b, const double* c, const double* d, int n);
void tdma_solve(bool peri, double* x, const double* a, const double* b, const double* c, const double* d,
                int n);
void build_lhs(const Family& fam, int n, int bc1, int bc2, int acc, Lhs& out);

}  // namespace orc
