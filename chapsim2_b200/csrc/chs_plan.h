// Host-side operator plans for the compact finite-difference line operators.
//
// A plan describes one operator Get_{x,y,z}_{midp,1der}_{C2P,P2C,C2C,P2P}
// (src/basics_operations2.f90:2739-4800) on a line of fixed length as:
//   * a bulk two-coefficient stencil,
//   * up to four boundary rows given as sparse linear forms over the input
//     line and the four boundary values fbc(1:4),
//   * an optional (cyclic) Thomas solve with a pre-factorised LHS,
//   * an optional y-mapping multiplier and Neumann overrides.
// The GPU kernel in chs_kernels.cu executes plans for batches of lines.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace chs {

constexpr double kMaxp = 1.0e20;  // MAXP, src/modules.f90:142

enum Bc { BC_INTERIOR = 0, BC_PERIODIC = 1, BC_SYMMETRIC = 2, BC_ASYMMETRIC = 3, BC_DIRICHLET = 4,
          BC_NEUMANN = 5, BC_INTRPL = 6 };
enum Acc { ACC_CD2 = 1, ACC_CD4 = 2, ACC_CP4 = 3, ACC_CP6 = 4 };
enum Fam { D1C2C = 0, D1P2P = 1, D1C2P = 2, D1P2C = 3, M1C2P = 4, M1P2C = 5 };

inline bool fam_c_input(int f) { return f == D1C2C || f == D1C2P || f == M1C2P; }
inline bool fam_p_output(int f) { return f == D1P2P || f == D1C2P || f == M1C2P; }
inline bool fam_deriv(int f) { return f <= D1P2C; }

// Compact-scheme coefficients of one operator family at one accuracy:
// lhs[row][col][bc] (alpha, 1, alpha) and rhs[row][col][bc], rows 0..4.
struct CoefSet {
  double lhs[5][3][7];
  double rhs[5][6][7];
};
// coef(fam, acc) for acc = 1..4
const CoefSet& coef(int fam, int acc);

constexpr int kMaxTerms = 10;
struct SpecialRow {
  int row;              // 0-based output row
  int nt;               // number of input terms
  int idx[kMaxTerms];   // 0-based input indices
  double w[kMaxTerms];
  double wb[4];         // weights on fbc(1..4)
};

// Device-visible plan (POD, passed by value to kernels).
struct OpPlan {
  int fam, nin, nout;
  int b_lo, b_hi;        // bulk output rows [b_lo, b_hi] (0-based, inclusive)
  int off[4];            // bulk input offsets relative to the output row
  double sgn, r1, r2;    // bulk: r1*(f[i+off0] + sgn f[i+off1]) + r2*(f[i+off2] + sgn f[i+off3])
  double dd;             // scaling applied to every row (1/h for derivatives, 1 for interpolation)
  int nspec;
  SpecialRow sp[4];
  int tdma;              // 0 none, 1 Thomas, 2 cyclic Thomas
  double b1;             // LHS b(1)
  double an, cn, inv_den;  // cyclic closure: a(n), c(n), 1/(b(n) + c(n) x1(1) + a(n) x1(n-1))
  // offsets (in doubles) of the LHS arrays inside the handle's device table:
  // a(n), c'(n), d(n) and the cyclic correction vector x1(n-1)
  int64_t la, lc, ld, lx1;
  int64_t lmap;          // y-mapping multiplier (nout) or -1
  int neu1, neu2;        // overwrite first/last row with fbc(1)/fbc(2)
  int needs_fbc;         // 1 if any boundary value is read
  int wrap;              // periodic explicit line whose boundary rows are the bulk stencil with
                         // wrapped indices: every row may use the bulk formula
};

// Builds plans and the LHS/mapping table they reference.
class PlanBook {
 public:
  // h: grid spacing of the direction; dp: ghost spacings (4) for C-input and P-input operators
  struct DirGeom {
    int nc, np;
    bool periodic;
    double dd;              // h1r
    double dp_c[4], dp_p[4];
    int64_t map_cc = -1, map_pt = -1;  // offsets of mapping arrays (y with stretching), -1 otherwise
  };
  DirGeom dir[3];
  int iacc = ACC_CP6;
  std::vector<double> table;  // LHS and mapping data uploaded to the device

  int64_t add_array(const std::vector<double>& v);
  // ibc0: nominal operation bc pair; has_fbc: boundary values supplied
  OpPlan make(int d, int fam, const int ibc0[2], bool has_fbc);

 private:
  struct LhsKey { int fam, n, b1, b2; int64_t la, lc, ld, lx1; double b1v, an, cn, inv_den; };
  std::vector<LhsKey> lhs_;
  const LhsKey& lhs(int fam, int n, int bc1, int bc2);
};

void reduce_bc(int fam, const int ibc0[2], bool has_fbc, int ibc[2]);

}  // namespace chs
