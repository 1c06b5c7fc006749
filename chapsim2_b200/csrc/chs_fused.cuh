// Fused substep kernels for the CD2 scheme: the momentum right-hand side of each component with the
// RK3 fractional step in one pass, the energy equation with its advance in one pass, and the pressure
// update with the projection (and q = g / rho_face) in one pass.
//
// The operator-by-operator substep (chs_solver.cu) writes every interpolated velocity and every
// velocity derivative to HBM and reads it back in the component sums.  Here each output value
// evaluates those inner operators where it needs them, from the primary fields themselves, so only
// the primary fields are read and only the right-hand sides are written.  Every operator is the same
// plan as the operator path's (the host builds these descriptors from the plans the substep would
// launch): x and z are periodic and every row is the two-point bulk formula with wrapped indices; a y
// operator with walls is a table of rows (FzRow), each at most three taps over the input line and
// the two wall planes, built from the plan's bulk formula, its boundary rows, the y metric and the
// Neumann overrides.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "chs_kernels.cuh"
#include "chs_thermo_dev.cuh"

namespace chs {

// One output row p of a y operator with walls:
//   v = w[0] f(p + o[0]) + w[1] f(p + o[1]) (+ w[2] f(p + o[2])) (+ wb[0] fbc0 + wb[1] fbc1)
// with the operator's 1/h and the row's y metric folded into the weights; a Neumann row is wb = 1.
struct FzRow {
  double w[3];
  double wb[2];
  int o[3];
  int flags;  // bit 0: tap 2 used; bit 1: wall plane 0 used; bit 2: wall plane 1 used
};

// One explicit CD2 operator.  row < 0: periodic line, every row r1*(two-point formula)*dd with
// wrapped indices; row >= 0: a y line with walls whose output row p is rows[row + p].
struct FzOp {
  int row;
  double r1, dd;
};

// op(conv) + w*op(visc) of one direction of one momentum component: one application of `a` on the
// combined expression conv + (s_visc*w)*visc when merged (the operator path's pair rule), else
// `a` on conv and `b` on visc with weight w
template <typename T>
struct FzPair {
  FzOp a, b;
  const T* fa;  // boundary planes [4][nx*nz] of a (the combined planes when merged) or null
  const T* fb;
  int merged;
};

// Slots of the inner operators (in the order of the operator path's derived quantities)
enum FzInner {
  // velocity interpolations and derivatives
  FI_QX_MX, FI_QX_DX, FI_QX_DY, FI_QX_MY, FI_QX_MZ, FI_QX_DZ,
  FI_QY_DX, FI_QY_MX, FI_QY_DY, FI_QY_MY, FI_QY_DZ, FI_QY_MZ,
  FI_QZ_DX, FI_QZ_MX, FI_QZ_MY, FI_QZ_DY, FI_QZ_MZ, FI_QZ_DZ,
  // variable properties: momentum interpolations and viscosity interpolations
  FI_GX_MX, FI_GX_MY, FI_GX_MZ, FI_GY_MX, FI_GY_MY, FI_GY_MZ, FI_GZ_MX, FI_GZ_MY, FI_GZ_MZ,
  FI_MU_Y, FI_MU_YX, FI_MU_X, FI_MU_XZ, FI_MU_YZ,
  // wall divergence of the y-viscous boundary value: d/dx of qxiy, d/dy of qyiy, d/dz of qziy
  FI_W_DX, FI_W_DY, FI_W_DZ,
  FI_COUNT
};

template <typename T>
struct FzMomentum {
  int n0, nc1, np1, n2;  // x cells (= points), y cells, y points, z cells (= points)
  int thermo;
  int periodic_y;
  const T *qx, *qy, *qz, *p;
  const T *gx, *gy, *gz, *mu;             // variable properties (else null)
  const T *fyqx, *fyqy, *fyqz, *fz, *fm;  // y wall planes of qx, qy, qz, zero momentum, viscosity
  FzOp in[FI_COUNT];
  FzPair<T> term[3][3];  // [component][direction]
  FzOp pres[3];          // pressure gradient of each component
  const T* fpres[3];
  T *m[3], *m0[3];       // right-hand sides (fractional-step increments) and their histories
  double rre, dt, gam, zeta, alpha;
  const FzRow* rows;     // row tables of the y operators
  // constant mass flux: the x component also writes, per CTA, the y-weighted sum of its outputs
  // (wy[j] * m, the numerator of the volume mean), for launch_fz_finalize_mean; null otherwise
  const double* wy;
  double* part;
};

// bulk[0] = (sum of the x pass's nblk per-CTA sums) / vol, in a fixed order (one CTA)
void launch_fz_finalize_mean(const double* part, int nblk, double* bulk, double vol, cudaStream_t st);
// the right-hand side of momentum component c (0 x, 1 y, 2 z) with the fractional step
// (m = dt*(gam*F + zeta*m0 + alpha*pfc), m0 = F); the advance q += m is left to launch_fz_update
template <typename T>
void launch_fz_momentum(const FzMomentum<T>& f, int c, cudaStream_t st);
// CTAs of the x component's launch (the length of f.part)
int fz_momentum_x_blocks(int n0, int nc1, int n2);

// wall planes of the y-viscous boundary value (fbcy_velo): fvisc2 = walls of
// s*(qydy_cpc - (qxdx_cpc + qydy_cpc + qzdz_cpc)/3)*(mu_y or c2) and fcomb = fconv2 + rre*fvisc2,
// each side into planes side and side + 2
template <typename T>
void launch_fz_wall_visc(const FzMomentum<T>& f, T* fvisc2, T* fcomb, const T* fconv2, cudaStream_t st);

// q advance after the mass-flux mean: ux += mx - bulk, uy += my, uz += mz, then the y walls of uy
// set to v0 / v1 (flags s0 / s1)
template <typename T>
void launch_fz_update(T* ux, T* uy, T* uz, const T* mx, const T* my, const T* mz, const double* bulk, int n0,
                      int nc1, int np1, int n2, int s0, double v0, int s1, double v1, cudaStream_t st);

// ---- energy equation (Solve_energy_eq, src/eq_energy.f90:148-458): per cell the sum over the three
// directions of d/dx_j[-g_j h_face + rPrRen kappa_face dT/dx_j] (face interpolations of h and
// kappa, temperature gradients), the fractional step and the rho*h update in one pass
enum FzEInner { FE_H_X, FE_H_Y, FE_H_Z, FE_K_X, FE_K_Y, FE_K_Z, FE_T_X, FE_T_Y, FE_T_Z, FE_RH_Y, FE_COUNT };
template <typename T>
struct FzEnergy {
  int n0, nc1, np1, n2;
  const T *gx, *gy, *gz, *h, *k, *t;
  const T *fh, *fk, *fqw, *fdtk;  // y wall planes: h, kappa, the wall gradient of T, kappa*dT/dy
  FzOp in[FE_COUNT];
  FzPair<T> term[3];              // conv + rPrRen*diffusion per direction (y: never merged)
  T *rhoh, *rhs0;
  double rpr, dt, gam, zeta;
  const FzRow* rows;
  // wall states after the update (walls flagged ws0 / ws1): the property lookup of rho*h
  // interpolated to each wall, into planes side and side + 2 of wh, wk, wm, wd
  ThermoTab tab;
  int ws0, ws1;
  T *wh, *wk, *wm, *wd;
};
// rhs0 <- F, rho*h += dt*(gam*F + zeta*rhs0) (energy_advance_kernel's arithmetic)
template <typename T>
void launch_fz_energy(const FzEnergy<T>& f, cudaStream_t st);
// wall rows, before the energy pass (mode 0): kappa*dT/dy into planes side and side + 2 of out;
// after it (mode 1): the wall states (rho*h interpolated to each flagged wall and looked up in the
// table: launch_wall_props on the wall rows of that interpolation); out unused
template <typename T>
void launch_fz_energy_walls(const FzEnergy<T>& f, int mode, T* out, cudaStream_t st);

// ---- pressure update and projection (src/eq_momentum2.f90:1577-1660, :1890) with, for variable
// properties, q = g / rho_face (convert_primary_conservative, src/para_conversion.f90:5-227)
enum FzPInner { FP_PX, FP_PY, FP_PZ, FP_DX, FP_DY, FP_DZ, FP_COUNT };
template <typename T>
struct FzProject {
  int n0, nc1, np1, n2;
  int thermo, periodic_y;
  const T* phi;
  T *p, *ux, *uy, *uz;            // pressure, advanced variables (g with variable properties, else q)
  T *qx, *qy, *qz;                // velocities (variable properties)
  const T* rho;
  const T *fphi, *fd;             // y planes of the pressure-correction gradient and of rho
  FzOp in[FP_COUNT];              // rho to the faces (3), d/dx_i phi (3)
  double coef;                    // -dt*alpha*sigma
  int s0, s1;                     // y walls of uy set to v0 / v1
  double v0, v1;
  const FzRow* rows;
  // upd: the advance of the momentum step (u += m - bulk, fz_update_kernel's arithmetic) is done
  // here, at each thread's own point, before the correction (the momentum step left u unchanged)
  int upd;
  const T *mx, *my, *mz;
  const double* bulk;
};
template <typename T>
void launch_fz_project(const FzProject<T>& f, cudaStream_t st);

// Poisson right-hand side coeff * (d/dx ux' + d/dy uy' + d/dz uz') of the advanced fields
// u' = u + m - bulk (y wall rows of uy' set to v0 / v1), formed at each face from u and m without
// storing u' (the projection stores it): the divergence of the operator path (run_fused on
// D1P2C of u') with the momentum advance folded in
template <typename T>
struct FzUpdateDiv {
  int n0, nc1, np1, n2;
  const T *ux, *uy, *uz, *mx, *my, *mz;
  const double* bulk;  // mass-flux mean subtracted from mx, or null
  int s0, s1;
  double v0, v1;
  FzOp dx, dy, dz;     // D1P2C: x and z periodic, y a row table
  const T* fdy;        // y wall planes of the y operator (a plan without boundary values never reads them)
  const FzRow* rows;
  T* out;
  double coeff;
};
template <typename T>
void launch_fz_update_div(const FzUpdateDiv<T>& f, cudaStream_t st);

}  // namespace chs
