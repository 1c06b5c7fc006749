// Fused substep kernels for the CD2 scheme: the momentum right-hand side of each component with the
// RK3 fractional step in one pass, the wall planes it needs, and the advance of the velocities.
//
// The operator-by-operator substep (chs_solver.cu) writes every interpolated velocity and every
// velocity derivative to HBM and reads it back in the component sums.  Here each output value
// evaluates those inner operators where it needs them, from the velocities (and momenta and
// viscosity with variable properties) themselves, so only the primary fields are read and only
// the right-hand sides are written.  Every operator is the same plan as the operator path's (the
// host builds this descriptor from the plans the substep would launch): x and z operators are
// periodic and use the bulk formula with wrapped indices; y operators use the bulk formula in
// their bulk range and the plan's boundary rows (sparse forms over the line and the wall planes)
// outside it, then the y metric and the Neumann overrides, exactly as stencil_op_kernel does.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "chs_kernels.cuh"

namespace chs {

// One explicit operator inside a fused kernel.  kind 0: periodic line whose every row is the bulk
// formula with wrapped indices; kind 1: bulk formula on rows [b_lo, b_hi], the plan's boundary
// rows (plans[plan]) elsewhere.
struct FzOp {
  int kind;
  int b_lo, b_hi;
  int lmap;   // offset of the y metric in the operator table, or -1
  int neu;    // bit 0: first row = fbc plane 0; bit 1: last row = fbc plane 1
  int nout;
  int plan;   // index of the full plan (boundary rows) in the device plan array
  double r1, r2, dd;
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
  const T *gx, *gy, *gz, *mu;           // variable properties (else null)
  const T *fyqx, *fyqy, *fyqz, *fz, *fm;  // y wall planes of qx, qy, qz, zero momentum, viscosity
  FzOp in[FI_COUNT];
  FzPair<T> term[3][3];  // [component][direction]
  FzOp pres[3];          // pressure gradient of each component
  const T* fpres[3];
  T *m[3], *m0[3];       // right-hand sides (fractional-step increments) and their histories
  double rre, dt, gam, zeta, alpha;
  const OpPlan* plans;   // device array of the full plans
  const double* table;   // operator table (y metric)
};

// rows at each y wall that take the launch with the plans' boundary rows (the others compile the
// bulk formulas only); valid when every y plan's bulk range covers rows 2 .. nout-3
constexpr int kFzEdge = 4;

// the right-hand side of momentum component c (0 x, 1 y, 2 z) with the fractional step
// (m = dt*(gam*F + zeta*m0 + alpha*pfc), m0 = F); the advance q += m is left to launch_fz_update.
// CD2 plans only (every bulk formula two-point); x and z periodic.
template <typename T>
void launch_fz_momentum(const FzMomentum<T>& f, int c, cudaStream_t st);

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

}  // namespace chs
