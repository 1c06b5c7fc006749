// MLP surrogate of the per-cell property update (rho*h -> T, rho, mu, kappa): hand-written
// FP32 training kernels and a BF16 tcgen05 inference kernel with the table lookup as fallback.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "chs_kernels.cuh"

namespace chs {

// network 1 -> 64 -> 64 -> 64 -> 4, tanh on the hidden layers; flat FP32 parameter layout
constexpr int MLP_H = 64;
constexpr int MLP_NOUT = 4;
constexpr int MLP_P_W1 = 0, MLP_P_B1 = 64, MLP_P_W2 = 128, MLP_P_B2 = 128 + 4096, MLP_P_W3 = MLP_P_B2 + 64,
              MLP_P_B3 = MLP_P_W3 + 4096, MLP_P_W4 = MLP_P_B3 + 64, MLP_P_B4 = MLP_P_W4 + 256,
              MLP_NPARAM = MLP_P_B4 + 4;

// normalisation: x = xa*rhoh + xb in [-1, 1]; property j = ya[j]*y_j + yb[j] (T, rho, mu, kappa)
struct MlpNorm {
  double xa, xb;
  double ya[MLP_NOUT], yb[MLP_NOUT];
};

// inference-side constants (FP32 copies of the small layers), passed by value
struct MlpSmall {
  float w1[MLP_H], b1[MLP_H], b2[MLP_H], b3[MLP_H], w4[MLP_NOUT * MLP_H], b4[MLP_NOUT];
};

struct MlpCheck {
  double tol;        // error bound on the network's T, as a fraction of the table's T range
  int win;           // the same bound in table rows: the rho*h bracket is searched within +-win rows
                     // of the row the network's T gives, else from scratch (fallback)
  int raw;           // 1: the network's outputs as they are (no table; tests of the network)
  int uniform_t;     // the table's T column is uniform (O(1) row from T), else bisection on T
  double t0, dt_tab;
};

// packed BF16 weights of the two 64x64 layers in the tensor-core shared-memory layout (16 KB)
void mlp_pack(const float* d_params, uint16_t* d_wpack, cudaStream_t st);

// seeded training samples: rho*h uniform in [dhmin, dhmax], targets from the table lookup
void mlp_make_samples(const ThermoTab& tb, const MlpNorm& nm, uint64_t seed, int n, float* x, float* y,
                      cudaStream_t st);

// one forward/backward pass over B samples (x[B], t[B][4]): loss (mean squared error over the B*4
// outputs) and gradients (flat, zeroed here); work holds 8*B*64 floats
void mlp_grad(const float* params, const float* x, const float* t, int B, float* grads, float* loss_dev,
              float* work, cudaStream_t st);

// training samples gathered by a seeded hash per step
void mlp_gather(const float* xs, const float* ys, int n, uint64_t seed, long long step, int B, float* x, float* t,
                cudaStream_t st);

void mlp_adam(float* params, const float* grads, float* m, float* v, int n, float lr, long long step,
              cudaStream_t st);

// property update by the network (tcgen05, BF16 weights, FP32 accumulation) with per-cell check
// and table fallback; nfallback counts the cells that took the table
template <typename T>
void launch_mlp_props(const ThermoTab& tb, const MlpNorm& nm, const MlpSmall& sm, const MlpCheck& ck,
                      const uint16_t* wpack, const T* rhoh, T* h, T* t, T* k, T* d, T* m, int64_t n,
                      unsigned long long* nfallback, cudaStream_t st);

}  // namespace chs
