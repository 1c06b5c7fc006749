// MLP surrogate of the per-cell property update (rho*h -> T, rho, mu, kappa) of
// Update_thermal_properties (src/eq_energy.f90:14-146, src/input_thermo.f90:393-446).
//
// Training: FP32 forward/backward/Adam kernels written here (no library), on seeded samples
// whose targets are the table lookup itself.  Inference: one CTA of 128 threads per tile of
// 128 cells; layer 1 (1 -> 64) and layer 4 (64 -> 4) on the CUDA cores, layers 2 and 3
// (64 x 64) as tcgen05.mma (BF16 operands in shared memory, FP32 accumulators in TMEM, read
// back with tcgen05.ld).  Every cell's result is checked against the table (rho*h of the
// predicted T) and replaced by the table lookup when the check fails.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "chs_mlp.cuh"
#include "chs_thermo_dev.cuh"

namespace chs {

namespace {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014)
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// ---------------------------------------------------------------------------
// samples and minibatches
// ---------------------------------------------------------------------------
__global__ void samples_kernel(const __grid_constant__ ThermoTab tb, const __grid_constant__ MlpNorm nm,
                               uint64_t seed, int n, float* __restrict__ x, float* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double u = (double)(mix64(seed + (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0);
    const double rh = tb.dhmin + u * (tb.dhmax - tb.dhmin);
    const CellProps p = props_from_dh(tb, rh);
    x[i] = (float)(nm.xa * rh + nm.xb);
    const double v[MLP_NOUT] = {p.t, p.d, p.m, p.k};
#pragma unroll
    for (int j = 0; j < MLP_NOUT; ++j) y[(size_t)i * MLP_NOUT + j] = (float)((v[j] - nm.yb[j]) / nm.ya[j]);
  }
}

__global__ void gather_kernel(const float* __restrict__ xs, const float* __restrict__ ys, int n, uint64_t seed,
                              long long step, int B, float* __restrict__ x, float* __restrict__ t) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    const uint64_t r = mix64(seed ^ mix64((uint64_t)step * (uint64_t)B + (uint64_t)b));
    const int i = (int)(r % (uint64_t)n);
    x[b] = xs[i];
#pragma unroll
    for (int j = 0; j < MLP_NOUT; ++j) t[(size_t)b * MLP_NOUT + j] = ys[(size_t)i * MLP_NOUT + j];
  }
}

// ---------------------------------------------------------------------------
// dense layers (FP32): Hout[B][N] = act(Hin[B][K] W^T + b), W is N x K row-major
// ---------------------------------------------------------------------------
template <int K, int N, bool ACT>
__global__ void dense_fwd_kernel(const float* __restrict__ Hin, const float* __restrict__ W,
                                 const float* __restrict__ bias, float* __restrict__ Hout, int B) {
  __shared__ float sW[N][K + 1];
  __shared__ float sb[N];
  for (int i = threadIdx.x; i < N * K; i += blockDim.x) sW[i / K][i % K] = W[i];
  for (int i = threadIdx.x; i < N; i += blockDim.x) sb[i] = bias[i];
  __syncthreads();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < B * N; e += gridDim.x * blockDim.x) {
    const int b = e / N, o = e - b * N;
    const float* h = Hin + (size_t)b * K;
    float acc = sb[o];
#pragma unroll 8
    for (int k = 0; k < K; ++k) acc = fmaf(h[k], sW[o][k], acc);
    Hout[e] = ACT ? tanhf(acc) : acc;
  }
}

// dY = d(loss)/dY for loss = mean over B*4 of (Y - T)^2; loss accumulated into *loss
__global__ void loss_kernel(const float* __restrict__ Y, const float* __restrict__ Tt, int B, float* __restrict__ dY,
                            float* __restrict__ loss) {
  __shared__ float red[256];
  const float inv = 1.0f / (float)(B * MLP_NOUT);
  float acc = 0.0f;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < B * MLP_NOUT; e += gridDim.x * blockDim.x) {
    const float r = Y[e] - Tt[e];
    dY[e] = 2.0f * r * inv;
    acc += r * r * inv;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

// dZin[B][K] = (dZ[B][N] W) * (1 - Hact^2)   (Hact = tanh output feeding this layer)
template <int K, int N>
__global__ void dense_bwd_data_kernel(const float* __restrict__ dZ, const float* __restrict__ W,
                                      const float* __restrict__ Hact, float* __restrict__ dZin, int B) {
  __shared__ float sW[N][K + 1];
  for (int i = threadIdx.x; i < N * K; i += blockDim.x) sW[i / K][i % K] = W[i];
  __syncthreads();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < B * K; e += gridDim.x * blockDim.x) {
    const int b = e / K, k = e - b * K;
    const float* z = dZ + (size_t)b * N;
    float acc = 0.0f;
#pragma unroll 4
    for (int o = 0; o < N; ++o) acc = fmaf(z[o], sW[o][k], acc);
    const float a = Hact[e];
    dZin[e] = acc * (1.0f - a * a);
  }
}

// dW[N][K] += sum_b dZ[b][n] Hin[b][k], db[n] += sum_b dZ[b][n]; one CTA per 64 samples
template <int K, int N>
__global__ void dense_bwd_weight_kernel(const float* __restrict__ dZ, const float* __restrict__ Hin, int B,
                                        float* __restrict__ dW, float* __restrict__ db) {
  constexpr int CH = 64;
  __shared__ float sZ[CH][N];
  __shared__ float sH[CH][K];
  const int b0 = blockIdx.x * CH;
  for (int i = threadIdx.x; i < CH * N; i += blockDim.x) {
    const int s = i / N, o = i - s * N;
    sZ[s][o] = (b0 + s < B) ? dZ[(size_t)(b0 + s) * N + o] : 0.0f;
  }
  for (int i = threadIdx.x; i < CH * K; i += blockDim.x) {
    const int s = i / K, k = i - s * K;
    sH[s][k] = (b0 + s < B) ? Hin[(size_t)(b0 + s) * K + k] : 0.0f;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < N * K + N; e += blockDim.x) {
    float acc = 0.0f;
    if (e < N * K) {
      const int o = e / K, k = e - o * K;
#pragma unroll 8
      for (int s = 0; s < CH; ++s) acc = fmaf(sZ[s][o], sH[s][k], acc);
      atomicAdd(&dW[e], acc);
    } else {
      const int o = e - N * K;
#pragma unroll 8
      for (int s = 0; s < CH; ++s) acc += sZ[s][o];
      atomicAdd(&db[o], acc);
    }
  }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float c1, float c2) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1.0e-8f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// BF16 copies of W2 and W3 in the no-swizzle K-major core-matrix layout of the tensor-core
// operands: element (n, k) of a 64 x 64 layer at byte (k/8)*1024 + (n/8)*128 + (n%8)*16 + (k%8)*2
__global__ void pack_kernel(const float* __restrict__ params, uint16_t* __restrict__ out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 2 * 4096; e += gridDim.x * blockDim.x) {
    const int layer = e / 4096, r = e - layer * 4096;
    const int n = r / 64, k = r - n * 64;
    const float w = params[(layer == 0 ? MLP_P_W2 : MLP_P_W3) + r];
    const int byte = (k >> 3) * 1024 + (n >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
    const __nv_bfloat16 bw = __float2bfloat16_rn(w);
    out[layer * 4096 + byte / 2] = *reinterpret_cast<const uint16_t*>(&bw);
  }
}

// ---------------------------------------------------------------------------
// tcgen05 inference
// ---------------------------------------------------------------------------
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// hardware tanh of two packed BF16 values (the activations that feed the next BF16 MMA)
__device__ __forceinline__ uint32_t tanh_bf16x2(uint32_t x) {
  uint32_t y;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(x));
  return y;
}

// shared-memory matrix descriptor, no swizzle, K-major: start, leading-dimension byte offset
// (between the two 8-element K chunks of one MMA), stride byte offset (between 8-row groups),
// descriptor version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: kind::f16, A and B BF16, D FP32, both K-major, M = 128, N = 64
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :
      : "r"(tmem), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}


__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
               : "r"(taddr));
}

// bounded wait on an mbarrier phase: false when it did not complete within ~2e9 cycles
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 2000000000LL) return false;
  }
}

// one 128 x 64 x 64 layer: D(tmem) = A(sA) * W(sW)^T, K in four steps of 16
__device__ __forceinline__ void issue_layer(uint32_t tmem, uint32_t sa, uint32_t sw, uint32_t bar) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const uint64_t a = umma_desc(sa + kk * 2 * 2048, 2048, 128);
    const uint64_t b = umma_desc(sw + kk * 2 * 1024, 1024, 128);
    mma_bf16(tmem, a, b, kk > 0 ? 1u : 0u);
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

template <typename T>
__global__ void __launch_bounds__(128, 6) mlp_props_kernel(
    const __grid_constant__ ThermoTab tb, const __grid_constant__ MlpNorm nm, const __grid_constant__ MlpSmall sm,
    const __grid_constant__ MlpCheck ck, const uint16_t* __restrict__ wpack, const T* __restrict__ rhoh,
    T* __restrict__ h, T* __restrict__ t, T* __restrict__ k, T* __restrict__ d, T* __restrict__ m, int64_t n,
    unsigned long long* __restrict__ nfallback) {
  __shared__ __align__(1024) uint8_t sA[128 * 64 * 2];
  __shared__ __align__(1024) uint8_t sW[2 * 64 * 64 * 2];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < 1024; i += 128) reinterpret_cast<uint4*>(sW)[i] = reinterpret_cast<const uint4*>(wpack)[i];
  const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&mbar));
  const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(sA));
  const uint32_t sw = static_cast<uint32_t>(__cvta_generic_to_shared(sW));
  if (tid == 0) {
    failed = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const uint32_t slot = static_cast<uint32_t>(__cvta_generic_to_shared(&tmem_slot));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(64u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  const int rowoff = (tid >> 3) * 128 + (tid & 7) * 16;

  for (int64_t tile = blockIdx.x; tile * 128 < n; tile += gridDim.x) {
    const int64_t c = tile * 128 + tid;
    const bool valid = c < n;
    const double rh = valid ? (double)rhoh[c] : tb.dhmin;
    const float x = (float)(nm.xa * rh + nm.xb);
    // layer 1 (CUDA cores) -> A operand
#pragma unroll
    for (int kc = 0; kc < 8; ++kc) {
      uint32_t q[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o = kc * 8 + 2 * j;
        q[j] = tanh_bf16x2(pack_bf16x2(fmaf(sm.w1[o], x, sm.b1[o]), fmaf(sm.w1[o + 1], x, sm.b1[o + 1])));
      }
      *reinterpret_cast<uint4*>(sA + kc * 2048 + rowoff) = make_uint4(q[0], q[1], q[2], q[3]);
    }
    // layers 2 and 3 on the tensor cores; the accumulators are read back in two halves of 32
    // columns: layer 2's activations go to the A operand, layer 3's straight into layer 4 (CUDA
    // cores), which forms T only unless the raw network outputs are asked for
    float y4[MLP_NOUT];
#pragma unroll
    for (int j = 0; j < MLP_NOUT; ++j) y4[j] = sm.b4[j];
#pragma unroll
    for (int layer = 0; layer < 2; ++layer) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (failed) break;
      // one thread issues the MMAs and waits for their commit; the others wait at the barrier
      // (no issue slots spent polling)
      if (tid == 0) {
        issue_layer(tmem, sa, sw + layer * 8192, bar);
        if (!mbar_wait(bar, phase)) failed = 1;
      }
      phase ^= 1;
      // a wait that gave up leaves the accumulators unread: every thread sees the flag here
      __syncthreads();
      if (failed) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const float* bias = layer == 0 ? sm.b2 : sm.b3;
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        uint32_t r[32];
        tmem_ld32(tl + hh * 32, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (layer == 0) {
#pragma unroll
          for (int kc = 0; kc < 4; ++kc) {
            uint32_t q[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int o = kc * 8 + 2 * j;
              q[j] = tanh_bf16x2(pack_bf16x2(__uint_as_float(r[o]) + bias[hh * 32 + o],
                                             __uint_as_float(r[o + 1]) + bias[hh * 32 + o + 1]));
            }
            *reinterpret_cast<uint4*>(sA + (hh * 4 + kc) * 2048 + rowoff) = make_uint4(q[0], q[1], q[2], q[3]);
          }
        } else {
#pragma unroll
          for (int o = 0; o < 32; ++o) {
            const float v = tanh_fast(__uint_as_float(r[o]) + bias[hh * 32 + o]);
            y4[0] = fmaf(sm.w4[hh * 32 + o], v, y4[0]);
            if (ck.raw) {
#pragma unroll
              for (int j = 1; j < MLP_NOUT; ++j) y4[j] = fmaf(sm.w4[j * 64 + hh * 32 + o], v, y4[j]);
            }
          }
        }
      }
    }
    __syncthreads();
    if (failed) break;
    double y[MLP_NOUT];
#pragma unroll
    for (int j = 0; j < MLP_NOUT; ++j) y[j] = nm.ya[j] * (double)y4[j] + nm.yb[j];
    // the network's T selects the table row where the rho*h search starts; the table judges it
    // exactly (the search from that row is verified, else it runs from scratch), so the stored
    // properties are always the table lookup's
    bool fb = false;
    if (valid && !ck.raw) {
      int hint = -1;
      if (ck.win < 0) {
        // no hint: the full table search for every cell
      } else if (ck.uniform_t) {
        const double f = (y[0] - ck.t0) / ck.dt_tab;
        if (f >= 0.0 && f <= (double)(tb.n - 1)) hint = (int)f;
      } else if (y[0] >= __ldg(tb.t) && y[0] <= __ldg(tb.t + tb.n - 1)) {
        int i1, i2;
        double w1;
        tab_bracket(tb.t, tb.n, y[0], i1, i2, w1);
        hint = i1;
      }
      bool hit = false;
      const CellProps p = props_from_dh(tb, rh, hint, ck.win, &hit);
      fb = !hit;
      h[c] = T(p.h);
      t[c] = T(p.t);
      k[c] = T(p.k);
      d[c] = T(p.d);
      m[c] = T(p.m);
    } else if (valid) {
      h[c] = T(rh / y[1]);
      t[c] = T(y[0]);
      d[c] = T(y[1]);
      m[c] = T(y[2]);
      k[c] = T(y[3]);
    }
    const unsigned mask = __ballot_sync(0xffffffffu, fb);
    if (lane == 0 && mask) atomicAdd(nfallback, (unsigned long long)__popc(mask));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (failed && tid == 0) atomicAdd(nfallback, 1ull << 62);  // error marker read by the host
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64u));
  }
}

}  // namespace

void mlp_pack(const float* d_params, uint16_t* d_wpack, cudaStream_t st) {
  pack_kernel<<<32, 256, 0, st>>>(d_params, d_wpack);
}

void mlp_make_samples(const ThermoTab& tb, const MlpNorm& nm, uint64_t seed, int n, float* x, float* y,
                      cudaStream_t st) {
  samples_kernel<<<148 * 8, 256, 0, st>>>(tb, nm, seed, n, x, y);
}

void mlp_gather(const float* xs, const float* ys, int n, uint64_t seed, long long step, int B, float* x, float* t,
                cudaStream_t st) {
  gather_kernel<<<(B + 255) / 256, 256, 0, st>>>(xs, ys, n, seed, step, B, x, t);
}

void mlp_grad(const float* P, const float* x, const float* t, int B, float* G, float* loss, float* work,
              cudaStream_t st) {
  const size_t bh = (size_t)B * MLP_H;
  float *H1 = work, *H2 = work + bh, *H3 = work + 2 * bh, *Y = work + 3 * bh, *dY = Y + (size_t)B * MLP_NOUT;
  float *dZ3 = work + 4 * bh, *dZ2 = work + 5 * bh, *dZ1 = work + 6 * bh;
  cudaMemsetAsync(G, 0, MLP_NPARAM * sizeof(float), st);
  cudaMemsetAsync(loss, 0, sizeof(float), st);
  const int gb = (int)((bh + 255) / 256) > 148 * 8 ? 148 * 8 : (int)((bh + 255) / 256);
  const int gw = (B + 63) / 64;
  dense_fwd_kernel<1, 64, true><<<gb, 256, 0, st>>>(x, P + MLP_P_W1, P + MLP_P_B1, H1, B);
  dense_fwd_kernel<64, 64, true><<<gb, 256, 0, st>>>(H1, P + MLP_P_W2, P + MLP_P_B2, H2, B);
  dense_fwd_kernel<64, 64, true><<<gb, 256, 0, st>>>(H2, P + MLP_P_W3, P + MLP_P_B3, H3, B);
  dense_fwd_kernel<64, 4, false><<<gb, 256, 0, st>>>(H3, P + MLP_P_W4, P + MLP_P_B4, Y, B);
  loss_kernel<<<64, 256, 0, st>>>(Y, t, B, dY, loss);
  dense_bwd_weight_kernel<64, 4><<<gw, 256, 0, st>>>(dY, H3, B, G + MLP_P_W4, G + MLP_P_B4);
  dense_bwd_data_kernel<64, 4><<<gb, 256, 0, st>>>(dY, P + MLP_P_W4, H3, dZ3, B);
  dense_bwd_weight_kernel<64, 64><<<gw, 256, 0, st>>>(dZ3, H2, B, G + MLP_P_W3, G + MLP_P_B3);
  dense_bwd_data_kernel<64, 64><<<gb, 256, 0, st>>>(dZ3, P + MLP_P_W3, H2, dZ2, B);
  dense_bwd_weight_kernel<64, 64><<<gw, 256, 0, st>>>(dZ2, H1, B, G + MLP_P_W2, G + MLP_P_B2);
  dense_bwd_data_kernel<64, 64><<<gb, 256, 0, st>>>(dZ2, P + MLP_P_W2, H1, dZ1, B);
  dense_bwd_weight_kernel<1, 64><<<gw, 256, 0, st>>>(dZ1, x, B, G + MLP_P_W1, G + MLP_P_B1);
}

void mlp_adam(float* params, const float* grads, float* m, float* v, int n, float lr, long long step,
              cudaStream_t st) {
  const float c1 = 1.0f / (1.0f - std::pow(0.9f, (float)step));
  const float c2 = 1.0f / (1.0f - std::pow(0.999f, (float)step));
  adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(params, grads, m, v, n, lr, c1, c2);
}

template <typename T>
void launch_mlp_props(const ThermoTab& tb, const MlpNorm& nm, const MlpSmall& sm, const MlpCheck& ck,
                      const uint16_t* wpack, const T* rhoh, T* h, T* t, T* k, T* d, T* m, int64_t n,
                      unsigned long long* nfallback, cudaStream_t st) {
  int64_t tiles = (n + 127) / 128;
  if (tiles > 148 * 6) tiles = 148 * 6;  // six CTAs per SM: 6 x 64 TMEM columns, 6 x 32 KB shared
  if (tiles < 1) tiles = 1;
  mlp_props_kernel<T><<<(unsigned)tiles, 128, 0, st>>>(tb, nm, sm, ck, wpack, rhoh, h, t, k, d, m, n, nfallback);
}
template void launch_mlp_props<double>(const ThermoTab&, const MlpNorm&, const MlpSmall&, const MlpCheck&,
                                       const uint16_t*, const double*, double*, double*, double*, double*, double*,
                                       int64_t, unsigned long long*, cudaStream_t);
template void launch_mlp_props<float>(const ThermoTab&, const MlpNorm&, const MlpSmall&, const MlpCheck&,
                                      const uint16_t*, const float*, float*, float*, float*, float*, float*,
                                      int64_t, unsigned long long*, cudaStream_t);

}  // namespace chs
