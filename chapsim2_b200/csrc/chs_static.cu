// Periodic 3D pressure Poisson solve that uses no device memory beyond a fixed module-level
// work array (chs_poisson_periodic_static in include/chapsim_gpu.h).
//
// The algorithm is the handle path's poisson_000 branch (src/poisson_1stderivcomp.f90:1016-1195):
// real FFT in x, complex FFTs in y and z, division by -(kx'^2 + ky'^2 + kz'^2) with the
// modified wavenumbers of the periodic C2P derivative of the chosen scheme
// (src/poisson_1stderivcomp.f90:2448-2503), and the inverse transforms.  The same kernels
// run; only the spectrum and the tables live in `g_static_work` instead of handle memory.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <memory>
#include <mutex>

#include "../../include/chapsim_gpu.h"
#include "chs_kernels.cuh"
#include "chs_plan.h"

namespace {

using namespace chs;

// Capacity: spectrum of nx/2+1 by ny by nz complex values, and FFT lengths up to kMaxLen.
constexpr size_t kSpecMax = size_t(1) << 20;  // complex values (16 MiB)
constexpr int kMaxLen = 4096;
// table region after the spectrum: three twiddle tables of kMaxLen complex values, then the
// three squared-wavenumber arrays of kMaxLen doubles (packed two per complex slot)
constexpr size_t kTabTw = 3 * (size_t)kMaxLen;
constexpr size_t kTabK2 = 3 * (size_t)kMaxLen / 2;
constexpr size_t kWorkLen = kSpecMax + kTabTw + kTabK2;
// 16 MiB of spectrum + 192 KiB of twiddles + 96 KiB of squared wavenumbers = 16 MiB + 288 KiB
static_assert(kWorkLen * sizeof(double2) == (size_t(16) << 20) + (size_t(288) << 10), "work array size");

__device__ __align__(256) double2 g_static_work[kWorkLen];

// Tables currently held by g_static_work, per device.  The array lives in the device context, so
// the key also records the context's unique id: after cudaDeviceReset (or any new primary context)
// the array comes back zeroed and the id differs, which forces the set-up to run again.
struct Key {
  bool valid;
  unsigned long long ctx_id;
  int nc[3];
  double len[3];
  int iacc;
};
// host staging of one device's tables (the set-up waits for the copies before it reuses them)
struct Staging {
  double2 tw[3][kMaxLen];
  double k2[3][kMaxLen];
};
constexpr int kMaxDevices = 64;
Key g_key[kMaxDevices];
std::unique_ptr<Staging> g_stage[kMaxDevices];
// one lock per device: a set-up that waits for its stream blocks only callers of the same device
std::mutex g_mu[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context, through the runtime's driver entry points
// (the library does not link the driver library directly).
cudaError_t current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  if (!get_current || !get_id) return cudaErrorNotSupported;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return cudaErrorDeviceUninitialized;
  if (get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorDeviceUninitialized;
  return cudaSuccess;
}

int fail(char* err, size_t errlen, int code, const char* fmt, ...) {
  if (err && errlen) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
  }
  return code;
}

bool radix_plan(int n, FftPlan& fp) {
  fp = FftPlan{};
  fp.n = n;
  int m = n;
  while (m % 4 == 0) { fp.radix[fp.nst++] = 4; m /= 4; }
  while (m % 2 == 0) { fp.radix[fp.nst++] = 2; m /= 2; }
  while (m % 3 == 0) { fp.radix[fp.nst++] = 3; m /= 3; }
  return m == 1;
}

void twiddles(int n, double2* tw) {
  const double pi = 3.141592653589793238462643383279502884;
  for (int k = 0; k < n; ++k) tw[k] = make_double2(std::cos(2.0 * pi * k / n), -std::sin(2.0 * pi * k / n));
}

// squared modified wavenumbers of the periodic C2P first derivative, as the handle path builds them
void mod_k2(int n, double len, double dh, int iacc, double* v) {
  const double pi = 2.0 * std::asin(1.0);
  const CoefSet& cs = coef(D1C2P, iacc);
  const double alc = cs.lhs[2][0][BC_PERIODIC];
  const double ac = cs.rhs[2][0][BC_PERIODIC] / dh, bc = cs.rhs[2][1][BC_PERIODIC] / dh;
  for (int i = 0; i < n; ++i) v[i] = 0.0;
  for (int i = 1; i <= n / 2 + 1; ++i) {
    const double w = 2.0 * pi * double(i - 1) / double(n);
    double wp = ac * 2.0 * dh * std::sin(w * 0.5) + bc * 2.0 * dh * std::sin(3.0 * 0.5 * w);
    wp = wp / (1.0 + 2.0 * alc * std::cos(w));
    const double q = double(n) * wp / len;
    v[i - 1] = q * q;
  }
  for (int i = n / 2 + 2; i <= n; ++i) v[i - 1] = v[n - i + 1];
}

}  // namespace

extern "C" int chs_poisson_periodic_static(double* d_rhs, const int nc[3], const double len[3], int iacc,
                                           void* stream, char* err, size_t errlen) {
  if (!d_rhs || !nc || !len) return fail(err, errlen, CHS_ERR_ARG, "null argument");
  if (iacc < 1 || iacc > 4)
    return fail(err, errlen, CHS_ERR_ARG, "iacc must be 1 (CD2) .. 4 (CP6), got %d", iacc);
  for (int d = 0; d < 3; ++d) {
    if (nc[d] < 2 || nc[d] > kMaxLen)
      return fail(err, errlen, CHS_ERR_ARG, "nc[%d] = %d outside 2..%d", d, nc[d], kMaxLen);
    if (!(len[d] > 0.0)) return fail(err, errlen, CHS_ERR_ARG, "len[%d] must be positive", d);
  }
  FftPlan fx, fy, fz;
  if (!radix_plan(nc[0], fx) || !radix_plan(nc[1], fy) || !radix_plan(nc[2], fz))
    return fail(err, errlen, CHS_ERR_ARG, "FFT lengths must be of the form 2^a 3^b (got %d %d %d)", nc[0], nc[1],
                nc[2]);
  const int nxh = nc[0] / 2 + 1;
  const size_t nspec = (size_t)nxh * nc[1] * nc[2];
  if (nspec > kSpecMax)
    return fail(err, errlen, CHS_ERR_ARG,
                "grid too large for the static work array: (nx/2+1)*ny*nz = %zu complex values, limit %zu", nspec,
                kSpecMax);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(err, errlen, CHS_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(err, errlen, CHS_ERR_ARG, "device ordinal %d not supported", dev);
  double2* work = nullptr;
  e = cudaGetSymbolAddress(reinterpret_cast<void**>(&work), g_static_work);
  if (e != cudaSuccess) return fail(err, errlen, CHS_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
  double2* spec = work;
  double2* tw = work + kSpecMax;
  double* k2 = reinterpret_cast<double*>(work + kSpecMax + kTabTw);
  fx.tw = tw;
  fy.tw = tw + kMaxLen;
  fz.tw = tw + 2 * kMaxLen;
  const double* k2x = k2;
  const double* k2y = k2 + kMaxLen;
  const double* k2z = k2 + 2 * kMaxLen;

  unsigned long long ctx_id = 0;
  e = current_context_id(&ctx_id);
  if (e != cudaSuccess) return fail(err, errlen, CHS_ERR_CUDA, "context id: %s", cudaGetErrorString(e));
  {
    // set-up: (re)write the tables when this device's context holds tables of another grid, or
    // none (a new context starts with a zeroed array)
    std::lock_guard<std::mutex> lock(g_mu[dev]);
    Key& k = g_key[dev];
    const bool same = k.valid && k.ctx_id == ctx_id && k.iacc == iacc && k.nc[0] == nc[0] && k.nc[1] == nc[1] &&
                      k.nc[2] == nc[2] && k.len[0] == len[0] && k.len[1] == len[1] && k.len[2] == len[2];
    if (!same) {
      k.valid = false;
      if (!g_stage[dev]) g_stage[dev] = std::make_unique<Staging>();
      Staging& sg = *g_stage[dev];
      const FftPlan* fp[3] = {&fx, &fy, &fz};
      for (int d = 0; d < 3; ++d) {
        twiddles(nc[d], sg.tw[d]);
        mod_k2(nc[d], len[d], len[d] / nc[d], iacc, sg.k2[d]);
        e = cudaMemcpyAsync(const_cast<double2*>(fp[d]->tw), sg.tw[d], nc[d] * sizeof(double2),
                            cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(k2 + (size_t)d * kMaxLen, sg.k2[d], nc[d] * sizeof(double), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return fail(err, errlen, CHS_ERR_CUDA, "table upload: %s", cudaGetErrorString(e));
      }
      // the staging arrays are reused by this device's next set-up
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return fail(err, errlen, CHS_ERR_CUDA, "table upload: %s", cudaGetErrorString(e));
      k.valid = true;
      k.ctx_id = ctx_id;
      k.iacc = iacc;
      for (int d = 0; d < 3; ++d) {
        k.nc[d] = nc[d];
        k.len[d] = len[d];
      }
    }
  }

  const int n0 = nc[0], n1 = nc[1], n2 = nc[2];
  try {
    launch_rfft_x(fx, d_rhs, spec, n1 * n2, st);
    launch_cfft_axis(fy, spec, nxh, n2, (int64_t)nxh * n1, nxh, -1, st);
    launch_cfft_axis(fz, spec, nxh, n1, nxh, (int64_t)nxh * n1, -1, st);
    launch_spectral_divide(spec, nxh, n1, n2, k2x, k2y, k2z, 1.0 / ((double)n0 * (double)n1 * (double)n2), st);
    launch_cfft_axis(fz, spec, nxh, n1, nxh, (int64_t)nxh * n1, +1, st);
    launch_cfft_axis(fy, spec, nxh, n2, (int64_t)nxh * n1, nxh, +1, st);
    launch_irfft_x(fx, spec, d_rhs, n1 * n2, 1.0, st);
  } catch (const std::exception& ex) {
    return fail(err, errlen, CHS_ERR_ARG, "%s", ex.what());
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(err, errlen, CHS_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
  return CHS_OK;
}
