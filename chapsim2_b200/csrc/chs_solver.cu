// Handle, device state and the RK3 substep of the B200 CHAPSim2 hot path,
// behind the C ABI of include/chapsim_gpu.h.
//
// Substep structure (Solve_momentum_eq, src/eq_momentum2.f90:1799-1932):
//   1. derived velocity quantities (interpolations/derivatives, :347-508),
//   2. momentum RHS terms accumulated straight into mx/my/mz and px/py/pz
//      (x :796-966, y :978-1242, z :1262-1457), products evaluated while the
//      operator tiles are staged,
//   3. fractional step (:35-71), mass-flux driving (:1547-1562),
//   4. q += rhs, wall enforcement (src/bc_dirichlet.f90:461-516),
//   5. Poisson RHS (:1663-1718), Poisson solve, p += phi, projection (:1577-1660).
// All state stays in HBM; the substep is captured once into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/chapsim_gpu.h"
#include "chs_fused.cuh"
#include "chs_kernels.cuh"
#include "chs_mlp.cuh"
#include "chs_plan.h"

using namespace chs;

namespace {

enum { V_QX = 0, V_QY = 1, V_QZ = 2, V_PR = 3, V_TM = 4 };
enum { JSELF = 0, JGRAD = 1, JPROD = 2 };

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define CK(x)                                                                                     \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));      \
  } while (0)

// build_bc_symm_operation (src/bc_general.f90:455-509)
void symm_op(const int ibc[2], int mbc[2][3], const int* jbc) {
  for (int i = 0; i < 2; ++i) mbc[i][0] = mbc[i][1] = mbc[i][2] = ibc[i];
  for (int i = 0; i < 2; ++i) {
    if (jbc) {
      const int a = ibc[i], b = jbc[i];
      if ((a == BC_SYMMETRIC || a == BC_ASYMMETRIC) && (b == BC_SYMMETRIC || b == BC_ASYMMETRIC)) {
        mbc[i][JPROD] = (a == b) ? BC_SYMMETRIC : BC_ASYMMETRIC;
      } else if (a != b) {
        if (a == BC_DIRICHLET) mbc[i][0] = mbc[i][1] = mbc[i][2] = a;
        if (b == BC_DIRICHLET) mbc[i][0] = mbc[i][1] = mbc[i][2] = b;
      }
    } else {
      if (ibc[i] == BC_SYMMETRIC) { mbc[i][JGRAD] = BC_ASYMMETRIC; }
      else if (ibc[i] == BC_ASYMMETRIC) { mbc[i][JGRAD] = BC_SYMMETRIC; mbc[i][JPROD] = BC_SYMMETRIC; }
    }
  }
}
struct Pair { int v[2]; };
Pair prod_of(const int a[2], const int b[2]) {
  int m[2][3];
  symm_op(a, m, b);
  return Pair{{m[0][JPROD], m[1][JPROD]}};
}
Pair tau_of(const int var[2], const int ftp[2]) {
  int m[2][3];
  symm_op(var, m, nullptr);
  int g[2] = {m[0][JGRAD], m[1][JGRAD]};
  return prod_of(ftp, g);
}

// complex FFT plan: radix 4s, then 2, then 3s
FftPlan make_fft(int n, std::vector<double2>& tw_host) {
  FftPlan fp{};
  fp.n = n;
  int m = n;
  fp.nst = 0;
  while (m % 4 == 0) { fp.radix[fp.nst++] = 4; m /= 4; }
  while (m % 2 == 0) { fp.radix[fp.nst++] = 2; m /= 2; }
  while (m % 3 == 0) { fp.radix[fp.nst++] = 3; m /= 3; }
  if (m != 1) throw std::runtime_error("FFT length must be of the form 2^a 3^b");
  tw_host.resize(n);
  const double pi = 3.141592653589793238462643383279502884;
  for (int k = 0; k < n; ++k) tw_host[k] = make_double2(std::cos(2.0 * pi * k / n), -std::sin(2.0 * pi * k / n));
  return fp;
}

}  // namespace

struct chs_handle {
  // configuration
  int nc[3], np[3];
  bool periodic_y, stretch_y;
  int iacc, ifft, idriven;
  bool mixed = false;  // FP32 fields and operators, FP64 Poisson / mass flux / diagnostics
  double h[3];
  double dt, rre, sigma2p;
  double tGamma[4], tZeta[4], tAlpha[4];
  int ibc[3][5][2];
  double fbcy[5][2];
  Pair mbcx_cov1, mbcy_cov1, mbcz_cov1, mbcx_tau1, mbcy_tau1, mbcz_tau1;
  Pair mbcx_cov2, mbcy_cov2, mbcz_cov2, mbcx_tau2, mbcy_tau2, mbcz_tau2;
  Pair mbcx_cov3, mbcy_cov3, mbcz_cov3, mbcx_tau3, mbcy_tau3, mbcz_tau3;
  bool fbcy_velo = false;
  std::vector<double> mpcc, mppt;

  // device
  int device = 0;
  cudaStream_t st = nullptr;
  PlanBook book;
  std::map<std::tuple<int, int, int, int, int>, OpPlan> plans;
  double* table = nullptr;
  std::vector<std::pair<void*, size_t>> allocs;
  int tune_block = 0, tune_lt = 0;  // launch shapes picked by chs_autotune (0 = defaults)
  int tune_fuse = 0;                // 1: fused operator sums (chs_autotune decides; off by default)
  // fused substep kernels for the explicit schemes (chs_fused.cu): 1 on by default, 0 the
  // operator-by-operator path (chs_set_fusion)
  int kfuse = 1;
  // >= 0 while chs_profile_class captures a substep: launches of other kernel classes are left out
  int only_kind = -1;
  FzRow* fz_rows = nullptr;  // device row tables of the y operators (chs_fused.cuh)
  double* fz_part = nullptr;  // per-CTA partial sums of the mass-flux mean from the fused x pass
  // plan key -> first row of its table in fz_rows (-1: no table: periodic, or not representable)
  std::map<std::tuple<int, int, int, int, int>, int> fz_index;
  long long launches = 0;
  std::string err;

  size_t n_pcc, n_cpc, n_ccp, n_ccc, n_ppc, n_pcp, n_cpp;
  double *qx, *qy, *qz, *pres, *pcor;
  double *mx0, *my0, *mz0, *mx, *my, *mz, *px, *py, *pz;
  double *qxix, *qxdx, *qxdy, *qxiy, *qxiz, *qxdz;
  double *qydx, *qyix, *qydy, *qyiy, *qydz, *qyiz;
  double *qzdx, *qzix, *qziy, *qzdy, *qziz, *qzdz;
  double *div, *qxdx_cpc, *qydy_cpc, *qzdz_cpc;
  double *fb_qx, *fb_qy, *fb_qz, *fb_pr, *fb_mpr, *fb_conv2, *fb_visc2, *fb_comb, *fb_maxp;
  double *wy, *partial, *scal;
  double* stage = nullptr;  // mixed precision: FP64 staging for host transfers
  // variable-property (thermal) state: src/modules.f90:412-681
  bool thermo = false;
  ThermoTab tab{};
  double rPrRen = 0.0;
  double *gx = nullptr, *gy = nullptr, *gz = nullptr;
  double *rhoh = nullptr, *hEnth = nullptr, *tTemp = nullptr, *kCond = nullptr, *dDens = nullptr, *mVisc = nullptr;
  double *erhs = nullptr, *erhs0 = nullptr;
  double *gxix = nullptr, *gxiy = nullptr, *gxiz = nullptr, *gyix = nullptr, *gyiy = nullptr, *gyiz = nullptr;
  double *gzix = nullptr, *gziy = nullptr, *gziz = nullptr;
  double *muiy_cpc = nullptr, *muixy_ppc = nullptr, *mu_pcc = nullptr, *muixz_pcp = nullptr, *muiyz_cpp = nullptr;
  double *h_pcc = nullptr, *h_cpc = nullptr, *h_ccp = nullptr, *k_pcc = nullptr, *k_cpc = nullptr, *k_ccp = nullptr;
  double *dTx = nullptr, *dTy = nullptr, *dTz = nullptr, *dh_cpc = nullptr;
  double *fb_h = nullptr, *fb_k = nullptr, *fb_m = nullptr, *fb_d = nullptr, *fb_qw = nullptr, *fb_zero = nullptr;
  double *fb_dtk = nullptr;
  Pair ebcx_conv, ebcy_conv, ebcz_conv, ebcx_difu, ebcy_difu, ebcz_difu, ftpy;
  // MLP surrogate of the property update
  bool mlp_ready = false;
  int mlp_mode = 0;  // 0: table lookups (the reference's method), 1: network with table fallback
  float* mlp_params = nullptr;
  uint16_t* mlp_wpack = nullptr;
  unsigned long long* mlp_nfb = nullptr;
  MlpNorm mlp_norm{};
  MlpSmall mlp_small{};
  MlpCheck mlp_check{};
  std::vector<double> tab_host_t, tab_host_rhoh;
  // running statistics (post_statistics.f90): 0 pr, 1-3 u, 4-9 uu vv ww uv uw vw, 10 T, 11 TT
  double* stat[12] = {};
  double vol = 0.0;
  int npart = 0;
  // Poisson
  FftPlan fx{}, fy{}, fz{};
  double2* spec = nullptr;
  double *lamx = nullptr, *lamz = nullptr, *pa = nullptr, *pb = nullptr, *pc = nullptr;
  double *yzr = nullptr, *yd = nullptr;  // precomputed y-solve factors
  double *k2x = nullptr, *k2y = nullptr, *k2z = nullptr;
  double *ayby = nullptr, *ptab = nullptr;  // poisson_010 cosine factors and pentadiagonal rows
  double* pfac = nullptr;                   // and the elimination factors per (kx, |kz|)
  // graphs per substep (1..3) and for a whole step
  cudaGraphExec_t gexec[4] = {nullptr, nullptr, nullptr, nullptr};
  // the energy and momentum parts of substeps 1..3 as separate graphs (host-array pipeline)
  cudaGraphExec_t gpart[2][4] = {{nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
  long long kernels_per_part[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
  long long kernels_per_sub[4] = {0, 0, 0, 0};
  bool capturing = false;
  // Dataflow scheduling of a captured substep.  Each launch names the buffers it reads and
  // writes; it goes to one of up to kLanes streams and waits (by event) only for the launches it
  // depends on: the last writer of every buffer it touches and, for the buffers it writes, the
  // readers since that write.  The captured graph then holds the true dependency edges, so
  // independent operators (the derived velocity gradients, the three momentum components, the
  // energy fluxes) run concurrently and fill each other's ramp-up and tail.  Every node keeps a
  // vector clock (per lane, the latest node of that lane it already follows); a launch goes to a
  // lane whose last node it already follows, so stream order adds no false edge when one exists.
  // Launches that name no buffers act as barriers.  Only active while a substep graph is
  // captured; eager runs stay on `st` in program order.
  static constexpr int kLanes = 8;
  // lanes used by the next capture (1: one stream, program order).  Measured fastest on the
  // 128x96x128 channel and heated-channel substeps: three for FP64 fields, four for FP32 (20-25 %
  // over one lane; more lanes lose again).  Set with the precision in setup_host.
  int dag_lanes = 3;
  cudaStream_t lane[kLanes] = {};
  bool dag_on = false;
  struct BufSpan { uintptr_t lo, hi; int id; };
  struct BufState { int writer = -1; std::vector<int> readers; };
  struct Clock { int v[kLanes]; };
  std::vector<BufSpan> spans;
  std::vector<BufState> bstate;
  std::vector<int> node_lane;
  std::vector<Clock> node_vc;
  std::vector<cudaEvent_t> evpool;
  int lane_last[kLanes];
  int fence = -1, cur_node = -1;
  struct Bufs { const void* p[16]; int n = 0; };
  std::vector<int> pend_r, pend_w, deps;
  int buf_id(const void* q) const {
    const uintptr_t a = reinterpret_cast<uintptr_t>(q);
    size_t lo = 0, hi = spans.size();
    while (lo < hi) {
      const size_t m = (lo + hi) / 2;
      if (spans[m].hi <= a) lo = m + 1;
      else hi = m;
    }
    if (lo < spans.size() && spans[lo].lo <= a && a < spans[lo].hi) return spans[lo].id;
    return (int)spans.size();  // not a handle buffer: one shared id, ordered conservatively
  }
  cudaEvent_t node_event(int n) {
    while ((int)evpool.size() <= n) {
      cudaEvent_t e;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      evpool.push_back(e);
    }
    return evpool[n];
  }
  // vector clock of a node that follows the nodes in `ds`
  Clock clock_after(const std::vector<int>& ds) const {
    Clock c;
    for (int l = 0; l < kLanes; ++l) c.v[l] = -1;
    for (int d : ds) {
      for (int l = 0; l < kLanes; ++l) c.v[l] = std::max(c.v[l], node_vc[d].v[l]);
      c.v[node_lane[d]] = std::max(c.v[node_lane[d]], d);
    }
    return c;
  }
  void dag_start() {
    if (dag_lanes <= 1) return;
    for (int l = 1; l < dag_lanes; ++l)
      if (!lane[l]) CK(cudaStreamCreateWithFlags(&lane[l], cudaStreamNonBlocking));
    lane[0] = st;
    spans.clear();
    for (size_t i = 0; i < allocs.size(); ++i) {
      const uintptr_t a = reinterpret_cast<uintptr_t>(allocs[i].first);
      spans.push_back(BufSpan{a, a + allocs[i].second, (int)i});
    }
    std::sort(spans.begin(), spans.end(), [](const BufSpan& x, const BufSpan& y) { return x.lo < y.lo; });
    bstate.assign(spans.size() + 1, BufState{});
    // node 0: the fork on the capturing stream; every lane starts after it
    node_lane.assign(1, 0);
    node_vc.assign(1, Clock{});
    for (int l = 0; l < kLanes; ++l) node_vc[0].v[l] = -1;
    CK(cudaEventRecord(node_event(0), st));
    for (int l = 1; l < dag_lanes; ++l) CK(cudaStreamWaitEvent(lane[l], node_event(0), 0));
    for (int l = 0; l < kLanes; ++l) lane_last[l] = l == 0 ? 0 : -1;
    fence = 0;
    cur_node = -1;
    dag_on = true;
  }
  // join every lane back into the capturing stream (also on error paths, before the capture ends)
  void dag_stop() {
    if (!dag_on) return;
    dag_on = false;
    const Clock& c0 = node_vc[lane_last[0]];
    for (int l = 1; l < dag_lanes; ++l)
      if (lane_last[l] > c0.v[l]) cudaStreamWaitEvent(st, node_event(lane_last[l]), 0);
  }
  // make lane `ln` wait for the nodes in ds; returns the new node's clock
  Clock join_into(int ln, std::vector<int>& ds) {
    std::sort(ds.begin(), ds.end(), std::greater<int>());
    ds.erase(std::unique(ds.begin(), ds.end()), ds.end());
    Clock have;
    for (int l = 0; l < kLanes; ++l) have.v[l] = -1;
    if (lane_last[ln] >= 0) {
      have = node_vc[lane_last[ln]];
      have.v[ln] = lane_last[ln];
    }
    for (int d : ds) {
      const int L = node_lane[d];
      if (have.v[L] >= d) continue;  // already follows d (stream order or an earlier wait)
      CK(cudaStreamWaitEvent(lane[ln], node_event(d), 0));
      for (int l = 0; l < kLanes; ++l) have.v[l] = std::max(have.v[l], node_vc[d].v[l]);
      have.v[L] = std::max(have.v[L], d);
    }
    return have;
  }
  cudaStream_t dag_begin(const Bufs& R, const Bufs& W) {
    if (!dag_on) return st;
    pend_r.clear();
    pend_w.clear();
    for (int i = 0; i < R.n; ++i)
      if (R.p[i]) pend_r.push_back(buf_id(R.p[i]));
    for (int i = 0; i < W.n; ++i)
      if (W.p[i]) pend_w.push_back(buf_id(W.p[i]));
    deps.assign(1, fence);
    for (int b : pend_r)
      if (bstate[b].writer >= 0) deps.push_back(bstate[b].writer);
    for (int b : pend_w) {
      if (bstate[b].writer >= 0) deps.push_back(bstate[b].writer);
      for (int r : bstate[b].readers) deps.push_back(r);
    }
    const Clock need = clock_after(deps);
    // a lane whose last node the launch already follows adds no false edge; prefer the lane of the
    // latest dependency (no wait needed for it), else the lane idle longest
    int latest = *std::max_element(deps.begin(), deps.end());
    int ln = -1;
    if (lane_last[node_lane[latest]] == latest) ln = node_lane[latest];
    for (int l = 0; l < dag_lanes && ln < 0; ++l)
      if (lane_last[l] <= need.v[l]) ln = l;
    if (ln < 0) {
      ln = 0;
      for (int l = 1; l < dag_lanes; ++l)
        if (lane_last[l] < lane_last[ln]) ln = l;
    }
    const Clock c = join_into(ln, deps);
    cur_node = (int)node_lane.size();
    node_lane.push_back(ln);
    node_vc.push_back(c);
    return lane[ln];
  }
  void dag_end() {
    if (!dag_on) return;
    const int n = cur_node, ln = node_lane[n];
    CK(cudaEventRecord(node_event(n), lane[ln]));
    lane_last[ln] = n;
    for (int b : pend_r) bstate[b].readers.push_back(n);
    for (int b : pend_w) {
      bstate[b].writer = n;
      bstate[b].readers.clear();
    }
    cur_node = -1;
  }
  // a launch that names no buffers: runs on `st` after everything before it, and everything after
  // it waits for it
  cudaStream_t dag_barrier_begin() {
    if (!dag_on) return st;
    deps.clear();
    for (int l = 0; l < dag_lanes; ++l)
      if (lane_last[l] >= 0) deps.push_back(lane_last[l]);
    const Clock c = join_into(0, deps);
    cur_node = (int)node_lane.size();
    node_lane.push_back(0);
    node_vc.push_back(c);
    return st;
  }
  void dag_barrier_end() {
    if (!dag_on) return;
    const int n = cur_node;
    CK(cudaEventRecord(node_event(n), st));
    lane_last[0] = n;
    for (auto& b : bstate) {
      b.writer = -1;
      b.readers.clear();
    }
    fence = n;
    cur_node = -1;
  }

  // per-kernel profiling (chs_profile_substep)
  bool profiling = false;
  struct Rec { int kind, dir; double bytes; cudaEvent_t e0, e1; };
  std::vector<Rec> recs;
  // while a profiled substep is captured, the events become event-record nodes of the graph
  void prof_record(cudaEvent_t e) {
    if (capturing) CK(cudaEventRecordWithFlags(e, st, cudaEventRecordExternal));
    else CK(cudaEventRecord(e, st));
  }
  cudaEvent_t prof_begin() {
    cudaEvent_t e = nullptr;
    if (profiling) { CK(cudaEventCreate(&e)); prof_record(e); }
    return e;
  }
  void prof_end(cudaEvent_t e0, int kind, int dir, double bytes) {
    if (!profiling) return;
    cudaEvent_t e1;
    CK(cudaEventCreate(&e1));
    prof_record(e1);
    recs.push_back(Rec{kind, dir, bytes, e0, e1});
  }

  template <class T>
  T* dalloc(size_t n) {
    void* p = nullptr;
    CK(cudaMalloc(&p, n * sizeof(T) + 64));
    CK(cudaMemsetAsync(p, 0, n * sizeof(T) + 64, st));
    allocs.push_back({p, n * sizeof(T) + 64});
    return static_cast<T*>(p);
  }
  const OpPlan& plan(int d, int fam, Pair bc, bool has_fbc) {
    auto key = std::make_tuple(d, fam, bc.v[0], bc.v[1], has_fbc ? 1 : 0);
    auto it = plans.find(key);
    if (it != plans.end()) return it->second;
    if (capturing) throw std::runtime_error("operator plan missing from the prepared set");
    OpPlan p = book.make(d, fam, bc.v, has_fbc);
    return plans.emplace(key, p).first->second;
  }
};

// buffers a launch reads or writes (null entries are ignored)
template <class... Ps>
chs_handle::Bufs bufs(Ps... ps) {
  static_assert(sizeof...(Ps) <= 16, "too many buffers");
  chs_handle::Bufs b;
  ((b.p[b.n++] = static_cast<const void*>(ps)), ...);
  return b;
}

namespace {

Pair P2(const int v[2]) { return Pair{{v[0], v[1]}}; }
void upload_table(chs_handle* H);

template <class T>
struct Id { using type = T; };

// parts of a substep: the energy equation (variable-property runs) and the momentum equation
enum { PART_ENERGY = 1, PART_MOMENTUM = 2, PART_ALL = 3 };
const int kPer2[2] = {BC_PERIODIC, BC_PERIODIC};

// input expression: up to two terms (see LineIOT)
template <typename T>
struct SrcT {
  TermT<T> t[2] = {{nullptr, nullptr, T_NONE, 0.0, 0.0}, {nullptr, nullptr, T_NONE, 0.0, 0.0}};
  int narrays() const {
    int n = 0;
    for (const auto& x : t) n += (x.X ? 1 : 0) + (x.Y ? 1 : 0) + (x.Z ? 1 : 0);
    return n;
  }
};
template <typename T>
SrcT<T> src(const T* a, double s = 1.0) { SrcT<T> x; x.t[0] = TermT<T>{a, nullptr, T_X, s, 0.0}; return x; }
template <typename T>
SrcT<T> prod(const T* a, const T* b, double s) { SrcT<T> x; x.t[0] = TermT<T>{a, b, T_XY, s, 0.0}; return x; }
template <typename T>
SrcT<T> lin(const T* a, const T* b, double c1, double s) {
  SrcT<T> x; x.t[0] = TermT<T>{a, b, T_XpY, s, c1}; return x;
}
// s * (a + c1*b) * m, or lin(a, b, c1, s) when m is null (constant properties: mu = 1)
template <typename T>
SrcT<T> linm(const T* a, const T* b, double c1, double s, const T* m) {
  SrcT<T> x;
  x.t[0] = m ? TermT<T>{a, b, T_XpYZ, s, c1, m} : TermT<T>{a, b, T_XpY, s, c1};
  return x;
}
// a + w * b, for two single-term expressions
template <typename T>
SrcT<T> plus(const SrcT<T>& a, const SrcT<T>& b, double w) {
  SrcT<T> x = a;
  x.t[1] = b.t[0];
  x.t[1].s *= w;
  return x;
}

// the RK3 fractional step an O_FRAC operator applies to its output (see OutMode)
template <typename T>
struct FracStep {
  T* rhs0;
  T* qupd;
  double dt, gam, zeta, alpha;
};

// run one operator: direction d, family fam, operation bc, boundary planes fbc (null = absent)
template <typename T>
void run_op(chs_handle* H, int d, int fam, Pair bc, const typename Id<T>::type* fbc, const SrcT<T>& in,
            const int n_in[3], T* out, bool accumulate, double g, int omode = O_STORE,
            const typename Id<T>::type* onum = nullptr, const FracStep<T>* frac = nullptr) {
  const size_t tsz = H->book.table.size();
  const OpPlan& P = H->plan(d, fam, bc, fbc != nullptr);
  if (H->book.table.size() != tsz) upload_table(H);
  LineIOT<T> io{};
  io.t[0] = in.t[0];
  io.t[1] = in.t[1];
  io.fbc = fbc;
  io.out = out;
  io.accumulate = accumulate ? 1 : 0;
  io.g = g;
  io.n1 = n_in[0]; io.n2 = n_in[1]; io.n3 = n_in[2];
  io.omode = omode;
  io.onum = onum;
  io.block = H->tune_block;
  io.lt_max = H->tune_lt;
  if (omode == O_FRAC) {
    if (!frac) throw std::logic_error("O_FRAC operator without its fractional-step data");
    io.rhs0 = frac->rhs0;
    io.qupd = frac->qupd;
    io.dt = frac->dt; io.gam = frac->gam; io.zeta = frac->zeta; io.alpha = frac->alpha;
  }
  const double nin_tot = (double)n_in[0] * n_in[1] * n_in[2];
  const double nout_tot = nin_tot / P.nin * P.nout;
  const int narr = in.narrays();
  const double nrw = omode == O_FRAC ? (io.qupd ? 6.0 : 4.0) : ((accumulate || omode != O_STORE) ? 2.0 : 1.0);
  const double bytes = (double)sizeof(T) * (narr * nin_tot + nrw * nout_tot);
  const bool rmw = accumulate || omode == O_FRAC;
  if (H->only_kind >= 0 && H->only_kind != 0) return;
  cudaStream_t s = H->dag_begin(bufs(io.t[0].X, io.t[0].Y, io.t[0].Z, io.t[1].X, io.t[1].Y, io.t[1].Z, io.fbc, io.onum,
                                     rmw ? out : nullptr),
                                bufs(out, io.rhs0, io.qupd));
  cudaEvent_t e0 = H->prof_begin();
  launch_line_op(d, P, io, H->table, s);
  H->prof_end(e0, 0, d, bytes);
  H->dag_end();
  H->launches++;
}

// profile wrapper for the other kernel classes; without a buffer list the launch is a barrier of
// the dataflow schedule
#define PROF(H, kind, bytes, ...)                       \
  do {                                                   \
    if ((H)->only_kind >= 0 && (H)->only_kind != (kind)) break; \
    (H)->dag_barrier_begin();                            \
    cudaEvent_t e0_ = (H)->prof_begin();                 \
    __VA_ARGS__;                                         \
    (H)->prof_end(e0_, kind, -1, (bytes));               \
    (H)->dag_barrier_end();                              \
  } while (0)
// the same with the buffers read (R) and written (W); the launch expression uses `st`, which here
// names the lane the schedule picked
#define PROFD(H, kind, bytes, R, W, ...)                 \
  do {                                                   \
    if ((H)->only_kind >= 0 && (H)->only_kind != (kind)) break; \
    cudaStream_t st = (H)->dag_begin(R, W);              \
    cudaEvent_t e0_ = (H)->prof_begin();                 \
    __VA_ARGS__;                                         \
    (H)->prof_end(e0_, kind, -1, (bytes));               \
    (H)->dag_end();                                      \
  } while (0)

// op(a; fbc1) + w*op(b; fbc2).  When both terms use the same plan the sum runs as one launch
// on the combined input (the operator is linear in its input and boundary values); fcomb must
// then hold fbc1 + w*fbc2 when the two planes differ.
template <typename T>
void run_pair(chs_handle* H, int d, int fam, Pair bc1, const typename Id<T>::type* f1, const SrcT<T>& a, Pair bc2,
              const typename Id<T>::type* f2, const SrcT<T>& b, double w, const int n_in[3], T* out, bool accumulate,
              const typename Id<T>::type* fcomb) {
  const bool same = bc1.v[0] == bc2.v[0] && bc1.v[1] == bc2.v[1] && ((f1 == nullptr) == (f2 == nullptr)) &&
                    (f1 == f2 || fcomb != nullptr);
  if (same) {
    const T* f = (f1 == f2) ? f1 : fcomb;
    run_op<T>(H, d, fam, bc1, f, plus(a, b, w), n_in, out, accumulate, 1.0);
  } else {
    run_op<T>(H, d, fam, bc1, f1, a, n_in, out, accumulate, 1.0);
    run_op<T>(H, d, fam, bc2, f2, b, n_in, out, true, w);
  }
}

// One term of a fused sum: operator (direction, family, boundary pair, planes), input
// expression, input extents, weight and group (0 flux, 1 pressure gradient)
template <typename T>
struct OpTerm {
  int d, fam;
  Pair bc;
  const T* fbc;
  SrcT<T> in;
  int n_in[3];
  double g;
  int group;
};

template <typename T>
OpTerm<T> term(int d, int fam, Pair bc, const T* fbc, const SrcT<T>& in, const int n_in[3], double g, int group) {
  return OpTerm<T>{d, fam, bc, fbc, in, {n_in[0], n_in[1], n_in[2]}, g, group};
}

// the terms of op(a; f1) + w*op(b; f2), merged into one when they share a plan (as run_pair)
template <typename T>
void pair_terms(std::vector<OpTerm<T>>& v, int d, int fam, Pair bc1, const typename Id<T>::type* f1,
                const SrcT<T>& a, Pair bc2, const typename Id<T>::type* f2, const SrcT<T>& b, double w,
                const int n_in[3], const typename Id<T>::type* fcomb, int group) {
  const bool same = bc1.v[0] == bc2.v[0] && bc1.v[1] == bc2.v[1] && ((f1 == nullptr) == (f2 == nullptr)) &&
                    (f1 == f2 || fcomb != nullptr);
  if (same) {
    v.push_back(term<T>(d, fam, bc1, (f1 == f2) ? f1 : fcomb, plus(a, b, w), n_in, 1.0, group));
  } else {
    v.push_back(term<T>(d, fam, bc1, f1, a, n_in, 1.0, group));
    v.push_back(term<T>(d, fam, bc2, f2, b, n_in, w, group));
  }
}

// Sum of explicit operators with an epilogue, as one fused launch when every plan is explicit
// (no line solve) and the terms fit, else as the equivalent sequence of line operators followed by
// the elementwise epilogue.  out has extents m; for EP_FRAC the fallback puts the pressure
// gradient in pfc_scratch.
template <typename T>
bool run_fused(chs_handle* H, const std::vector<OpTerm<T>>& terms, T* out, const int m[3], int epilogue, T* rhs0,
               int isub, T* pfc_scratch, T* rhoh = nullptr, bool props = false, bool prefer_fused = false,
               T* qupd = nullptr) {
  const size_t tsz = H->book.table.size();
  bool fuse = (H->tune_fuse || prefer_fused) && !terms.empty() && (int)terms.size() <= kMaxFusedTerms;
  for (const auto& t : terms) {
    const OpPlan& P = H->plan(t.d, t.fam, t.bc, t.fbc != nullptr);
    if (P.tdma || (t.fam != D1C2P && t.fam != D1P2C)) fuse = false;
  }
  if (H->book.table.size() != tsz) upload_table(H);
  const double nout = (double)m[0] * m[1] * m[2];
  if (fuse) {
    FusedIO<T> F{};
    F.nterm = (int)terms.size();
    double bytes = 0.0;
    for (int i = 0; i < F.nterm; ++i) {
      const OpTerm<T>& t = terms[i];
      FusedTerm<T>& ft = F.term[i];
      ft.P = H->plan(t.d, t.fam, t.bc, t.fbc != nullptr);
      ft.dir = t.d;
      ft.t[0] = t.in.t[0];
      ft.t[1] = t.in.t[1];
      ft.fbc = t.fbc;
      ft.n1 = t.n_in[0]; ft.n2 = t.n_in[1]; ft.n3 = t.n_in[2];
      ft.nlines = (int)num_lines(t.d, t.n_in[0], t.n_in[1], t.n_in[2]);
      ft.g = t.g;
      ft.group = t.group;
      bytes += (double)sizeof(T) * t.in.narrays() * t.n_in[0] * t.n_in[1] * t.n_in[2];
    }
    F.out = out;
    F.m1 = m[0]; F.m2 = m[1]; F.m3 = m[2];
    F.epilogue = epilogue;
    F.rhs0 = rhs0;
    F.dt = H->dt; F.gam = H->tGamma[isub]; F.zeta = H->tZeta[isub]; F.alpha = H->tAlpha[isub];
    F.rhoh = rhoh;
    F.props = props ? 1 : 0;
    if (props) {
      const int n = (int)H->n_ccc;
      (void)n;
      F.h = reinterpret_cast<T*>(H->hEnth); F.t = reinterpret_cast<T*>(H->tTemp);
      F.k = reinterpret_cast<T*>(H->kCond); F.d = reinterpret_cast<T*>(H->dDens);
      F.m = reinterpret_cast<T*>(H->mVisc);
      F.tab = H->tab;
    }
    const double ob = epilogue == EP_STORE ? 1.0 : epilogue == EP_ACCUM ? 2.0 : epilogue == EP_FRAC ? 3.0
                                                                          : (props ? 9.0 : 4.0);
    bytes += (double)sizeof(T) * ob * nout;
    chs_handle::Bufs rd, wr;
    for (const auto& t : terms) {
      for (int q = 0; q < 2; ++q)
        for (const void* a : {(const void*)t.in.t[q].X, (const void*)t.in.t[q].Y, (const void*)t.in.t[q].Z})
          if (a) rd.p[rd.n++] = a;
      if (t.fbc) rd.p[rd.n++] = t.fbc;
    }
    wr.p[wr.n++] = out;
    for (const void* a : {(const void*)rhs0, (const void*)rhoh}) if (a) wr.p[wr.n++] = a;
    if (props)
      for (const void* a : {(const void*)H->hEnth, (const void*)H->tTemp, (const void*)H->kCond,
                            (const void*)H->dDens, (const void*)H->mVisc})
        wr.p[wr.n++] = a;
    if (H->only_kind >= 0 && H->only_kind != 0) return false;
    cudaStream_t ls = H->dag_begin(rd, wr);
    cudaEvent_t e0 = H->prof_begin();
    launch_fused(F, H->table, ls);
    H->prof_end(e0, 0, -1, bytes);
    H->dag_end();
    H->launches++;
    return false;
  }
  // fallback: one line operator per term, then the elementwise epilogue.  A fractional step with
  // one pressure-gradient term that comes last runs as that operator's O_FRAC store (no separate
  // gradient array, no separate pass), and then also advances qupd when given.
  int n1 = 0;
  for (const auto& t : terms) n1 += t.group == 1 ? 1 : 0;
  const bool frac_in_op = epilogue == EP_FRAC && n1 == 1 && terms.back().group == 1 && terms.front().group == 0;
  T* tgt0 = out;
  bool first0 = epilogue != EP_ACCUM, first1 = true;
  for (const auto& t : terms) {
    if (t.group == 0) {
      run_op<T>(H, t.d, t.fam, t.bc, t.fbc, t.in, t.n_in, tgt0, !first0, t.g);
      first0 = false;
    } else if (frac_in_op) {
      const FracStep<T> fs{rhs0, qupd, H->dt, H->tGamma[isub], H->tZeta[isub], H->tAlpha[isub]};
      run_op<T>(H, t.d, t.fam, t.bc, t.fbc, t.in, t.n_in, out, false, t.g, O_FRAC, nullptr, &fs);
    } else {
      run_op<T>(H, t.d, t.fam, t.bc, t.fbc, t.in, t.n_in, pfc_scratch, !first1, t.g);
      first1 = false;
    }
  }
  if (frac_in_op) return qupd != nullptr;
  if (epilogue == EP_FRAC) {
    PROFD(H, 3, 5.0 * sizeof(T) * nout, bufs(pfc_scratch), bufs(out, rhs0),
         launch_fractional_step(out, rhs0, pfc_scratch, (int64_t)nout, H->dt, H->tGamma[isub], H->tZeta[isub],
                                H->tAlpha[isub], st));
    H->launches++;
  } else if (epilogue == EP_ENERGY && props) {
    // fractional step, rho*h update and table property update in one pass
    PROFD(H, 3, 10.0 * sizeof(T) * nout, bufs(), bufs(out, rhs0, rhoh, H->hEnth, H->tTemp, H->kCond, H->dDens, H->mVisc),
          launch_energy_advance_props<T>(H->tab, out, rhs0, rhoh, reinterpret_cast<T*>(H->hEnth),
                                         reinterpret_cast<T*>(H->tTemp), reinterpret_cast<T*>(H->kCond),
                                         reinterpret_cast<T*>(H->dDens), reinterpret_cast<T*>(H->mVisc),
                                         (int64_t)nout, H->dt, H->tGamma[isub], H->tZeta[isub], st));
    H->launches++;
  } else if (epilogue == EP_ENERGY) {
    PROFD(H, 3, 5.0 * sizeof(T) * nout, bufs(), bufs(out, rhs0, rhoh),
         launch_energy_advance<T>(out, rhs0, rhoh, (int64_t)nout, H->dt, H->tGamma[isub], H->tZeta[isub], st));
    H->launches++;
  }
  return false;
}

void build_bcs(chs_handle* H, const chs_config* c) {
  std::memcpy(H->ibc, c->nominal_bc, sizeof(H->ibc));
  std::memcpy(H->fbcy, c->fbcy_const, sizeof(H->fbcy));
  for (int n = 0; n < 2; ++n) {  // config_calc_basic_ibc (src/bc_general.f90:141-184)
    if (H->ibc[0][V_QX][n] == BC_SYMMETRIC) H->ibc[0][V_QX][n] = BC_ASYMMETRIC;
    if (H->ibc[1][V_QY][n] == BC_SYMMETRIC) H->ibc[1][V_QY][n] = BC_ASYMMETRIC;
    if (H->ibc[2][V_QZ][n] == BC_SYMMETRIC) H->ibc[2][V_QZ][n] = BC_ASYMMETRIC;
    if (H->ibc[0][V_QX][n] == BC_DIRICHLET) H->ibc[0][V_PR][n] = BC_NEUMANN;
    if (H->ibc[1][V_QY][n] == BC_DIRICHLET) { H->ibc[1][V_PR][n] = BC_NEUMANN; H->fbcy[V_PR][n] = 0.0; }
    if (H->ibc[2][V_QZ][n] == BC_DIRICHLET) H->ibc[2][V_PR][n] = BC_NEUMANN;
  }
  for (int n = 0; n < 2; ++n)
    for (int v = 0; v < 5; ++v)
      if (H->ibc[0][v][n] != BC_PERIODIC || H->ibc[2][v][n] != BC_PERIODIC)
        throw std::invalid_argument("x and z must be periodic (channel / Taylor-Green configurations)");
  int ftp[3][2];
  for (int d = 0; d < 3; ++d)
    for (int n = 0; n < 2; ++n)
      ftp[d][n] = H->ibc[d][V_TM][n] == BC_NEUMANN ? BC_DIRICHLET : H->ibc[d][V_TM][n];
  auto& B = H->ibc;
  // energy-equation operations (config_calc_eqs_ibc, src/bc_general.f90:660-685)
  H->ftpy = Pair{{ftp[1][0], ftp[1][1]}};
  H->ebcx_conv = prod_of(B[0][V_QX], ftp[0]);
  H->ebcy_conv = prod_of(B[1][V_QY], ftp[1]);
  H->ebcz_conv = prod_of(B[2][V_QZ], ftp[2]);
  H->ebcx_difu = tau_of(B[0][V_TM], ftp[0]);
  H->ebcy_difu = tau_of(B[1][V_TM], ftp[1]);
  H->ebcz_difu = tau_of(B[2][V_TM], ftp[2]);
  // config_calc_eqs_ibc (src/bc_general.f90:512-677)
  H->mbcx_cov1 = prod_of(B[0][V_QX], B[0][V_QX]);
  H->mbcy_cov1 = prod_of(B[1][V_QY], B[1][V_QX]);
  H->mbcz_cov1 = prod_of(B[2][V_QZ], B[2][V_QX]);
  H->mbcx_tau1 = tau_of(B[0][V_QX], ftp[0]);
  H->mbcy_tau1 = tau_of(B[1][V_QX], ftp[1]);
  H->mbcz_tau1 = tau_of(B[2][V_QX], ftp[2]);
  H->mbcx_cov2 = prod_of(B[0][V_QX], B[0][V_QY]);
  H->mbcy_cov2 = prod_of(B[1][V_QY], B[1][V_QY]);
  H->mbcz_cov2 = prod_of(B[2][V_QZ], B[2][V_QY]);
  H->mbcx_tau2 = tau_of(B[0][V_QY], ftp[0]);
  H->mbcy_tau2 = tau_of(B[1][V_QY], ftp[1]);
  H->mbcz_tau2 = tau_of(B[2][V_QY], ftp[2]);
  H->mbcx_cov3 = prod_of(B[0][V_QX], B[0][V_QZ]);
  H->mbcy_cov3 = prod_of(B[1][V_QY], B[1][V_QZ]);
  H->mbcz_cov3 = prod_of(B[2][V_QZ], B[2][V_QZ]);
  H->mbcx_tau3 = tau_of(B[0][V_QZ], ftp[0]);
  H->mbcy_tau3 = tau_of(B[1][V_QZ], ftp[1]);
  H->mbcz_tau3 = tau_of(B[2][V_QZ], ftp[2]);
  H->fbcy_velo = false;
  for (int v = V_QX; v <= V_QZ; ++v)
    for (int n = 0; n < 2; ++n)
      if (B[1][v][n] == BC_DIRICHLET || B[1][v][n] == BC_INTERIOR) H->fbcy_velo = true;
  if (H->periodic_y && H->fbcy_velo) throw std::invalid_argument("inconsistent y boundary conditions");
}

// operator-plan geometry (host only): ghost spacings and y metric of the 1D wrappers
// (src/basics_operations2.f90:2739-3950)
void setup_book(chs_handle* H, const chs_config* c) {
  const int nc1 = H->nc[1], np1 = H->np[1];
  std::vector<double> yp(c->yp, c->yp + nc1 + 1), yc(c->yc, c->yc + nc1);
  std::vector<double> mppt(c->ymap_pt, c->ymap_pt + nc1 + 1), mpcc(c->ymap_cc, c->ymap_cc + nc1);
  H->mpcc = mpcc;
  H->mppt = mppt;
  PlanBook& bk = H->book;
  bk.iacc = H->iacc;
  for (int d : {0, 2}) {
    auto& G = bk.dir[d];
    G.nc = H->nc[d]; G.np = H->np[d]; G.periodic = true; G.dd = 1.0 / H->h[d];
    const double hh = H->h[d];
    G.dp_c[0] = hh; G.dp_c[2] = hh * 2.0; G.dp_c[1] = hh; G.dp_c[3] = hh * 2.0;
    G.dp_p[0] = hh * 2.0; G.dp_p[2] = hh * 4.0; G.dp_p[1] = hh * 2.0; G.dp_p[3] = hh * 4.0;
  }
  auto& G = bk.dir[1];
  G.nc = nc1; G.np = np1; G.periodic = H->periodic_y; G.dd = 1.0 / H->h[1];
  G.dp_c[0] = (yc[0] - yp[0]) * 2.0;
  G.dp_c[2] = (yc[1] - yp[0]) * 2.0;
  G.dp_c[1] = (yp[np1 - 1] - yc[nc1 - 1]) * 2.0;
  G.dp_c[3] = (yp[np1 - 1] - yc[nc1 - 2]) * 2.0;
  G.dp_p[0] = (yp[1] - yp[0]) * 2.0;
  G.dp_p[2] = (yp[2] - yp[0]) * 2.0;
  G.dp_p[1] = (yp[np1 - 1] - yp[np1 - 2]) * 2.0;
  G.dp_p[3] = (yp[np1 - 1] - yp[np1 - 3]) * 2.0;
  if (H->stretch_y) {
    G.map_cc = bk.add_array(mpcc);
    G.map_pt = bk.add_array(std::vector<double>(mppt.begin(), mppt.begin() + np1));
  }
}

// scalars, boundary conditions and plan geometry (no device work)
void setup_host(chs_handle* H, const chs_config* c) {
  for (int d = 0; d < 3; ++d) {
    if (c->nc[d] < 8) throw std::invalid_argument("at least 8 cells per direction are required");
    H->nc[d] = c->nc[d];
  }
  H->periodic_y = false;
  for (int v = 0; v < 5; ++v)
    for (int n = 0; n < 2; ++n)
      if (c->nominal_bc[1][v][n] == BC_PERIODIC) H->periodic_y = true;
  H->np[0] = H->nc[0];
  H->np[1] = H->periodic_y ? H->nc[1] : H->nc[1] + 1;
  H->np[2] = H->nc[2];
  H->stretch_y = c->istret != 0;
  H->iacc = c->iacc;
  H->ifft = c->ifft;
  H->idriven = c->idriven;
  if (H->iacc < 1 || H->iacc > 4) throw std::invalid_argument("iacc must be 1..4");
  if (H->ifft != 2 && H->ifft != 3) throw std::invalid_argument("ifft must be 2 or 3");
  if (H->ifft == 2 && H->periodic_y) throw std::invalid_argument("FISHPACK Poisson needs non-periodic y");
  if (H->ifft == 3 && !H->periodic_y) {
    // poisson_010 (src/poisson_1stderivcomp.f90:1457-1816): cosine modes in y, split odd/even
    if (H->nc[1] % 2) throw std::invalid_argument("3D-FFT Poisson with y walls needs an even ny");
    if (c->istret != 0 && c->istret != 1 && c->istret != 2)
      throw std::invalid_argument("3D-FFT Poisson with y walls supports istret 0, 1 and 2");
    if (c->istret != 0 && !(c->rstret > 0.0)) throw std::invalid_argument("3FMD stretching needs rstret > 0");
  }
  if (c->precision != CHS_FP64 && c->precision != CHS_MIXED) throw std::invalid_argument("unknown precision mode");
  H->mixed = c->precision == CHS_MIXED;
  H->dag_lanes = H->mixed ? 4 : 3;
  H->h[0] = c->lxx / H->nc[0];
  H->h[2] = c->lzz / H->nc[2];
  H->h[1] = H->stretch_y ? 1.0 / H->nc[1] : (c->lyt - c->lyb) / H->nc[1];
  H->dt = c->dt;
  H->rre = 1.0 / c->ren;
  H->sigma2p = 1.0;
  // RK3 constants (src/input_general.f90:851-886)
  H->tGamma[0] = 1.0; H->tGamma[1] = 8.0 / 15.0; H->tGamma[2] = 5.0 / 12.0; H->tGamma[3] = 3.0 * 0.25;
  H->tZeta[0] = 0.0; H->tZeta[1] = 0.0; H->tZeta[2] = -17.0 / 60.0; H->tZeta[3] = -5.0 / 12.0;
  for (int i = 0; i < 4; ++i) H->tAlpha[i] = H->tGamma[i] + H->tZeta[i];
  build_bcs(H, c);
  setup_book(H, c);
}

// device buffers and Poisson tables
void setup_device(chs_handle* H, const chs_config* c) {
  const int nc0 = H->nc[0], nc1 = H->nc[1], nc2 = H->nc[2], np1 = H->np[1];
  const std::vector<double>& mpcc = H->mpcc;
  const std::vector<double>& mppt = H->mppt;
  CK(cudaStreamCreateWithFlags(&H->st, cudaStreamNonBlocking));
  H->n_pcc = (size_t)H->np[0] * nc1 * nc2;
  H->n_cpc = (size_t)nc0 * np1 * nc2;
  H->n_ccp = (size_t)nc0 * nc1 * H->np[2];
  H->n_ccc = (size_t)nc0 * nc1 * nc2;
  H->n_ppc = (size_t)H->np[0] * np1 * nc2;
  H->n_pcp = (size_t)H->np[0] * nc1 * H->np[2];
  H->n_cpp = (size_t)nc0 * np1 * H->np[2];
  H->qx = H->dalloc<double>(H->n_pcc); H->qy = H->dalloc<double>(H->n_cpc); H->qz = H->dalloc<double>(H->n_ccp);
  H->pres = H->dalloc<double>(H->n_ccc); H->pcor = H->dalloc<double>(H->n_ccc);
  H->mx0 = H->dalloc<double>(H->n_pcc); H->my0 = H->dalloc<double>(H->n_cpc); H->mz0 = H->dalloc<double>(H->n_ccp);
  H->mx = H->dalloc<double>(H->n_pcc); H->my = H->dalloc<double>(H->n_cpc); H->mz = H->dalloc<double>(H->n_ccp);
  H->px = H->dalloc<double>(H->n_pcc); H->py = H->dalloc<double>(H->n_cpc); H->pz = H->dalloc<double>(H->n_ccp);
  H->qxix = H->dalloc<double>(H->n_ccc); H->qxdx = H->dalloc<double>(H->n_ccc);
  H->qxdy = H->dalloc<double>(H->n_ppc); H->qxiy = H->dalloc<double>(H->n_ppc);
  H->qxiz = H->dalloc<double>(H->n_pcp); H->qxdz = H->dalloc<double>(H->n_pcp);
  H->qydx = H->dalloc<double>(H->n_ppc); H->qyix = H->dalloc<double>(H->n_ppc);
  H->qydy = H->dalloc<double>(H->n_ccc); H->qyiy = H->dalloc<double>(H->n_ccc);
  H->qydz = H->dalloc<double>(H->n_cpp); H->qyiz = H->dalloc<double>(H->n_cpp);
  H->qzdx = H->dalloc<double>(H->n_pcp); H->qzix = H->dalloc<double>(H->n_pcp);
  H->qziy = H->dalloc<double>(H->n_cpp); H->qzdy = H->dalloc<double>(H->n_cpp);
  H->qziz = H->dalloc<double>(H->n_ccc); H->qzdz = H->dalloc<double>(H->n_ccc);
  H->div = H->dalloc<double>(H->n_ccc);
  if (H->fbcy_velo) {
    H->qxdx_cpc = H->dalloc<double>(H->n_cpc);
    H->qydy_cpc = H->dalloc<double>(H->n_cpc);
    H->qzdz_cpc = H->dalloc<double>(H->n_cpc);
  }
  const size_t nl = (size_t)nc0 * nc2;  // y lines (x and z are periodic: np = nc)
  H->fb_qx = H->dalloc<double>(4 * nl); H->fb_qy = H->dalloc<double>(4 * nl); H->fb_qz = H->dalloc<double>(4 * nl);
  H->fb_pr = H->dalloc<double>(4 * nl); H->fb_mpr = H->dalloc<double>(4 * nl);
  H->fb_conv2 = H->dalloc<double>(4 * nl); H->fb_visc2 = H->dalloc<double>(4 * nl);
  H->fb_comb = H->dalloc<double>(4 * nl);
  H->fb_maxp = H->dalloc<double>(4 * nl);
  auto fill = [&](double* p, double v0, double v1) {
    if (H->mixed) launch_fbcy_const(reinterpret_cast<float*>(p), nc0, nc2, v0, v1, H->st);
    else launch_fbcy_const(p, nc0, nc2, v0, v1, H->st);
  };
  fill(H->fb_qx, H->fbcy[V_QX][0], H->fbcy[V_QX][1]);
  fill(H->fb_qy, H->fbcy[V_QY][0], H->fbcy[V_QY][1]);
  fill(H->fb_qz, H->fbcy[V_QZ][0], H->fbcy[V_QZ][1]);
  fill(H->fb_pr, H->fbcy[V_PR][0], H->fbcy[V_PR][1]);
  fill(H->fb_mpr, -H->fbcy[V_PR][0], -H->fbcy[V_PR][1]);
  fill(H->fb_conv2, -H->fbcy[V_QY][0] * H->fbcy[V_QY][0], -H->fbcy[V_QY][1] * H->fbcy[V_QY][1]);
  fill(H->fb_maxp, kMaxp, kMaxp);
  if (H->mixed) {
    size_t m = H->n_pcc;
    for (size_t v : {H->n_cpc, H->n_ccp, H->n_ccc}) m = v > m ? v : m;
    H->stage = H->dalloc<double>(m);
  }
  H->launches += 7;

  // volume weights dy(j)*dx*dz (src/tools_general.f90:1229-1253)
  std::vector<double> wy(nc1);
  H->vol = 0.0;
  for (int j = 0; j < nc1; ++j) {
    double dy = H->h[1];
    if (H->stretch_y) dy = H->h[1] / mpcc[j];
    wy[j] = dy * H->h[0] * H->h[2];
    H->vol += wy[j] * (double)H->np[0] * (double)nc2;
  }
  H->wy = H->dalloc<double>(nc1);
  CK(cudaMemcpyAsync(H->wy, wy.data(), nc1 * sizeof(double), cudaMemcpyHostToDevice, H->st));
  H->npart = 148 * 4;
  H->partial = H->dalloc<double>(2 * H->npart);
  H->fz_part = H->dalloc<double>(fz_momentum_x_blocks(nc0, nc1, nc2));
  H->scal = H->dalloc<double>(16);

  // Poisson tables
  std::vector<double2> tw;
  const int nxh = nc0 / 2 + 1;
  // twiddles in FP64 and, for the FP32 spectrum of the mixed form, rounded to FP32
  auto upload_tw = [&](FftPlan& fp) {
    double2* d = H->dalloc<double2>(tw.size());
    CK(cudaMemcpyAsync(d, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, H->st));
    fp.tw = d;
    std::vector<float2> twf(tw.size());
    for (size_t m = 0; m < tw.size(); ++m) twf[m] = make_float2((float)tw[m].x, (float)tw[m].y);
    float2* f = H->dalloc<float2>(twf.size());
    CK(cudaMemcpyAsync(f, twf.data(), twf.size() * sizeof(float2), cudaMemcpyHostToDevice, H->st));
    CK(cudaStreamSynchronize(H->st));  // twf is a local vector
    fp.twf = f;
  };
  H->fx = make_fft(nc0, tw);
  upload_tw(H->fx);
  H->fz = make_fft(nc2, tw);
  upload_tw(H->fz);
  H->spec = H->dalloc<double2>((size_t)nxh * nc1 * nc2);
  const double pi = 2.0 * std::asin(1.0);
  if (H->ifft == 2) {
    if (nc0 % 2 || nc2 % 2) throw std::invalid_argument("FISHPACK path needs even nx and nz");
    // fishpack_root_1D eigenvalues (src/poisson_fishpack.f90:60-110), one per complex mode
    auto roots = [&](int N, double c1, std::vector<double>& lam) {
      const double dxr = pi / (2.0 * (double)N);
      lam.assign(N, 0.0);
      for (int k = 0; k < N; ++k) {
        const int kk = k <= N / 2 ? k : N - k;
        if (kk == 0) lam[k] = 0.0;
        else if (2 * kk == N) lam[k] = -4.0 * c1;
        else {
          const double s = std::sin(double(2 * kk) * dxr);
          lam[k] = -4.0 * c1 * s * s;
        }
      }
    };
    std::vector<double> lx, lz;
    roots(nc0, 1.0 / (H->h[0] * H->h[0]), lx);
    roots(nc2, 1.0 / (H->h[2] * H->h[2]), lz);
    lx.resize(nxh);
    H->lamx = H->dalloc<double>(nxh);
    H->lamz = H->dalloc<double>(nc2);
    CK(cudaMemcpyAsync(H->lamx, lx.data(), nxh * sizeof(double), cudaMemcpyHostToDevice, H->st));
    CK(cudaMemcpyAsync(H->lamz, lz.data(), nc2 * sizeof(double), cudaMemcpyHostToDevice, H->st));
    // y coefficients (src/poisson_fishpack.f90:312-323), Cartesian
    const double h2r = 1.0 / (H->h[1] * H->h[1]);
    std::vector<double> a(nc1), b(nc1), cc(nc1);
    for (int j = 0; j < nc1; ++j) {
      a[j] = h2r * mpcc[j] * mppt[j] * 1.0 * 1.0;
      cc[j] = h2r * mpcc[j] * mppt[j + 1] * 1.0 * 1.0;
    }
    for (int j = 0; j < nc1; ++j) b[j] = -(a[j] + cc[j]);
    b[0] = b[0] + a[0]; a[0] = 0.0;
    b[nc1 - 1] = b[nc1 - 1] + cc[nc1 - 1]; cc[nc1 - 1] = 0.0;
    H->pa = H->dalloc<double>(nc1); H->pb = H->dalloc<double>(nc1); H->pc = H->dalloc<double>(nc1);
    CK(cudaMemcpyAsync(H->pa, a.data(), nc1 * sizeof(double), cudaMemcpyHostToDevice, H->st));
    CK(cudaMemcpyAsync(H->pb, b.data(), nc1 * sizeof(double), cudaMemcpyHostToDevice, H->st));
    CK(cudaMemcpyAsync(H->pc, cc.data(), nc1 * sizeof(double), cudaMemcpyHostToDevice, H->st));
    H->yzr = H->dalloc<double>((size_t)nxh * nc1 * nc2);
    H->yd = H->dalloc<double>((size_t)nxh * nc1 * nc2);
    launch_ysolve_factor(H->yzr, H->yd, nxh, nc1, nc2, H->pa, H->pb, H->pc, H->lamx, H->lamz, H->st);
    H->launches++;
  } else {
    H->fy = make_fft(nc1, tw);
    double2* d = H->dalloc<double2>(tw.size());
    CK(cudaMemcpyAsync(d, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, H->st));
    H->fy.tw = d;
    // modified wavenumbers of the periodic C2P derivative (src/poisson_1stderivcomp.f90:2448-2503)
    const CoefSet& cs = coef(D1C2P, H->iacc);
    const double alc = cs.lhs[2][0][BC_PERIODIC];
    auto k2 = [&](int n, double len, double dh) {
      const double ac = cs.rhs[2][0][BC_PERIODIC] / dh, bc = cs.rhs[2][1][BC_PERIODIC] / dh;
      std::vector<double> v(n, 0.0);
      for (int i = 1; i <= n / 2 + 1; ++i) {
        const double w = 2.0 * pi * double(i - 1) / double(n);
        double wp = ac * 2.0 * dh * std::sin(w * 0.5) + bc * 2.0 * dh * std::sin(3.0 * 0.5 * w);
        wp = wp / (1.0 + 2.0 * alc * std::cos(w));
        const double q = double(n) * wp / len;
        v[i - 1] = q * q;
      }
      for (int i = n / 2 + 2; i <= n; ++i) v[i - 1] = v[n - i + 1];
      return v;
    };
    auto kx = k2(nc0, c->lxx, H->h[0]);
    auto ky = k2(nc1, c->lyt - c->lyb, H->h[1]);
    auto kz = k2(nc2, c->lzz, H->h[2]);
    kx.resize(nxh);
    if (!H->periodic_y) {
      // poisson_010.  abxyz for bcy = 1 (src/poisson_1stderivcomp.f90:2376-2382)
      std::vector<double> ab(2 * (size_t)nc1);
      for (int j = 1; j <= nc1; ++j) {
        ab[j - 1] = std::sin(double(j - 1) * pi * 0.5 / double(nc1));
        ab[nc1 + j - 1] = std::cos(double(j - 1) * pi * 0.5 / double(nc1));
      }
      H->ayby = H->dalloc<double>(ab.size());
      CK(cudaMemcpyAsync(H->ayby, ab.data(), ab.size() * sizeof(double), cudaMemcpyHostToDevice, H->st));
      // waves for bcy = 1 (:2484-2501): w = pi (j-1)/nym; yky = nym wp (stretched grid), yk2 = (nym wp / yly)^2
      const double dy = H->h[1], yly = c->lyt - c->lyb;
      const double ac = cs.rhs[2][0][BC_PERIODIC] / dy, bc = cs.rhs[2][1][BC_PERIODIC] / dy;
      std::vector<double> yky(nc1, 0.0);
      ky.assign(nc1, 0.0);
      for (int j = 2; j <= nc1; ++j) {
        const double w = 2.0 * pi * 0.5 * double(j - 1) / double(nc1);
        double wp = ac * 2.0 * dy * std::sin(w * 0.5) + (bc * 2.0 * dy) * std::sin(3.0 * 0.5 * w);
        wp = wp / (1.0 + 2.0 * alc * std::cos(w));
        yky[j - 1] = H->stretch_y ? double(nc1) * wp : double(nc1) * wp / yly;
        const double q = double(nc1) * wp / yly;
        ky[j - 1] = q * q;
      }
      if (H->stretch_y) {
        // matrice_refinement for istret 1 or 2 (:2718-3046) with unit transfer factors: per system
        // (odd modes cw22 = yky(2j-1), even modes cw2 = yky(2j)) and row the diagonals a(.,1), a(.,2),
        // the two added terms of the main diagonal, a(.,4) and a(.,5)
        const int hh = nc1 / 2;
        const double beta = c->rstret;
        const double alpha = (-1.0 + std::sqrt(1.0 + 4.0 * pi * pi * beta * beta)) / beta * 0.5;
        double xa0 = alpha / pi + 0.5 / beta / pi;
        double xa1 = c->istret == 1 ? +1.0 / 4.0 / beta / pi : -1.0 / 4.0 / beta / pi;
        xa0 = xa0 / yly;
        xa1 = xa1 / yly;
        const double xa0_2 = xa0 * xa0, xa1_2 = xa1 * xa1, xa01 = xa0 * xa1, xa0p1_2 = (xa0 + xa1) * (xa0 + xa1);
        std::vector<double> tab(12 * (size_t)hh, 0.0);
        for (int sy = 0; sy < 2; ++sy) {
          std::vector<double> w(hh + 2, 0.0);  // 1-based
          for (int j = 1; j <= hh; ++j) w[j] = yky[2 * j - 2 + sy];
          double* A1 = tab.data() + (size_t)sy * 6 * hh;
          double *A2 = A1 + hh, *T1 = A1 + 2 * hh, *T2 = A1 + 3 * hh, *A4 = A1 + 4 * hh, *A5 = A1 + 5 * hh;
          for (int j = 1; j <= hh; ++j) {
            const int r = j - 1;
            if (j >= 2 && j <= hh - 1) {
              T1[r] = xa0_2 * (w[j] * w[j]);
              T2[r] = xa1_2 * w[j] * (w[j - 1] + w[j + 1]);
            } else if (j == 1) {
              T1[r] = (sy == 0 ? xa0_2 : xa0_2 - xa1_2) * (w[1] * w[1]);
              T2[r] = xa1_2 * w[1] * w[2];
            } else {
              T1[r] = (sy == 0 ? xa0_2 : xa0p1_2) * (w[hh] * w[hh]);
              T2[r] = xa1_2 * w[hh] * w[hh - 1];
            }
            if (j >= 2 && j <= hh - 1) A4[r] = xa01 * (w[j + 1] * (w[j] + w[j + 1]));
            if (j == 1) A4[r] = sy == 0 ? 2.0 * xa01 * (w[1] * w[2] + w[2] * w[2])
                                        : (xa0 - xa1) * xa1 * (w[1] * w[2]) + xa0 * xa1 * (w[2] * w[2]);
            if (sy == 1 && j == hh - 1) A4[r] = xa0 * xa1 * w[hh - 1] * w[hh] + (xa0 + xa1) * xa1 * (w[hh] * w[hh]);
            if (sy == 1 && j == hh) A4[r] = 0.0;
            if (j <= hh - 2) A5[r] = xa1_2 * (-(w[j + 1] * w[j + 2]));
            if (sy == 0 && j == 1) A5[r] = 2.0 * A5[r];
            if (j >= 2) A2[r] = xa01 * (w[j - 1] * (w[j] + w[j - 1]));
            if (sy == 1 && j == 2) A2[r] = xa0 * xa1 * (w[2] * w[1]) + (xa0 + xa1) * xa1 * (w[1] * w[1]);
            if (sy == 1 && j == hh) A2[r] = (xa0 + xa1) * xa1 * (w[hh] * w[hh - 1]) + xa0 * xa1 * (w[hh - 1] * w[hh - 1]);
            if (j >= 3) A1[r] = xa1_2 * (-(w[j - 1] * w[j - 2]));
          }
        }
        H->ptab = H->dalloc<double>(tab.size());
        CK(cudaMemcpyAsync(H->ptab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, H->st));
        H->k2x = H->dalloc<double>(nxh);
        H->k2z = H->dalloc<double>(nc2);
        CK(cudaMemcpyAsync(H->k2x, kx.data(), nxh * sizeof(double), cudaMemcpyHostToDevice, H->st));
        CK(cudaMemcpyAsync(H->k2z, kz.data(), nc2 * sizeof(double), cudaMemcpyHostToDevice, H->st));
        H->pfac = H->dalloc<double>((size_t)8 * hh * (nc2 / 2 + 1) * nxh);
        launch_dct_y_factor(H->pfac, nxh, nc2, nc1, H->k2x, H->k2z, H->ptab, H->st);
        H->launches++;
      }
    }
    if (!H->k2x) {
      H->k2x = H->dalloc<double>(nxh);
      H->k2z = H->dalloc<double>(nc2);
      CK(cudaMemcpyAsync(H->k2x, kx.data(), nxh * sizeof(double), cudaMemcpyHostToDevice, H->st));
      CK(cudaMemcpyAsync(H->k2z, kz.data(), nc2 * sizeof(double), cudaMemcpyHostToDevice, H->st));
    }
    H->k2y = H->dalloc<double>(nc1);
    CK(cudaMemcpyAsync(H->k2y, ky.data(), nc1 * sizeof(double), cudaMemcpyHostToDevice, H->st));
  }
}

void drop_graphs(chs_handle* H) {
  for (auto& g : H->gexec)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto& row : H->gpart)
    for (auto& g : row)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// plans are created lazily; the table must be on the device before any launch.  Captured
// graphs hold the table pointer, so they are dropped when the table moves.
void upload_table(chs_handle* H) {
  drop_graphs(H);
  if (H->table) { CK(cudaFreeAsync(H->table, H->st)); H->table = nullptr; }
  const size_t n = H->book.table.size() + 4;
  CK(cudaMallocAsync(&H->table, n * sizeof(double), H->st));
  CK(cudaMemcpyAsync(H->table, H->book.table.data(), H->book.table.size() * sizeof(double), cudaMemcpyHostToDevice,
                     H->st));
}

// The row table of a y operator with walls for the fused kernels: every output row as at most three
// taps over the input line plus the two wall planes, with 1/h and the row's y metric folded into the
// weights (the plan's bulk formula on its bulk rows, its boundary rows elsewhere, the Neumann
// overrides as a unit wall weight).  False when the plan does not fit that form.
bool fz_rows_of(const chs_handle* H, int fam, const OpPlan& P, std::vector<FzRow>& out) {
  if (P.tdma || P.r2 != 0.0) return false;
  const int nin = P.nin, nout = P.nout;
  const std::vector<double>& tab = H->book.table;
  for (int p = 0; p < nout; ++p) {
    FzRow r{};
    const int pc = p < 0 ? 0 : (p > nin - 1 ? nin - 1 : p);  // a valid input row for unused taps
    for (int t = 0; t < 3; ++t) r.o[t] = pc - p;
    if (P.neu1 && p == 0) {
      r.wb[0] = 1.0;
      r.flags = 2;
    } else if (P.neu2 && p == nout - 1) {
      r.wb[1] = 1.0;
      r.flags = 4;
    } else {
      const double sc = P.dd * (P.lmap >= 0 ? tab[P.lmap + p] : 1.0);
      if (p >= P.b_lo && p <= P.b_hi) {
        const double r1 = P.r1;
        if (fam == M1P2C) { r.o[0] = 0; r.o[1] = 1; r.w[0] = r1 * sc; r.w[1] = r1 * sc; }
        else if (fam == M1C2P) { r.o[0] = 0; r.o[1] = -1; r.w[0] = r1 * sc; r.w[1] = r1 * sc; }
        else if (fam == D1C2P) { r.o[0] = 0; r.o[1] = -1; r.w[0] = r1 * sc; r.w[1] = -r1 * sc; }
        else if (fam == D1P2C) { r.o[0] = 1; r.o[1] = 0; r.w[0] = r1 * sc; r.w[1] = -r1 * sc; }
        else return false;
      } else {
        for (int s = 0; s < P.nspec; ++s) {
          const SpecialRow& R = P.sp[s];
          if (R.row != p) continue;
          if (R.nt > 3 || R.wb[2] != 0.0 || R.wb[3] != 0.0) return false;
          for (int t = 0; t < R.nt; ++t) {
            r.o[t] = R.idx[t] - p;
            r.w[t] = R.w[t] * sc;
          }
          if (R.nt == 3) r.flags |= 1;
          if (R.wb[0] != 0.0) { r.wb[0] = R.wb[0] * sc; r.flags |= 2; }
          if (R.wb[1] != 0.0) { r.wb[1] = R.wb[1] * sc; r.flags |= 4; }
        }
      }
    }
    for (int t = 0; t < 3; ++t)
      if (p + r.o[t] < 0 || p + r.o[t] >= nin) return false;
    out.push_back(r);
  }
  return true;
}

// the row tables of every y plan built so far, uploaded as one device array (fz_index gives each
// plan's first row)
void upload_fz_rows(chs_handle* H) {
  drop_graphs(H);
  std::vector<FzRow> v;
  H->fz_index.clear();
  for (const auto& kv : H->plans) {
    const int d = std::get<0>(kv.first), fam = std::get<1>(kv.first);
    int at = -1;
    if (d == 1 && !kv.second.wrap) {
      std::vector<FzRow> r;
      if (fz_rows_of(H, fam, kv.second, r)) {
        at = (int)v.size();
        v.insert(v.end(), r.begin(), r.end());
      }
    }
    H->fz_index[kv.first] = at;
  }
  if (H->fz_rows) { CK(cudaFreeAsync(H->fz_rows, H->st)); H->fz_rows = nullptr; }
  if (v.empty()) v.push_back(FzRow{});  // periodic y: no tables, a valid pointer all the same
  CK(cudaMallocAsync(&H->fz_rows, v.size() * sizeof(FzRow), H->st));
  CK(cudaMemcpyAsync(H->fz_rows, v.data(), v.size() * sizeof(FzRow), cudaMemcpyHostToDevice, H->st));
  // the host vector goes out of scope: wait for the copy
  CK(cudaStreamSynchronize(H->st));
}

template <typename T>
void poisson_device(chs_handle* H, T* rhs) {
  const int nc0 = H->nc[0], nc1 = H->nc[1], nc2 = H->nc[2];
  const int nxh = nc0 / 2 + 1;
  cudaStream_t st = H->st;
  const double nreal = (double)nc0 * nc1 * nc2, nspec = (double)nxh * nc1 * nc2;
  if (H->ifft == 2 && sizeof(T) == sizeof(float) && H->fx.twf && H->fz.twf) {
    // mixed form, FISHPACK: the x and z transforms in FP32 on an FP32 spectrum, the y solve (the
    // wall-normal tridiagonal systems and the pinned kx = kz = 0 mode) in FP64
    float2* sp = reinterpret_cast<float2*>(H->spec);
    const double b_r2c = 4.0 * nreal + 8.0 * nspec, b_c2c = 16.0 * nspec;
    PROF(H, 1, b_r2c, launch_rfft_x(H->fx, rhs, sp, nc1 * nc2, st));
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, sp, nxh, nc1, nxh, (int64_t)nxh * nc1, -1, st));
    PROF(H, 2, 32.0 * nspec, launch_ysolve(sp, nxh, nc1, nc2, H->yzr, H->yd, H->pa, st));
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, sp, nxh, nc1, nxh, (int64_t)nxh * nc1, +1, st));
    PROF(H, 1, b_r2c, launch_irfft_x(H->fx, sp, rhs, nc1 * nc2, 1.0 / ((double)nc0 * (double)nc2), st));
    H->launches += 5;
    return;
  }
  const double b_r2c = (double)sizeof(T) * nreal + 16.0 * nspec, b_c2c = 32.0 * nspec;
  PROF(H, 1, b_r2c, launch_rfft_x(H->fx, rhs, H->spec, nc1 * nc2, st));
  if (H->ifft == 2) {
    // fishpack_fft_simple (src/poisson_fishpack.f90:354-490)
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, H->spec, nxh, nc1, nxh, (int64_t)nxh * nc1, -1, st));
    PROF(H, 2, 48.0 * nspec, launch_ysolve(H->spec, nxh, nc1, nc2, H->yzr, H->yd, H->pa, st));
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, H->spec, nxh, nc1, nxh, (int64_t)nxh * nc1, +1, st));
    PROF(H, 1, b_r2c, launch_irfft_x(H->fx, H->spec, rhs, nc1 * nc2, 1.0 / ((double)nc0 * (double)nc2), st));
    H->launches += 5;
  } else if (!H->periodic_y) {
    // poisson_010 (src/poisson_1stderivcomp.f90:1457-1816): x and z transforms around the y
    // stage (the FFT normalisation 1/(nx ny nz) is applied there, after the forward transforms)
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, H->spec, nxh, nc1, nxh, (int64_t)nxh * nc1, -1, st));
    PROF(H, 2, b_c2c, launch_dct_y(H->fy, H->spec, nxh, nc2, H->ayby, H->k2x, H->k2z, H->k2y, H->ptab, H->pfac,
                                   1.0 / ((double)nc0 * (double)nc1 * (double)nc2), st));
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, H->spec, nxh, nc1, nxh, (int64_t)nxh * nc1, +1, st));
    PROF(H, 1, b_r2c, launch_irfft_x(H->fx, H->spec, rhs, nc1 * nc2, 1.0, st));
    H->launches += 5;
  } else {
    // poisson_000 (src/poisson_1stderivcomp.f90:1016-1195)
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fy, H->spec, nxh, nc2, (int64_t)nxh * nc1, nxh, -1, st));
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, H->spec, nxh, nc1, nxh, (int64_t)nxh * nc1, -1, st));
    PROF(H, 3, b_c2c, launch_spectral_divide(H->spec, nxh, nc1, nc2, H->k2x, H->k2y, H->k2z,
                                             1.0 / ((double)nc0 * (double)nc1 * (double)nc2), st));
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fz, H->spec, nxh, nc1, nxh, (int64_t)nxh * nc1, +1, st));
    PROF(H, 1, b_c2c, launch_cfft_axis(H->fy, H->spec, nxh, nc2, (int64_t)nxh * nc1, nxh, +1, st));
    PROF(H, 1, b_r2c, launch_irfft_x(H->fx, H->spec, rhs, nc1 * nc2, 1.0, st));
    H->launches += 7;
  }
}

// the substep body (enqueued on H->st; capturable); T is the field type
// ---- fused momentum path for the explicit schemes (chs_fused.cu)
// The descriptor names, for every inner and outer operator of the momentum equation, the same plan
// the operator path below launches (direction, family, boundary pair, whether boundary planes are
// given); a plan that is not an explicit one, or an x/z plan that is not periodic with the bulk
// formula everywhere, sends the substep down the operator path.
struct FzBuild {
  chs_handle* H;
  bool ok = true;
  const OpPlan* plan = nullptr;  // the plan of the last op()
  FzOp op(int d, int fam, Pair bc, bool has_fbc) {
    FzOp o{};
    auto key = std::make_tuple(d, fam, bc.v[0], bc.v[1], has_fbc ? 1 : 0);
    auto it = H->plans.find(key);
    auto ix = H->fz_index.find(key);
    if (it == H->plans.end() || ix == H->fz_index.end()) { ok = false; return o; }
    const OpPlan& P = it->second;
    // CD2 only: every bulk formula two-point; x and z periodic (bulk formula everywhere); a y
    // plan either periodic too or with a row table
    if (P.tdma || P.r2 != 0.0) ok = false;
    if (d != 1 && !P.wrap) ok = false;
    if (d == 1 && (H->periodic_y != (P.wrap != 0) || (!P.wrap && ix->second < 0))) ok = false;
    // the fused kernels' interior blocks (rows 4 .. n-5) take every y operator's bulk formula at
    // every level: each bulk range must cover rows 2 .. nout-3
    if (d == 1 && !P.wrap && (P.b_lo > 2 || P.b_hi < P.nout - 3)) ok = false;
    o.row = P.wrap ? -1 : ix->second;
    plan = &P;
    o.r1 = P.r1;
    o.dd = P.dd;
    return o;
  }
  // pair_terms' rule: one operator on the combined expression when both terms share the plan
  template <typename T>
  FzPair<T> pair(int d, int fam, Pair bc1, const T* f1, Pair bc2, const T* f2, const T* fcomb) {
    FzPair<T> p{};
    const bool same = bc1.v[0] == bc2.v[0] && bc1.v[1] == bc2.v[1] && ((f1 == nullptr) == (f2 == nullptr)) &&
                      (f1 == f2 || fcomb != nullptr);
    if (same) {
      const T* f = (f1 == f2) ? f1 : fcomb;
      p.a = op(d, fam, bc1, f != nullptr);
      p.fa = f;
      p.merged = 1;
    } else {
      p.a = op(d, fam, bc1, f1 != nullptr);
      p.fa = f1;
      const OpPlan* pa = plan;
      p.b = op(d, fam, bc2, f2 != nullptr);
      p.fb = f2;
      p.merged = 0;
      // the interior rows run one operator on the combined expression: one bulk formula
      if (pa && plan && (pa->r1 != plan->r1 || pa->dd != plan->dd || pa->lmap != plan->lmap)) ok = false;
      // periodic directions run one operator on the combined expression: one bulk formula
      if ((d != 1 || H->periodic_y) && (p.a.r1 != p.b.r1 || p.a.dd != p.b.dd)) ok = false;
    }
    return p;
  }
};

// Momentum right-hand sides, fractional step, mass-flux mean and advance of the substep in four
// launches (wall planes, fused momentum, mean, advance) instead of the ~50 of the operator path.
// Returns false (nothing launched) when the configuration needs the operator path.
template <typename T>
bool fused_momentum(chs_handle* H, int isub, double* ux, double* uy, double* uz, bool defer_update) {
  if (!H->kfuse || H->iacc != ACC_CD2 || !H->fz_rows) return false;
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const auto& B = H->ibc;
  const bool TH = H->thermo;
  const int nc0 = H->nc[0], nc1 = H->nc[1], nc2 = H->nc[2], np1 = H->np[1];
  const T* any = A(H->fb_maxp);
  const T* fyqx = H->periodic_y ? nullptr : A(H->fb_qx);
  const T* fyqy = H->periodic_y ? nullptr : A(H->fb_qy);
  const T* fyqz = H->periodic_y ? nullptr : A(H->fb_qz);
  const T* fympr = H->periodic_y ? nullptr : A(H->fb_mpr);
  const T* fz = TH ? A(H->fb_zero) : nullptr;
  const Pair bx_qx = P2(B[0][V_QX]), by_qx = P2(B[1][V_QX]), bz_qx = P2(B[2][V_QX]);
  const Pair bx_qy = P2(B[0][V_QY]), by_qy = P2(B[1][V_QY]), bz_qy = P2(B[2][V_QY]);
  const Pair bx_qz = P2(B[0][V_QZ]), by_qz = P2(B[1][V_QZ]), bz_qz = P2(B[2][V_QZ]);
  const Pair bx_pr = P2(B[0][V_PR]), by_pr = P2(B[1][V_PR]), bz_pr = P2(B[2][V_PR]);
  const Pair per = P2(kPer2);
  FzBuild b{H};
  FzMomentum<T> F{};
  F.n0 = nc0; F.nc1 = nc1; F.np1 = np1; F.n2 = nc2;
  F.thermo = TH ? 1 : 0;
  F.periodic_y = H->periodic_y ? 1 : 0;
  if (TH && H->periodic_y) return false;
  F.qx = A(H->qx); F.qy = A(H->qy); F.qz = A(H->qz); F.p = A(H->pres);
  if (TH) { F.gx = A(H->gx); F.gy = A(H->gy); F.gz = A(H->gz); F.mu = A(H->mVisc); F.fm = A(H->fb_m); }
  F.fyqx = fyqx; F.fyqy = fyqy; F.fyqz = fyqz; F.fz = fz;
  // inner operators: the derived quantities of the operator path (same plan keys)
  F.in[FI_QX_MX] = b.op(0, M1P2C, bx_qx, true);
  F.in[FI_QX_DX] = b.op(0, D1P2C, bx_qx, true);
  F.in[FI_QX_DY] = b.op(1, D1C2P, by_qx, fyqx != nullptr);
  F.in[FI_QX_MY] = b.op(1, M1C2P, by_qx, fyqx != nullptr);
  F.in[FI_QX_MZ] = b.op(2, M1C2P, bz_qx, true);
  F.in[FI_QX_DZ] = b.op(2, D1C2P, bz_qx, true);
  F.in[FI_QY_DX] = b.op(0, D1C2P, bx_qy, true);
  F.in[FI_QY_MX] = b.op(0, M1C2P, bx_qy, true);
  F.in[FI_QY_DY] = b.op(1, D1P2C, by_qy, false);
  F.in[FI_QY_MY] = b.op(1, M1P2C, by_qy, fyqy != nullptr);
  F.in[FI_QY_DZ] = b.op(2, D1C2P, bz_qy, true);
  F.in[FI_QY_MZ] = b.op(2, M1C2P, bz_qy, true);
  F.in[FI_QZ_DX] = b.op(0, D1C2P, bx_qz, true);
  F.in[FI_QZ_MX] = b.op(0, M1C2P, bx_qz, true);
  F.in[FI_QZ_MY] = b.op(1, M1C2P, by_qz, fyqz != nullptr);
  F.in[FI_QZ_DY] = b.op(1, D1C2P, by_qz, fyqz != nullptr);
  F.in[FI_QZ_MZ] = b.op(2, M1P2C, bz_qz, true);
  F.in[FI_QZ_DZ] = b.op(2, D1P2C, bz_qz, false);
  if (TH) {
    F.in[FI_GX_MX] = b.op(0, M1P2C, bx_qx, true);
    F.in[FI_GX_MY] = b.op(1, M1C2P, by_qx, true);
    F.in[FI_GX_MZ] = b.op(2, M1C2P, bz_qx, true);
    F.in[FI_GY_MX] = b.op(0, M1C2P, bx_qy, true);
    F.in[FI_GY_MY] = b.op(1, M1P2C, by_qy, true);
    F.in[FI_GY_MZ] = b.op(2, M1C2P, bz_qy, true);
    F.in[FI_GZ_MX] = b.op(0, M1C2P, bx_qz, true);
    F.in[FI_GZ_MY] = b.op(1, M1C2P, by_qz, true);
    F.in[FI_GZ_MZ] = b.op(2, M1P2C, bz_qz, true);
    F.in[FI_MU_Y] = b.op(1, M1C2P, H->ftpy, true);
    F.in[FI_MU_YX] = b.op(0, M1C2P, per, true);
    F.in[FI_MU_X] = b.op(0, M1C2P, per, true);
    F.in[FI_MU_XZ] = b.op(2, M1C2P, per, false);
    F.in[FI_MU_YZ] = b.op(2, M1C2P, per, false);
  }
  if (H->fbcy_velo) {
    F.in[FI_W_DX] = b.op(0, D1P2C, bx_qx, false);
    F.in[FI_W_DY] = b.op(1, D1C2P, by_qy, fyqy != nullptr);
    F.in[FI_W_DZ] = b.op(2, D1P2C, bz_qz, false);
  }
  // outer operators of the three components, as the operator path pairs them
  const T* fconv2 = H->fbcy_velo ? A(H->fb_conv2) : A(H->fb_maxp);
  const T* fvisc2 = H->fbcy_velo ? A(H->fb_visc2) : A(H->fb_maxp);
  F.term[0][0] = b.pair<T>(0, D1C2P, H->mbcx_cov1, any, H->mbcx_tau1, any, (const T*)nullptr);
  F.term[0][1] = b.pair<T>(1, D1P2C, H->mbcy_cov1, (const T*)nullptr, H->mbcy_tau1, (const T*)nullptr, (const T*)nullptr);
  F.term[0][2] = b.pair<T>(2, D1P2C, H->mbcz_cov1, (const T*)nullptr, H->mbcz_tau1, (const T*)nullptr, (const T*)nullptr);
  F.term[1][0] = b.pair<T>(0, D1P2C, H->mbcx_cov2, (const T*)nullptr, H->mbcx_tau2, (const T*)nullptr, (const T*)nullptr);
  F.term[1][1] = b.pair<T>(1, D1C2P, H->mbcy_cov2, fconv2, H->mbcy_tau2, fvisc2, (const T*)A(H->fb_comb));
  F.term[1][2] = b.pair<T>(2, D1P2C, H->mbcz_cov2, (const T*)nullptr, H->mbcz_tau2, (const T*)nullptr, (const T*)nullptr);
  F.term[2][0] = b.pair<T>(0, D1P2C, H->mbcx_cov3, (const T*)nullptr, H->mbcx_tau3, (const T*)nullptr, (const T*)nullptr);
  F.term[2][1] = b.pair<T>(1, D1P2C, H->mbcy_cov3, (const T*)nullptr, H->mbcy_tau3, (const T*)nullptr, (const T*)nullptr);
  F.term[2][2] = b.pair<T>(2, D1C2P, H->mbcz_cov3, any, H->mbcz_tau3, any, (const T*)nullptr);
  F.pres[0] = b.op(0, D1C2P, bx_pr, true);
  F.pres[1] = b.op(1, D1C2P, by_pr, fympr != nullptr);
  F.pres[2] = b.op(2, D1C2P, bz_pr, true);
  F.fpres[0] = any; F.fpres[1] = fympr; F.fpres[2] = any;
  if (!b.ok) return false;
  if (H->idriven == 1) {
    F.wy = H->wy;
    F.part = H->fz_part;
  }
  F.m[0] = A(H->mx); F.m[1] = A(H->my); F.m[2] = A(H->mz);
  F.m0[0] = A(H->mx0); F.m0[1] = A(H->my0); F.m0[2] = A(H->mz0);
  F.rre = H->rre;
  F.dt = H->dt; F.gam = H->tGamma[isub]; F.zeta = H->tZeta[isub]; F.alpha = H->tAlpha[isub];
  F.rows = H->fz_rows;
  const double nf = (double)sizeof(T) * H->n_ccc;
  if (H->fbcy_velo) {
    PROFD(H, 3, (double)sizeof(T) * 16.0 * nc0 * nc2,
          bufs(H->qx, H->qy, H->qz, H->fb_qy, H->fb_conv2, TH ? H->mVisc : nullptr, TH ? H->fb_m : nullptr),
          bufs(H->fb_visc2, H->fb_comb), launch_fz_wall_visc<T>(F, A(H->fb_visc2), A(H->fb_comb), fconv2, st));
    H->launches++;
  }
  {
    // one pass per component: rhs0 read and written, rhs written, and a third of the shared inputs
    // q (3), p [+ g (3), mu] (the three components together read each input once); the three run
    // concurrently on the dataflow lanes, x and z also beside the wall-row kernel (only the y
    // component's y term reads its planes)
    double* mo[3] = {H->mx, H->my, H->mz};
    double* m0[3] = {H->mx0, H->my0, H->mz0};
    for (int c = 0; c < 3; ++c) {
      PROFD(H, 4, nf * ((TH ? 8.0 : 4.0) / 3.0 + 3.0),
            bufs(H->qx, H->qy, H->qz, H->pres, TH ? H->gx : nullptr, TH ? H->gy : nullptr, TH ? H->gz : nullptr,
                 TH ? H->mVisc : nullptr, c == 1 ? H->fb_comb : nullptr, c == 1 ? H->fb_visc2 : nullptr,
                 H->fb_conv2, H->fb_qx, H->fb_qz, H->fb_qy, TH ? H->fb_m : nullptr),
            bufs(mo[c], m0[c], c == 0 && F.part ? H->fz_part : nullptr), launch_fz_momentum<T>(F, c, st));
      H->launches++;
    }
  }
  const double* bulk = nullptr;
  if (H->idriven == 1) {
    // the mass-flux mean from the x pass's per-CTA sums
    const int nblk = fz_momentum_x_blocks(nc0, nc1, nc2);
    PROFD(H, 3, 8.0 * nblk, bufs(H->fz_part), bufs(H->scal),
          launch_fz_finalize_mean(H->fz_part, nblk, H->scal + 0, H->vol, st));
    bulk = H->scal + 0;
    H->launches++;
  }
  if (defer_update) return true;  // the advance is folded into fused_update_div and fused_project
  const int w0 = B[1][V_QY][0] == BC_DIRICHLET, w1 = B[1][V_QY][1] == BC_DIRICHLET;
  PROFD(H, 3, nf * 9.0, bufs(H->mx, H->my, H->mz, bulk), bufs(ux, uy, uz),
        launch_fz_update<T>(A(ux), A(uy), A(uz), A(H->mx), A(H->my), A(H->mz), bulk, nc0, nc1, np1, nc2, w0,
                            H->fbcy[V_QY][0], w1, H->fbcy[V_QY][1], st));
  H->launches++;
  return true;
}

// The Poisson right-hand side with the momentum advance folded in (FzUpdateDiv); launch false:
// only whether it can run.
template <typename T>
bool fused_update_div(chs_handle* H, int isub, double* ux, double* uy, double* uz, int w0, int w1, bool launch) {
  if (!H->kfuse || H->iacc != ACC_CD2 || !H->fz_rows) return false;
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const auto& B = H->ibc;
  FzBuild b{H};
  FzUpdateDiv<T> F{};
  F.n0 = H->nc[0]; F.nc1 = H->nc[1]; F.np1 = H->np[1]; F.n2 = H->nc[2];
  F.ux = A(ux); F.uy = A(uy); F.uz = A(uz);
  F.mx = A(H->mx); F.my = A(H->my); F.mz = A(H->mz);
  F.bulk = H->idriven == 1 ? H->scal + 0 : nullptr;
  F.s0 = w0; F.s1 = w1;
  F.v0 = H->fbcy[V_QY][0]; F.v1 = H->fbcy[V_QY][1];
  // the plans of the operator path's divergence terms
  F.dx = b.op(0, D1P2C, P2(B[0][V_QX]), true);
  F.dy = b.op(1, D1P2C, P2(B[1][V_QY]), false);
  F.dz = b.op(2, D1P2C, P2(B[2][V_QZ]), false);
  F.fdy = A(H->fb_maxp);
  F.rows = H->fz_rows;
  F.out = A(H->pcor);
  F.coeff = 1.0 / (H->tAlpha[isub] * H->sigma2p * H->dt);
  if (!b.ok || H->periodic_y) return false;
  if (!launch) return true;
  const double nf = (double)sizeof(T) * H->n_ccc;
  PROFD(H, 4, nf * 7.0, bufs(ux, uy, uz, H->mx, H->my, H->mz, F.bulk), bufs(H->pcor),
        launch_fz_update_div<T>(F, st));
  H->launches++;
  return true;
}

// Energy equation in four launches (wall gradients, fused energy pass, property update, wall
// states) instead of the ~14 of the operator path; false when it needs the operator path.
template <typename T>
bool fused_energy(chs_handle* H, int isub) {
  if (!H->kfuse || H->iacc != ACC_CD2 || !H->fz_rows || H->periodic_y) return false;
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const auto& B = H->ibc;
  const T* any = A(H->fb_maxp);
  const Pair per = P2(kPer2);
  FzBuild b{H};
  FzEnergy<T> F{};
  F.n0 = H->nc[0]; F.nc1 = H->nc[1]; F.np1 = H->np[1]; F.n2 = H->nc[2];
  F.gx = A(H->gx); F.gy = A(H->gy); F.gz = A(H->gz);
  F.h = A(H->hEnth); F.k = A(H->kCond); F.t = A(H->tTemp);
  F.fh = A(H->fb_h); F.fk = A(H->fb_k); F.fqw = A(H->fb_qw); F.fdtk = A(H->fb_dtk);
  // the operator path's energy_body_t plans
  F.in[FE_H_X] = b.op(0, M1C2P, per, true);
  F.in[FE_H_Y] = b.op(1, M1C2P, H->ftpy, true);
  F.in[FE_H_Z] = b.op(2, M1C2P, per, true);
  F.in[FE_K_X] = b.op(0, M1C2P, per, true);
  F.in[FE_K_Y] = b.op(1, M1C2P, H->ftpy, true);
  F.in[FE_K_Z] = b.op(2, M1C2P, per, true);
  F.in[FE_T_X] = b.op(0, D1C2P, P2(B[0][V_TM]), true);
  F.in[FE_T_Y] = b.op(1, D1C2P, P2(B[1][V_TM]), true);
  F.in[FE_T_Z] = b.op(2, D1C2P, P2(B[2][V_TM]), true);
  F.in[FE_RH_Y] = b.op(1, M1C2P, H->ftpy, false);
  F.term[0] = b.pair<T>(0, D1P2C, H->ebcx_conv, any, H->ebcx_difu, any, (const T*)nullptr);
  F.term[1].a = b.op(1, D1P2C, H->ebcy_conv, false);
  F.term[1].fa = nullptr;
  F.term[1].b = b.op(1, D1P2C, H->ebcy_difu, true);
  F.term[1].fb = A(H->fb_dtk);
  F.term[1].merged = 0;
  F.term[2] = b.pair<T>(2, D1P2C, H->ebcz_conv, (const T*)nullptr, H->ebcz_difu, (const T*)nullptr,
                        (const T*)nullptr);
  if (!b.ok) return false;
  F.rhoh = A(H->rhoh);
  F.rhs0 = A(H->erhs0);
  F.rpr = H->rPrRen;
  F.dt = H->dt; F.gam = H->tGamma[isub]; F.zeta = H->tZeta[isub];
  F.rows = H->fz_rows;
  const int nc0 = H->nc[0], nc2 = H->nc[2];
  const double nf = (double)sizeof(T) * H->n_ccc;
  PROFD(H, 3, (double)sizeof(T) * 12.0 * nc0 * nc2, bufs(H->tTemp, H->kCond, H->fb_qw, H->fb_k), bufs(H->fb_dtk),
        launch_fz_energy_walls<T>(F, 0, A(H->fb_dtk), st));
  H->launches++;
  // read g (3), h, kappa, T, rhs0, rho*h; write rhs0, rho*h
  PROFD(H, 4, nf * 10.0,
        bufs(H->gx, H->gy, H->gz, H->hEnth, H->kCond, H->tTemp, H->fb_h, H->fb_k, H->fb_qw, H->fb_dtk),
        bufs(H->rhoh, H->erhs0), launch_fz_energy<T>(F, st));
  H->launches++;
  if (H->mlp_mode != 1) {
    PROFD(H, 3, nf * 6.0, bufs(H->rhoh), bufs(H->hEnth, H->tTemp, H->kCond, H->dDens, H->mVisc),
          launch_property_update<T>(H->tab, A(H->rhoh), A(H->hEnth), A(H->tTemp), A(H->kCond), A(H->dDens),
                                    A(H->mVisc), (int64_t)H->n_ccc, st));
  } else {
    PROFD(H, 3, 6.0 * sizeof(T) * H->n_ccc, bufs(H->rhoh, H->mlp_wpack),
          bufs(H->hEnth, H->tTemp, H->kCond, H->dDens, H->mVisc, H->mlp_nfb),
          launch_mlp_props<T>(H->tab, H->mlp_norm, H->mlp_small, H->mlp_check, H->mlp_wpack, A(H->rhoh),
                              A(H->hEnth), A(H->tTemp), A(H->kCond), A(H->dDens), A(H->mVisc), (int64_t)H->n_ccc,
                              H->mlp_nfb, st));
  }
  H->launches++;
  const int s0 = B[1][V_TM][0] == BC_NEUMANN, s1 = B[1][V_TM][1] == BC_NEUMANN;
  if (s0 || s1) {
    F.tab = H->tab;
    F.ws0 = s0; F.ws1 = s1;
    F.wh = A(H->fb_h); F.wk = A(H->fb_k); F.wm = A(H->fb_m); F.wd = A(H->fb_d);
    PROFD(H, 3, (double)sizeof(T) * 12.0 * nc0 * nc2, bufs(H->rhoh), bufs(H->fb_h, H->fb_k, H->fb_m, H->fb_d),
          launch_fz_energy_walls<T>(F, 1, (T*)nullptr, st));
    H->launches++;
  }
  return true;
}

// Pressure update, projection, wall enforcement and (variable properties) q = g / rho_face in one
// launch instead of up to nine; false when the configuration needs the operator path.
template <typename T>
bool fused_project(chs_handle* H, int isub, double* ux, double* uy, double* uz, int w0, int w1, bool upd,
                   bool launch) {
  if (!H->kfuse || H->iacc != ACC_CD2 || !H->fz_rows) return false;
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const auto& B = H->ibc;
  const bool TH = H->thermo;
  const T* fypr = H->periodic_y ? nullptr : A(H->fb_pr);
  FzBuild b{H};
  FzProject<T> F{};
  F.n0 = H->nc[0]; F.nc1 = H->nc[1]; F.np1 = H->np[1]; F.n2 = H->nc[2];
  F.thermo = TH ? 1 : 0;
  F.periodic_y = H->periodic_y ? 1 : 0;
  F.phi = A(H->pcor);
  F.p = A(H->pres);
  F.ux = A(ux); F.uy = A(uy); F.uz = A(uz);
  F.fphi = fypr;
  F.in[FP_DX] = b.op(0, D1C2P, P2(B[0][V_PR]), true);
  F.in[FP_DY] = b.op(1, D1C2P, P2(B[1][V_PR]), fypr != nullptr);
  F.in[FP_DZ] = b.op(2, D1C2P, P2(B[2][V_PR]), true);
  if (TH) {
    if (H->periodic_y) return false;
    const Pair per = P2(kPer2);
    F.qx = A(H->qx); F.qy = A(H->qy); F.qz = A(H->qz);
    F.rho = A(H->dDens);
    F.fd = A(H->fb_d);
    F.in[FP_PX] = b.op(0, M1C2P, per, true);
    F.in[FP_PY] = b.op(1, M1C2P, H->ftpy, true);
    F.in[FP_PZ] = b.op(2, M1C2P, per, true);
  }
  if (!b.ok) return false;
  F.coef = -(H->dt * H->tAlpha[isub] * H->sigma2p);
  F.s0 = w0; F.s1 = w1;
  F.v0 = H->fbcy[V_QY][0]; F.v1 = H->fbcy[V_QY][1];
  F.rows = H->fz_rows;
  F.upd = upd ? 1 : 0;
  F.mx = A(H->mx); F.my = A(H->my); F.mz = A(H->mz);
  F.bulk = H->idriven == 1 ? H->scal + 0 : nullptr;
  if (!launch) return true;
  const double nf = (double)sizeof(T) * H->n_ccc;
  PROFD(H, 3, nf * (TH ? 13.0 : 9.0) + (upd ? 3.0 * nf : 0.0),
        bufs(H->pcor, H->fb_pr, TH ? H->dDens : nullptr, TH ? H->fb_d : nullptr, upd ? H->mx : nullptr,
             upd ? H->my : nullptr, upd ? H->mz : nullptr, upd ? F.bulk : nullptr),
        bufs(H->pres, ux, uy, uz, TH ? H->qx : nullptr, TH ? H->qy : nullptr, TH ? H->qz : nullptr),
        launch_fz_project<T>(F, st));
  H->launches++;
  return true;
}

template <typename T>
void energy_body_t(chs_handle* H, int isub);
template <typename T>
void substep_body_t(chs_handle* H, int isub, int parts) {
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  if ((parts & PART_ENERGY) && H->thermo && isub >= 1) energy_body_t<T>(H, isub);
  if (!(parts & PART_MOMENTUM)) return;
  const int nc0 = H->nc[0], nc1 = H->nc[1], nc2 = H->nc[2];
  const int np0 = H->np[0], np1 = H->np[1], np2 = H->np[2];
  const int s_pcc[3] = {np0, nc1, nc2}, s_cpc[3] = {nc0, np1, nc2}, s_ccp[3] = {nc0, nc1, np2};
  const int s_ccc[3] = {nc0, nc1, nc2}, s_ppc[3] = {np0, np1, nc2}, s_pcp[3] = {np0, nc1, np2};
  const int s_cpp[3] = {nc0, np1, np2};
  const auto& B = H->ibc;
  const Pair bx_qx = P2(B[0][V_QX]), by_qx = P2(B[1][V_QX]), bz_qx = P2(B[2][V_QX]);
  const Pair bx_qy = P2(B[0][V_QY]), by_qy = P2(B[1][V_QY]), bz_qy = P2(B[2][V_QY]);
  const Pair bx_qz = P2(B[0][V_QZ]), by_qz = P2(B[1][V_QZ]), bz_qz = P2(B[2][V_QZ]);
  const Pair bx_pr = P2(B[0][V_PR]), by_pr = P2(B[1][V_PR]), bz_pr = P2(B[2][V_PR]);
  const T* any = A(H->fb_maxp);  // periodic x/z never read their boundary planes
  const T* fyqx = H->periodic_y ? nullptr : A(H->fb_qx);
  const T* fyqy = H->periodic_y ? nullptr : A(H->fb_qy);
  const T* fyqz = H->periodic_y ? nullptr : A(H->fb_qz);
  const T* fypr = H->periodic_y ? nullptr : A(H->fb_pr);
  const T* fympr = H->periodic_y ? nullptr : A(H->fb_mpr);
  const double rre = H->rre, third = 1.0 / 3.0;
  const bool TH = H->thermo;
  // the advanced variable: momentum g for variable properties, velocity q otherwise
  double* ux = TH ? H->gx : H->qx;
  double* uy = TH ? H->gy : H->qy;
  double* uz = TH ? H->gz : H->qz;

  const int w0 = B[1][V_QY][0] == BC_DIRICHLET, w1 = B[1][V_QY][1] == BC_DIRICHLET;
  // fused path: the momentum advance u += m - bulk is not stored by itself but formed where the
  // Poisson right-hand side and the projection read u (both fused kernels must be available)
  const bool defer = fused_update_div<T>(H, isub, ux, uy, uz, w0, w1, false) &&
                     fused_project<T>(H, isub, ux, uy, uz, w0, w1, true, false);
  const bool mom_fused = fused_momentum<T>(H, isub, ux, uy, uz, defer);
  const bool upd = defer && mom_fused;
  if (!mom_fused) {
  // ---- 1. derived quantities (src/eq_momentum2.f90:347-508)
  run_op(H, 0, M1P2C, bx_qx, any, src(A(H->qx)), s_pcc, A(H->qxix), false, 1.0);
  run_op(H, 0, D1P2C, bx_qx, any, src(A(H->qx)), s_pcc, A(H->qxdx), false, 1.0);
  run_op(H, 1, D1C2P, by_qx, fyqx, src(A(H->qx)), s_pcc, A(H->qxdy), false, 1.0);
  run_op(H, 1, M1C2P, by_qx, fyqx, src(A(H->qx)), s_pcc, A(H->qxiy), false, 1.0);
  run_op(H, 2, M1C2P, bz_qx, any, src(A(H->qx)), s_pcc, A(H->qxiz), false, 1.0);
  run_op(H, 2, D1C2P, bz_qx, any, src(A(H->qx)), s_pcc, A(H->qxdz), false, 1.0);
  run_op(H, 0, D1C2P, bx_qy, any, src(A(H->qy)), s_cpc, A(H->qydx), false, 1.0);
  run_op(H, 0, M1C2P, bx_qy, any, src(A(H->qy)), s_cpc, A(H->qyix), false, 1.0);
  run_op(H, 1, D1P2C, by_qy, nullptr, src(A(H->qy)), s_cpc, A(H->qydy), false, 1.0);
  run_op(H, 1, M1P2C, by_qy, fyqy, src(A(H->qy)), s_cpc, A(H->qyiy), false, 1.0);
  run_op(H, 2, D1C2P, bz_qy, any, src(A(H->qy)), s_cpc, A(H->qydz), false, 1.0);
  run_op(H, 2, M1C2P, bz_qy, any, src(A(H->qy)), s_cpc, A(H->qyiz), false, 1.0);
  run_op(H, 0, D1C2P, bx_qz, any, src(A(H->qz)), s_ccp, A(H->qzdx), false, 1.0);
  run_op(H, 0, M1C2P, bx_qz, any, src(A(H->qz)), s_ccp, A(H->qzix), false, 1.0);
  run_op(H, 1, M1C2P, by_qz, fyqz, src(A(H->qz)), s_ccp, A(H->qziy), false, 1.0);
  run_op(H, 1, D1C2P, by_qz, fyqz, src(A(H->qz)), s_ccp, A(H->qzdy), false, 1.0);
  run_op(H, 2, M1P2C, bz_qz, any, src(A(H->qz)), s_ccp, A(H->qziz), false, 1.0);
  run_op(H, 2, D1P2C, bz_qz, nullptr, src(A(H->qz)), s_ccp, A(H->qzdz), false, 1.0);
  // ---- 1b. variable properties: interpolated g and mu (src/eq_momentum2.f90:576-703)
  if (TH) {
    const T* fz = A(H->fb_zero);  // no-slip walls: g = 0 there
    const Pair per = P2(kPer2);
    run_op(H, 0, M1P2C, bx_qx, any, src(A(H->gx)), s_pcc, A(H->gxix), false, 1.0);
    run_op(H, 1, M1C2P, by_qx, fz, src(A(H->gx)), s_pcc, A(H->gxiy), false, 1.0);
    run_op(H, 2, M1C2P, bz_qx, any, src(A(H->gx)), s_pcc, A(H->gxiz), false, 1.0);
    run_op(H, 0, M1C2P, bx_qy, any, src(A(H->gy)), s_cpc, A(H->gyix), false, 1.0);
    run_op(H, 1, M1P2C, by_qy, fz, src(A(H->gy)), s_cpc, A(H->gyiy), false, 1.0);
    run_op(H, 2, M1C2P, bz_qy, any, src(A(H->gy)), s_cpc, A(H->gyiz), false, 1.0);
    run_op(H, 0, M1C2P, bx_qz, any, src(A(H->gz)), s_ccp, A(H->gzix), false, 1.0);
    run_op(H, 1, M1C2P, by_qz, fz, src(A(H->gz)), s_ccp, A(H->gziy), false, 1.0);
    run_op(H, 2, M1P2C, bz_qz, any, src(A(H->gz)), s_ccp, A(H->gziz), false, 1.0);
    run_op(H, 1, M1C2P, H->ftpy, A(H->fb_m), src(A(H->mVisc)), s_ccc, A(H->muiy_cpc), false, 1.0);
    run_op(H, 0, M1C2P, per, any, src(A(H->muiy_cpc)), s_cpc, A(H->muixy_ppc), false, 1.0);
    run_op(H, 0, M1C2P, per, any, src(A(H->mVisc)), s_ccc, A(H->mu_pcc), false, 1.0);
    run_op(H, 2, M1C2P, per, nullptr, src(A(H->mu_pcc)), s_pcc, A(H->muixz_pcp), false, 1.0);
    run_op(H, 2, M1C2P, per, nullptr, src(A(H->muiy_cpc)), s_cpc, A(H->muiyz_cpp), false, 1.0);
  }
  // first factors of the convection products and viscosity factors of the stresses
  const T* c_xix = A(TH ? H->gxix : H->qxix);
  const T* c_yix = A(TH ? H->gyix : H->qyix);
  const T* c_zix = A(TH ? H->gzix : H->qzix);
  const T* c_xiy = A(TH ? H->gxiy : H->qxiy);
  const T* c_yiy = A(TH ? H->gyiy : H->qyiy);
  const T* c_ziy = A(TH ? H->gziy : H->qziy);
  const T* c_xiz = A(TH ? H->gxiz : H->qxiz);
  const T* c_yiz = A(TH ? H->gyiz : H->qyiz);
  const T* c_ziz = A(TH ? H->gziz : H->qziz);
  const T* mu_c = TH ? A(H->mVisc) : nullptr;
  const T* mu_xy = TH ? A(H->muixy_ppc) : nullptr;
  const T* mu_xz = TH ? A(H->muixz_pcp) : nullptr;
  const T* mu_yz = TH ? A(H->muiyz_cpp) : nullptr;

  // div = qxdx + qydy + qzdz (:512-534)
  PROFD(H, 3, 32.0 / 8.0 * sizeof(T) * H->n_ccc, bufs(H->qxdx, H->qydy, H->qzdz), bufs(H->div),
        launch_axpby(A(H->div), A(H->qxdx), 1.0, A(H->qydy), 1.0, (int64_t)H->n_ccc, st, A(H->qzdz), 1.0));
  H->launches += 1;
  if (H->fbcy_velo) {
    // wall divergence for the y-viscous boundary value (:374-442, :537-546)
    run_op(H, 0, D1P2C, bx_qx, nullptr, src(A(H->qxiy)), s_ppc, A(H->qxdx_cpc), false, 1.0);
    run_op(H, 1, D1C2P, by_qy, fyqy, src(A(H->qyiy)), s_ccc, A(H->qydy_cpc), false, 1.0);
    run_op(H, 2, D1P2C, bz_qz, nullptr, src(A(H->qziy)), s_cpp, A(H->qzdz_cpc), false, 1.0);
    // fbcy_div = walls of (qxdx + qydy + qzdz)_cpc; visc2 bc = (qydy_cpc - div/3) * 2 (:1156-1171)
    PROFD(H, 3, 32.0 / 8.0 * sizeof(T) * H->n_cpc, bufs(H->qydy_cpc, H->qzdz_cpc), bufs(H->qxdx_cpc),
          launch_axpby(A(H->qxdx_cpc), A(H->qxdx_cpc), 1.0, A(H->qydy_cpc), 1.0, (int64_t)H->n_cpc, st,
                       A(H->qzdz_cpc), 1.0));
    PROFD(H, 3, 48.0 / 8.0 * sizeof(T) * nc0 * nc2, bufs(H->qydy_cpc, H->qxdx_cpc, TH ? H->muiy_cpc : nullptr),
          bufs(H->fb_visc2),
         launch_fbcy_extract<T>(A(H->fb_visc2), A(H->qydy_cpc), A(H->qxdx_cpc), TH ? A(H->muiy_cpc) : nullptr,
                                -third, TH ? 2.0 : 1.0, 2.0, nc0, np1, nc2, st));
    H->launches += 2;
  }

  // ---- 2-3. momentum RHS and fractional step, one fused pass per component.  The convection and
  // diffusion terms of one direction share the operator (same family and boundary pair), and the
  // operator is linear in its input and boundary values, so op(conv) + rre*op(diff) is
  // op(conv + rre*diff); the three directions, the pressure gradient and the fractional step
  // (:35-71) are summed per output value.
  const int m_pcc[3] = {np0, nc1, nc2}, m_cpc[3] = {nc0, np1, nc2}, m_ccp[3] = {nc0, nc1, np2};
  // y and z: the fractional step's pressure-gradient operator also advances q (update_q with no
  // mass-flux correction); x waits for the mass-flux mean
  bool y_advanced = false, z_advanced = false;
  // x-momentum (:796-966)
  {
    std::vector<OpTerm<T>> t;
    pair_terms(t, 0, D1C2P, H->mbcx_cov1, any, prod(c_xix, A(H->qxix), -1.0), H->mbcx_tau1, any,
               linm(A(H->qxdx), A(H->div), -third, 2.0, mu_c), rre, s_ccc, nullptr, 0);
    pair_terms(t, 1, D1P2C, H->mbcy_cov1, nullptr, prod(c_yix, A(H->qxiy), -1.0), H->mbcy_tau1, nullptr,
               linm(A(H->qxdy), A(H->qydx), 1.0, 1.0, mu_xy), rre, s_ppc, nullptr, 0);
    pair_terms(t, 2, D1P2C, H->mbcz_cov1, nullptr, prod(c_zix, A(H->qxiz), -1.0), H->mbcz_tau1, nullptr,
               linm(A(H->qxdz), A(H->qzdx), 1.0, 1.0, mu_xz), rre, s_pcp, nullptr, 0);
    t.push_back(term<T>(0, D1C2P, bx_pr, any, src(A(H->pres), -1.0), s_ccc, 1.0, 1));
    run_fused<T>(H, t, A(H->mx), m_pcc, EP_FRAC, A(H->mx0), isub, A(H->px));
  }
  // y-momentum (:978-1242)
  if (H->fbcy_velo) {
    PROFD(H, 3, 24.0 / 8.0 * sizeof(T) * 4 * nc0 * nc2, bufs(H->fb_conv2, H->fb_visc2), bufs(H->fb_comb),
          launch_axpby(A(H->fb_comb), A(H->fb_conv2), 1.0, A(H->fb_visc2), rre, (int64_t)4 * nc0 * nc2, st));
    H->launches++;
  }
  {
    std::vector<OpTerm<T>> t;
    pair_terms(t, 0, D1P2C, H->mbcx_cov2, nullptr, prod(c_xiy, A(H->qyix), -1.0), H->mbcx_tau2, nullptr,
               linm(A(H->qxdy), A(H->qydx), 1.0, 1.0, mu_xy), rre, s_ppc, nullptr, 0);
    pair_terms(t, 1, D1C2P, H->mbcy_cov2, H->fbcy_velo ? A(H->fb_conv2) : A(H->fb_maxp),
               prod(A(H->qyiy), c_yiy, -1.0), H->mbcy_tau2, H->fbcy_velo ? A(H->fb_visc2) : A(H->fb_maxp),
               linm(A(H->qydy), A(H->div), -third, 2.0, mu_c), rre, s_ccc, A(H->fb_comb), 0);
    pair_terms(t, 2, D1P2C, H->mbcz_cov2, nullptr, prod(A(H->qyiz), c_ziy, -1.0), H->mbcz_tau2, nullptr,
               linm(A(H->qzdy), A(H->qydz), 1.0, 1.0, mu_yz), rre, s_cpp, nullptr, 0);
    t.push_back(term<T>(1, D1C2P, by_pr, fympr, src(A(H->pres), -1.0), s_ccc, 1.0, 1));
    y_advanced = run_fused<T>(H, t, A(H->my), m_cpc, EP_FRAC, A(H->my0), isub, A(H->py), nullptr, false, false,
                              A(uy));
  }
  // z-momentum (:1262-1457)
  {
    std::vector<OpTerm<T>> t;
    pair_terms(t, 0, D1P2C, H->mbcx_cov3, nullptr, prod(c_xiz, A(H->qzix), -1.0), H->mbcx_tau3, nullptr,
               linm(A(H->qxdz), A(H->qzdx), 1.0, 1.0, mu_xz), rre, s_pcp, nullptr, 0);
    pair_terms(t, 1, D1P2C, H->mbcy_cov3, nullptr, prod(c_yiz, A(H->qziy), -1.0), H->mbcy_tau3, nullptr,
               linm(A(H->qzdy), A(H->qydz), 1.0, 1.0, mu_yz), rre, s_cpp, nullptr, 0);
    pair_terms(t, 2, D1C2P, H->mbcz_cov3, any, prod(c_ziz, A(H->qziz), -1.0), H->mbcz_tau3, any,
               linm(A(H->qzdz), A(H->div), -third, 2.0, mu_c), rre, s_ccc, nullptr, 0);
    t.push_back(term<T>(2, D1C2P, bz_pr, any, src(A(H->pres), -1.0), s_ccc, 1.0, 1));
    z_advanced = run_fused<T>(H, t, A(H->mz), m_ccp, EP_FRAC, A(H->mz0), isub, A(H->pz), nullptr, false, false,
                              A(uz));
  }

  // ---- 3b. mass flux
  const double* bulk = nullptr;
  if (H->idriven == 1) {
    PROFD(H, 3, 8.0 / 8.0 * sizeof(T) * H->n_pcc, bufs(H->mx, H->wy), bufs(H->partial, H->scal),
         launch_weighted_mean(A(H->mx), H->wy, np0, nc1, nc2, H->partial, H->npart, H->scal + 0, H->vol, st));
    bulk = H->scal + 0;
    H->launches += 2;
  }
  // ---- 4. q += rhs, walls
  PROFD(H, 3, 24.0 / 8.0 * sizeof(T) * H->n_pcc, bufs(H->mx, bulk), bufs(ux),
        launch_update_q(A(ux), A(H->mx), bulk, (int64_t)H->n_pcc, st));
  if (!y_advanced) {
    PROFD(H, 3, 24.0 / 8.0 * sizeof(T) * H->n_cpc, bufs(H->my), bufs(uy),
          launch_update_q(A(uy), A(H->my), nullptr, (int64_t)H->n_cpc, st));
    H->launches++;
  }
  if (!z_advanced) {
    PROFD(H, 3, 24.0 / 8.0 * sizeof(T) * H->n_ccp, bufs(H->mz), bufs(uz),
          launch_update_q(A(uz), A(H->mz), nullptr, (int64_t)H->n_ccp, st));
    H->launches++;
  }
  H->launches += 1;
  if (w0 || w1) {
    PROFD(H, 3, 16.0 / 8.0 * sizeof(T) * nc0 * nc2, bufs(), bufs(uy),
          launch_set_yrows(A(uy), nc0, np1, nc2, w0, H->fbcy[V_QY][0], w1, H->fbcy[V_QY][1], st));
    H->launches++;
  }
  }  // operator path
  // ---- 5. Poisson RHS, solve, pressure and projection.  For variable properties the reference
  // adds (rho - rho_m1)/dt (Calculate_drhodt, src/eq_continuity.f90:26-78), but
  // Update_thermal_properties has already set rho_m1 = rho, so the term is zero and left out.
  const double coeff = 1.0 / (H->tAlpha[isub] * H->sigma2p * H->dt);
  if (upd) {
    fused_update_div<T>(H, isub, ux, uy, uz, w0, w1, true);
  } else {
    std::vector<OpTerm<T>> t = {term<T>(0, D1P2C, bx_qx, any, src(A(ux)), s_pcc, coeff, 0),
                                term<T>(1, D1P2C, by_qy, nullptr, src(A(uy)), s_cpc, coeff, 0),
                                term<T>(2, D1P2C, bz_qz, nullptr, src(A(uz)), s_ccp, coeff, 0)};
    // the divergence of three single-array terms: one fused pass (measured faster than three
    // accumulating operators; the momentum sums are not)
    run_fused<T>(H, t, A(H->pcor), s_ccc, EP_STORE, nullptr, isub, nullptr, nullptr, false, true);
  }
  poisson_device<T>(H, A(H->pcor));
  if (fused_project<T>(H, isub, ux, uy, uz, w0, w1, upd, true)) return;
  PROFD(H, 3, 24.0 / 8.0 * sizeof(T) * H->n_ccc, bufs(H->pcor), bufs(H->pres),
        launch_axpby(A(H->pres), A(H->pres), 1.0, A(H->pcor), 1.0, (int64_t)H->n_ccc, st));
  H->launches++;
  const double f = H->dt * H->tAlpha[isub] * H->sigma2p;
  run_op(H, 0, D1C2P, bx_pr, any, src(A(H->pcor)), s_ccc, A(ux), true, -f);
  run_op(H, 1, D1C2P, by_pr, fypr, src(A(H->pcor)), s_ccc, A(uy), true, -f);
  run_op(H, 2, D1C2P, bz_pr, any, src(A(H->pcor)), s_ccc, A(uz), true, -f);
  if (w0 || w1) {
    PROFD(H, 3, 16.0 / 8.0 * sizeof(T) * nc0 * nc2, bufs(), bufs(uy),
          launch_set_yrows(A(uy), nc0, np1, nc2, w0, H->fbcy[V_QY][0], w1, H->fbcy[V_QY][1], st));
    H->launches++;
  }
  // ---- 6. variable properties: q = g / rho_face (convert_primary_conservative IG2Q,
  // src/para_conversion.f90:5-227), the interpolation and the division in one pass per direction
  if (TH) {
    const Pair per = P2(kPer2);
    run_op(H, 0, M1C2P, per, any, src(A(H->dDens)), s_ccc, A(H->qx), false, 1.0, O_DIV, A(H->gx));
    run_op(H, 1, M1C2P, H->ftpy, A(H->fb_d), src(A(H->dDens)), s_ccc, A(H->qy), false, 1.0, O_DIV, A(H->gy));
    run_op(H, 2, M1C2P, per, any, src(A(H->dDens)), s_ccc, A(H->qz), false, 1.0, O_DIV, A(H->gz));
  }
}

// Solve_energy_eq (src/eq_energy.f90:405-458): energy RHS (Compute_energy_rhs, :179-401), the
// fractional step (:148-177), rho*h update and property update (:14-146).  The y diffusion
// boundary value is the wall row of kappa*dT/dy (the reference tests the x-velocity flag there and
// passes MAXP for an x-periodic channel); the top wall state uses row np(2) of the interpolated
// rho*h (the reference indexes np(1)).
template <typename T>
void energy_body_t(chs_handle* H, int isub) {
  if (fused_energy<T>(H, isub)) return;
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const int nc0 = H->nc[0], nc1 = H->nc[1], nc2 = H->nc[2];
  const int np0 = H->np[0], np1 = H->np[1], np2 = H->np[2];
  const int s_pcc[3] = {np0, nc1, nc2}, s_cpc[3] = {nc0, np1, nc2}, s_ccp[3] = {nc0, nc1, np2};
  const int s_ccc[3] = {nc0, nc1, nc2};
  const auto& B = H->ibc;
  const T* any = A(H->fb_maxp);
  const T* fz = A(H->fb_zero);
  const Pair per = P2(kPer2);
  const double rpr = H->rPrRen;
  // faces of h and kappa; temperature gradients
  run_op(H, 0, M1C2P, per, any, src(A(H->hEnth)), s_ccc, A(H->h_pcc), false, 1.0);
  run_op(H, 1, M1C2P, H->ftpy, A(H->fb_h), src(A(H->hEnth)), s_ccc, A(H->h_cpc), false, 1.0);
  run_op(H, 2, M1C2P, per, any, src(A(H->hEnth)), s_ccc, A(H->h_ccp), false, 1.0);
  run_op(H, 0, M1C2P, per, any, src(A(H->kCond)), s_ccc, A(H->k_pcc), false, 1.0);
  run_op(H, 1, M1C2P, H->ftpy, A(H->fb_k), src(A(H->kCond)), s_ccc, A(H->k_cpc), false, 1.0);
  run_op(H, 2, M1C2P, per, any, src(A(H->kCond)), s_ccc, A(H->k_ccp), false, 1.0);
  run_op(H, 0, D1C2P, P2(B[0][V_TM]), fz, src(A(H->tTemp)), s_ccc, A(H->dTx), false, 1.0);
  run_op(H, 1, D1C2P, P2(B[1][V_TM]), A(H->fb_qw), src(A(H->tTemp)), s_ccc, A(H->dTy), false, 1.0);
  run_op(H, 2, D1C2P, P2(B[2][V_TM]), fz, src(A(H->tTemp)), s_ccc, A(H->dTz), false, 1.0);
  PROFD(H, 3, 3.0 * sizeof(T) * nc0 * nc2, bufs(H->dTy, H->k_cpc), bufs(H->fb_dtk),
        launch_fbcy_extract<T>(A(H->fb_dtk), A(H->dTy), nullptr, A(H->k_cpc), 0.0, 1.0, 1.0, nc0, np1, nc2, st));
  H->launches++;
  // conv + diffusion per direction, the fractional step, the rho*h update and (table mode) the
  // property update in one fused pass
  const bool table_props = H->mlp_mode != 1;
  {
    std::vector<OpTerm<T>> t;
    pair_terms(t, 0, D1P2C, H->ebcx_conv, any, prod(A(H->gx), A(H->h_pcc), -1.0), H->ebcx_difu, any,
               prod(A(H->dTx), A(H->k_pcc), 1.0), rpr, s_pcc, nullptr, 0);
    t.push_back(term<T>(1, D1P2C, H->ebcy_conv, nullptr, prod(A(H->gy), A(H->h_cpc), -1.0), s_cpc, 1.0, 0));
    t.push_back(term<T>(1, D1P2C, H->ebcy_difu, A(H->fb_dtk), prod(A(H->dTy), A(H->k_cpc), 1.0), s_cpc, rpr, 0));
    pair_terms(t, 2, D1P2C, H->ebcz_conv, nullptr, prod(A(H->gz), A(H->h_ccp), -1.0), H->ebcz_difu, nullptr,
               prod(A(H->dTz), A(H->k_ccp), 1.0), rpr, s_ccp, nullptr, 0);
    run_fused<T>(H, t, A(H->erhs), s_ccc, EP_ENERGY, A(H->erhs0), isub, nullptr, A(H->rhoh), table_props);
  }
  if (!table_props) {
    PROFD(H, 3, 6.0 * sizeof(T) * H->n_ccc, bufs(H->rhoh, H->mlp_wpack),
          bufs(H->hEnth, H->tTemp, H->kCond, H->dDens, H->mVisc, H->mlp_nfb),
         launch_mlp_props<T>(H->tab, H->mlp_norm, H->mlp_small, H->mlp_check, H->mlp_wpack, A(H->rhoh),
                             A(H->hEnth), A(H->tTemp), A(H->kCond), A(H->dDens), A(H->mVisc), (int64_t)H->n_ccc,
                             H->mlp_nfb, st));
    H->launches++;
  }
  const int s0 = B[1][V_TM][0] == BC_NEUMANN, s1 = B[1][V_TM][1] == BC_NEUMANN;
  if (s0 || s1) {
    run_op(H, 1, M1C2P, H->ftpy, nullptr, src(A(H->rhoh)), s_ccc, A(H->dh_cpc), false, 1.0);
    PROFD(H, 3, 10.0 * sizeof(T) * nc0 * nc2, bufs(H->dh_cpc), bufs(H->fb_h, H->fb_k, H->fb_m, H->fb_d),
         launch_wall_props<T>(H->tab, A(H->dh_cpc), nc0, np1, nc2, s0, s1, A(H->fb_h), A(H->fb_k), A(H->fb_m),
                              A(H->fb_d), st));
    H->launches++;
  }
}

void substep_body(chs_handle* H, int isub, int parts = PART_ALL) {
  if (H->mixed) substep_body_t<float>(H, isub, parts);
  else substep_body_t<double>(H, isub, parts);
}

// Prepare every plan the substep uses (plans are host objects; the table must be final
// before the graph is captured).
void prepare_plans(chs_handle* H) {
  // dry run on a null stream is not possible; instead enumerate through a throw-away pass that
  // only builds plans: run_op builds the plan before launching, so a capture-free first substep
  // would launch kernels.  Plans are built here explicitly in the same order.
  struct Rec { int d, fam; Pair bc; bool f; };
  const auto& B = H->ibc;
  const bool y = !H->periodic_y;
  std::vector<Rec> r = {
      {0, M1P2C, P2(B[0][V_QX]), true}, {0, D1P2C, P2(B[0][V_QX]), true}, {1, D1C2P, P2(B[1][V_QX]), y},
      {1, M1C2P, P2(B[1][V_QX]), y}, {2, M1C2P, P2(B[2][V_QX]), true}, {2, D1C2P, P2(B[2][V_QX]), true},
      {0, D1C2P, P2(B[0][V_QY]), true}, {0, M1C2P, P2(B[0][V_QY]), true}, {1, D1P2C, P2(B[1][V_QY]), false},
      {1, M1P2C, P2(B[1][V_QY]), y}, {2, D1C2P, P2(B[2][V_QY]), true}, {2, M1C2P, P2(B[2][V_QY]), true},
      {0, D1C2P, P2(B[0][V_QZ]), true}, {0, M1C2P, P2(B[0][V_QZ]), true}, {1, M1C2P, P2(B[1][V_QZ]), y},
      {1, D1C2P, P2(B[1][V_QZ]), y}, {2, M1P2C, P2(B[2][V_QZ]), true}, {2, D1P2C, P2(B[2][V_QZ]), false},
      {0, D1C2P, H->mbcx_cov1, true}, {1, D1P2C, H->mbcy_cov1, false}, {2, D1P2C, H->mbcz_cov1, false},
      {0, D1C2P, P2(B[0][V_PR]), true}, {0, D1C2P, H->mbcx_tau1, true}, {1, D1P2C, H->mbcy_tau1, false},
      {2, D1P2C, H->mbcz_tau1, false}, {0, D1P2C, H->mbcx_cov2, false}, {1, D1C2P, H->mbcy_cov2, true},
      {2, D1P2C, H->mbcz_cov2, false}, {1, D1C2P, P2(B[1][V_PR]), y}, {0, D1P2C, H->mbcx_tau2, false},
      {1, D1C2P, H->mbcy_tau2, true}, {2, D1P2C, H->mbcz_tau2, false}, {0, D1P2C, H->mbcx_cov3, false},
      {1, D1P2C, H->mbcy_cov3, false}, {2, D1C2P, H->mbcz_cov3, true}, {2, D1C2P, P2(B[2][V_PR]), true},
      {0, D1P2C, H->mbcx_tau3, false}, {1, D1P2C, H->mbcy_tau3, false}, {2, D1C2P, H->mbcz_tau3, true},
      {0, D1P2C, P2(B[0][V_QX]), true}, {1, D1P2C, P2(B[1][V_QY]), false}, {2, D1P2C, P2(B[2][V_QZ]), false},
      {0, D1C2P, P2(B[0][V_PR]), true}, {1, D1C2P, P2(B[1][V_PR]), y}, {2, D1C2P, P2(B[2][V_PR]), true},
      {0, M1P2C, P2(B[0][V_QX]), true}, {1, M1P2C, P2(B[1][V_QY]), y}, {2, M1P2C, P2(B[2][V_QZ]), true},
  };
  if (H->fbcy_velo) {
    r.push_back({0, D1P2C, P2(B[0][V_QX]), false});
    r.push_back({1, D1C2P, P2(B[1][V_QY]), true});
    r.push_back({2, D1P2C, P2(B[2][V_QZ]), false});
  }
  for (const auto& x : r) H->plan(x.d, x.fam, x.bc, x.f);
  upload_table(H);
  upload_fz_rows(H);
}

// operator plans of the variable-property path (energy equation, g and mu interpolations,
// q <-> g conversion), in the order energy_body_t and substep_body_t use them
void prepare_thermo_plans(chs_handle* H) {
  const auto& B = H->ibc;
  const Pair per = P2(kPer2);
  struct Rec { int d, fam; Pair bc; bool f; };
  const std::vector<Rec> r = {
      {0, M1C2P, per, true}, {1, M1C2P, H->ftpy, true}, {2, M1C2P, per, true},
      {0, D1C2P, P2(B[0][V_TM]), true}, {1, D1C2P, P2(B[1][V_TM]), true}, {2, D1C2P, P2(B[2][V_TM]), true},
      {0, D1P2C, H->ebcx_conv, true}, {0, D1P2C, H->ebcx_difu, true},
      {1, D1P2C, H->ebcy_conv, false}, {1, D1P2C, H->ebcy_difu, true},
      {2, D1P2C, H->ebcz_conv, false}, {2, D1P2C, H->ebcz_difu, false},
      {1, M1C2P, H->ftpy, false},
      {0, M1P2C, P2(B[0][V_QX]), true}, {1, M1C2P, P2(B[1][V_QX]), true}, {2, M1C2P, P2(B[2][V_QX]), true},
      {0, M1C2P, P2(B[0][V_QY]), true}, {1, M1P2C, P2(B[1][V_QY]), true}, {2, M1C2P, P2(B[2][V_QY]), true},
      {0, M1C2P, P2(B[0][V_QZ]), true}, {1, M1C2P, P2(B[1][V_QZ]), true}, {2, M1P2C, P2(B[2][V_QZ]), true},
      {2, M1C2P, per, false},
  };
  for (const auto& x : r) H->plan(x.d, x.fam, x.bc, x.f);
  upload_table(H);
  upload_fz_rows(H);
}

// host-side lookup of the initial state from T (ftp_refresh_thermal_properties_from_T_undim,
// src/input_thermo.f90:272-307): bisection on the T column with the reference's sign test
struct HostFtp { double h, d, m, k, rhoh; };
HostFtp host_ftp_from_t(const chs_thermo* c, double t) {
  int a = 0, b = c->ntable - 1;
  while (b - a > 1) {
    const int m = a + (b - a) / 2;
    if ((c->t[a] - t) * (c->t[m] - t) > 1.0e-20) a = m;
    else b = m;
  }
  const double w1 = (c->t[b] - t) / (c->t[b] - c->t[a]), w2 = 1.0 - w1;
  HostFtp f;
  f.h = w1 * c->h[a] + w2 * c->h[b];
  f.d = w1 * c->d[a] + w2 * c->d[b];
  f.m = w1 * c->m[a] + w2 * c->m[b];
  f.k = w1 * c->k[a] + w2 * c->k[b];
  f.rhoh = f.d * f.h;
  return f;
}

template <typename T>
void thermo_fill_t(chs_handle* H, const HostFtp& f, double t_ini) {
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const int64_t n = (int64_t)H->n_ccc;
  const int64_t nl = (int64_t)H->nc[0] * H->nc[2];
  cudaStream_t st = H->st;
  launch_fill(A(H->rhoh), f.rhoh, n, st);
  launch_fill(A(H->hEnth), f.h, n, st);
  launch_fill(A(H->tTemp), t_ini, n, st);
  launch_fill(A(H->kCond), f.k, n, st);
  launch_fill(A(H->dDens), f.d, n, st);
  launch_fill(A(H->mVisc), f.m, n, st);
  launch_fill(A(H->fb_h), f.h, 4 * nl, st);
  launch_fill(A(H->fb_k), f.k, 4 * nl, st);
  launch_fill(A(H->fb_m), f.m, 4 * nl, st);
  launch_fill(A(H->fb_d), f.d, 4 * nl, st);
  // get_fbcy_iTh (src/bc_general.f90:784-805): planes 1, 2 = dT/dy at the Neumann walls, 3, 4 = 0
  launch_fill(A(H->fb_qw), H->fbcy[V_TM][0], nl, st);
  launch_fill(A(H->fb_qw) + nl, H->fbcy[V_TM][1], nl, st);
  H->launches += 12;
  // g = q * rho_face (convert_primary_conservative IQ2G, src/initialisation.f90:389)
  const int s_ccc[3] = {H->nc[0], H->nc[1], H->nc[2]};
  const Pair per = P2(kPer2);
  const T* any = A(H->fb_maxp);
  run_op(H, 0, M1C2P, per, any, src(A(H->dDens)), s_ccc, A(H->gx), false, 1.0, O_MUL, A(H->qx));
  run_op(H, 1, M1C2P, H->ftpy, A(H->fb_d), src(A(H->dDens)), s_ccc, A(H->gy), false, 1.0, O_MUL, A(H->qy));
  run_op(H, 2, M1C2P, per, any, src(A(H->dDens)), s_ccc, A(H->gz), false, 1.0, O_MUL, A(H->qz));
}

// error bound of the network's T (fraction of the table's T range) and the same bound in table rows;
// tol = 0: no network hint (every cell searches the table from scratch)
void set_mlp_tol(MlpCheck& ck, double tol, int n) {
  ck.tol = tol;
  ck.raw = 0;
  ck.win = tol > 0.0 ? std::max(1, (int)std::ceil(tol * (n - 1))) : -1;
}

void thermo_init(chs_handle* H, const chs_thermo* c) {
  if (H->periodic_y) throw std::invalid_argument("variable properties need the channel (y walls)");
  for (int v = V_QX; v <= V_QZ; ++v)
    if (H->fbcy[v][0] != 0.0 || H->fbcy[v][1] != 0.0)
      throw std::invalid_argument("variable properties need walls at rest");
  for (int n = 0; n < 2; ++n) {
    if (H->ibc[1][V_TM][n] != BC_NEUMANN) throw std::invalid_argument("variable properties need isoflux (Neumann T) y walls");
    if (H->ibc[0][V_TM][n] != BC_PERIODIC || H->ibc[2][V_TM][n] != BC_PERIODIC)
      throw std::invalid_argument("T must be periodic in x and z");
  }
  const int n = c->ntable;
  if (n < 2 || !c->t || !c->h || !c->d || !c->m || !c->k) throw std::invalid_argument("property table missing");
  std::vector<double> rhoh(n);
  for (int i = 0; i < n; ++i) rhoh[i] = c->d[i] * c->h[i];
  for (int i = 1; i < n; ++i) {
    if (!(c->t[i] > c->t[i - 1])) throw std::invalid_argument("property table must be sorted by increasing T");
    if (!(rhoh[i] > rhoh[i - 1]) || !(c->h[i] > c->h[i - 1]))
      throw std::invalid_argument("rho*h and h must increase with T for the rho*h lookup");
  }
  if (!(c->t_ini >= c->t[0] && c->t_ini <= c->t[n - 1])) throw std::invalid_argument("t_ini outside the table");
  double* cols = H->dalloc<double>((size_t)6 * n);
  const double* srcs[6] = {c->t, c->h, c->d, c->m, c->k, rhoh.data()};
  for (int j = 0; j < 6; ++j)
    CK(cudaMemcpyAsync(cols + (size_t)j * n, srcs[j], n * sizeof(double), cudaMemcpyHostToDevice, H->st));
  H->tab = ThermoTab{cols, cols + n, cols + 2 * n, cols + 3 * n, cols + 4 * n, cols + 5 * n, n,
                     *std::min_element(rhoh.begin(), rhoh.end()), *std::max_element(rhoh.begin(), rhoh.end())};
  {
    // bracket index of the strictly increasing rho*h and h columns (2n bins each).  For x fixed,
    // the sign test (col[a]-x)*(col[m]-x) > MINP holds on two rays (below col[a], above col[m])
    // and fails on the interval between them, so when both ends of a bin (widened by 1e-6 of a bin
    // against rounding of the bin index) take the same branch, and for the 'a = m' branch lie on
    // the same ray, every value of the bin takes that branch.  The index stores the state where
    // the ends first part; the device search continues from it along the same path.
    const int nb = 2 * n;
    std::vector<int> ixh(4 * (size_t)nb);
    const double* icol[2] = {rhoh.data(), c->h};
    for (int q = 0; q < 2; ++q) {
      const double* col = icol[q];
      const double lo = col[0], hi = col[n - 1], w = (hi - lo) / nb;
      const double del = std::max(1e-6 * w, 1e-13 * std::max(std::fabs(lo), std::fabs(hi)));
      for (int bi = 0; bi < nb; ++bi) {
        const double xl = lo + bi * w - del, xh = lo + (bi + 1) * w + del;
        int a = 0, b = n - 1;
        while (b - a > 1) {
          const int m = a + (b - a) / 2;
          const double ca = col[a], cm = col[m];
          const bool dl = (ca - xl) * (cm - xl) > 1.0e-20, dh = (ca - xh) * (cm - xh) > 1.0e-20;
          if (dl != dh || (dl && ((xl < ca) != (xh < ca)))) break;
          if (dl) a = m;
          else b = m;
        }
        ixh[(size_t)q * 2 * nb + 2 * bi] = a;
        ixh[(size_t)q * 2 * nb + 2 * bi + 1] = b;
      }
      H->tab.ix_lo[q] = lo;
      H->tab.ix_hi[q] = hi;
      H->tab.ix_iw[q] = 1.0 / w;
    }
    int2* ixd = H->dalloc<int2>(2 * (size_t)nb);
    CK(cudaMemcpyAsync(ixd, ixh.data(), ixh.size() * sizeof(int), cudaMemcpyHostToDevice, H->st));
    H->tab.ix[0] = ixd;
    H->tab.ix[1] = ixd + nb;
    H->tab.ix_nb = nb;
  }
  H->rPrRen = c->rPrRen;
  H->tab_host_t.assign(c->t, c->t + n);
  H->tab_host_rhoh = rhoh;
  {
    // normalisation of the surrogate: rho*h over the table range, outputs over their column ranges
    MlpNorm& nm = H->mlp_norm;
    nm.xa = 2.0 / (H->tab.dhmax - H->tab.dhmin);
    nm.xb = -1.0 - nm.xa * H->tab.dhmin;
    const double* cols[4] = {c->t, c->d, c->m, c->k};
    for (int j = 0; j < 4; ++j) {
      const double lo = *std::min_element(cols[j], cols[j] + n), hi = *std::max_element(cols[j], cols[j] + n);
      nm.ya[j] = hi > lo ? 0.5 * (hi - lo) : 1.0;
      nm.yb[j] = 0.5 * (hi + lo);
    }
    MlpCheck& ck = H->mlp_check;
    ck.t0 = c->t[0];
    ck.dt_tab = (c->t[n - 1] - c->t[0]) / (n - 1);
    double dev = 0.0;
    for (int i = 0; i < n; ++i) dev = std::max(dev, std::fabs(c->t[i] - (ck.t0 + i * ck.dt_tab)));
    ck.uniform_t = dev <= 1e-9 * (c->t[n - 1] - c->t[0]) ? 1 : 0;
    set_mlp_tol(ck, 1.0e-4, n);
  }
  const size_t nc = H->n_ccc;
  for (double** p : {&H->rhoh, &H->hEnth, &H->tTemp, &H->kCond, &H->dDens, &H->mVisc, &H->erhs, &H->erhs0,
                     &H->gxix, &H->gyiy, &H->gziz, &H->h_pcc, &H->h_ccp, &H->k_pcc, &H->k_ccp, &H->dTx, &H->dTz,
                     &H->mu_pcc})
    *p = H->dalloc<double>(nc + (size_t)H->nc[1] * H->nc[2] + (size_t)H->nc[0] * H->nc[1]);
  H->gx = H->dalloc<double>(H->n_pcc); H->gy = H->dalloc<double>(H->n_cpc); H->gz = H->dalloc<double>(H->n_ccp);
  for (double** p : {&H->gxiy, &H->gyix, &H->muixy_ppc}) *p = H->dalloc<double>(H->n_ppc);
  for (double** p : {&H->gxiz, &H->gzix, &H->muixz_pcp}) *p = H->dalloc<double>(H->n_pcp);
  for (double** p : {&H->gyiz, &H->gziy, &H->muiyz_cpp}) *p = H->dalloc<double>(H->n_cpp);
  for (double** p : {&H->muiy_cpc, &H->h_cpc, &H->k_cpc, &H->dTy, &H->dh_cpc}) *p = H->dalloc<double>(H->n_cpc);
  const size_t nl = (size_t)H->nc[0] * H->nc[2];
  for (double** p : {&H->fb_h, &H->fb_k, &H->fb_m, &H->fb_d, &H->fb_qw, &H->fb_zero, &H->fb_dtk})
    *p = H->dalloc<double>(4 * nl);
  H->thermo = true;
  prepare_thermo_plans(H);
  const HostFtp f = host_ftp_from_t(c, c->t_ini);
  if (H->mixed) thermo_fill_t<float>(H, f, c->t_ini);
  else thermo_fill_t<double>(H, f, c->t_ini);
  CK(cudaStreamSynchronize(H->st));
}

// ---- MLP surrogate: training and evaluation -------------------------------------------------
struct MlpBuffers {
  float *grads = nullptr, *m = nullptr, *v = nullptr, *work = nullptr, *xs = nullptr, *ys = nullptr;
  float *bx = nullptr, *bt = nullptr, *loss = nullptr;
  int B = 0, N = 0;
};

void mlp_alloc_core(chs_handle* H) {
  if (H->mlp_params) return;
  H->mlp_params = H->dalloc<float>(MLP_NPARAM);
  H->mlp_wpack = H->dalloc<uint16_t>(2 * 4096);
  H->mlp_nfb = H->dalloc<unsigned long long>(1);
}

// Xavier-uniform weights from a seeded splitmix64 stream, zero biases
void mlp_init_host(std::vector<float>& p, uint64_t seed) {
  p.assign(MLP_NPARAM, 0.0f);
  uint64_t st = seed;
  auto next = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int fan_out, int fan_in) {
    const double lim = std::sqrt(6.0 / (fan_in + fan_out));
    for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = (float)((2.0 * next() - 1.0) * lim);
  };
  fill(MLP_P_W1, MLP_H, 1);
  fill(MLP_P_W2, MLP_H, MLP_H);
  fill(MLP_P_W3, MLP_H, MLP_H);
  fill(MLP_P_W4, MLP_NOUT, MLP_H);
}

// host copy of the small layers and the BF16 packing of the 64x64 layers
void mlp_finalize(chs_handle* H) {
  std::vector<float> p(MLP_NPARAM);
  CK(cudaMemcpyAsync(p.data(), H->mlp_params, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, H->st));
  CK(cudaStreamSynchronize(H->st));
  MlpSmall& sm = H->mlp_small;
  for (int i = 0; i < MLP_H; ++i) {
    sm.w1[i] = p[MLP_P_W1 + i];
    sm.b1[i] = p[MLP_P_B1 + i];
    sm.b2[i] = p[MLP_P_B2 + i];
    sm.b3[i] = p[MLP_P_B3 + i];
  }
  for (int i = 0; i < MLP_NOUT * MLP_H; ++i) sm.w4[i] = p[MLP_P_W4 + i];
  for (int i = 0; i < MLP_NOUT; ++i) sm.b4[i] = p[MLP_P_B4 + i];
  mlp_pack(H->mlp_params, H->mlp_wpack, H->st);
  H->launches++;
  H->mlp_ready = true;
}

void mlp_train(chs_handle* H, const chs_mlp_train_cfg* c, chs_mlp_report* rep) {
  if (!H->thermo) throw std::invalid_argument("the MLP surrogate needs chs_thermo_init");
  if (c->nsamples < 1024 || c->batch < 64 || c->batch > 65536 || c->epochs < 1 || !(c->lr > 0.0))
    throw std::invalid_argument("bad MLP training configuration");
  mlp_alloc_core(H);
  cudaStream_t st = H->st;
  const int N = c->nsamples, B = c->batch;
  MlpBuffers b;
  auto ta = [&](size_t n) {
    float* p = nullptr;
    CK(cudaMallocAsync(&p, n * sizeof(float), st));
    CK(cudaMemsetAsync(p, 0, n * sizeof(float), st));
    return p;
  };
  b.grads = ta(MLP_NPARAM); b.m = ta(MLP_NPARAM); b.v = ta(MLP_NPARAM);
  b.work = ta((size_t)8 * B * MLP_H); b.xs = ta(N); b.ys = ta((size_t)4 * N);
  b.bx = ta(B); b.bt = ta((size_t)4 * B); b.loss = ta(1);
  std::vector<float> p0;
  mlp_init_host(p0, c->seed);
  CK(cudaMemcpyAsync(H->mlp_params, p0.data(), MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
  mlp_make_samples(H->tab, H->mlp_norm, c->seed ^ 0x5A5A5A5Aull, N, b.xs, b.ys, st);
  const long long steps = (long long)c->epochs * ((N + B - 1) / B);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, st));
  const double pi = 3.141592653589793238462643383279502884;
  for (long long s = 1; s <= steps; ++s) {
    mlp_gather(b.xs, b.ys, N, c->seed, s, B, b.bx, b.bt, st);
    mlp_grad(H->mlp_params, b.bx, b.bt, B, b.grads, b.loss, b.work, st);
    // cosine decay to 1% of the initial rate
    const double lr = c->lr * (0.01 + 0.99 * 0.5 * (1.0 + std::cos(pi * (double)s / (double)steps)));
    mlp_adam(H->mlp_params, b.grads, b.m, b.v, MLP_NPARAM, (float)lr, s, st);
  }
  CK(cudaEventRecord(e1, st));
  CK(cudaGetLastError());
  CK(cudaEventSynchronize(e1));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  float loss = 0.0f;
  CK(cudaMemcpyAsync(&loss, b.loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  for (float* q : {b.grads, b.m, b.v, b.work, b.xs, b.ys, b.bx, b.bt, b.loss}) CK(cudaFreeAsync(q, st));
  CK(cudaStreamSynchronize(st));
  H->launches += steps * 15 + 2;
  mlp_finalize(H);
  rep->final_loss = loss;
  rep->train_ms = ms;
  rep->steps = (int)steps;
}

// network (with the per-cell check at tol; tol < 0 accepts every network value) on n host values
void mlp_eval(chs_handle* H, int n, const double* rhoh, double tol, double* out, unsigned long long* nfb) {
  if (!H->mlp_ready) throw std::invalid_argument("the MLP surrogate is not trained");
  cudaStream_t st = H->st;
  double* d = nullptr;
  unsigned long long* cnt = nullptr;
  CK(cudaMallocAsync(&d, (size_t)6 * n * sizeof(double), st));
  CK(cudaMallocAsync(&cnt, sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
  CK(cudaMemcpyAsync(d, rhoh, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
  MlpCheck ck = H->mlp_check;
  if (tol < 0.0) ck.raw = 1;
  else set_mlp_tol(ck, tol, H->tab.n);
  double *t = d + n, *rho = d + 2 * (size_t)n, *mu = d + 3 * (size_t)n, *ka = d + 4 * (size_t)n, *h = d + 5 * (size_t)n;
  launch_mlp_props<double>(H->tab, H->mlp_norm, H->mlp_small, ck, H->mlp_wpack, d, h, t, ka, rho, mu, n, cnt, st);
  H->launches++;
  CK(cudaGetLastError());
  // out[5][n] = T, rho, mu, kappa, h
  CK(cudaMemcpyAsync(out, t, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out + n, rho, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out + 2 * (size_t)n, mu, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out + 3 * (size_t)n, ka, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(out + 4 * (size_t)n, h, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(nfb, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CK(cudaFreeAsync(d, st));
  CK(cudaFreeAsync(cnt, st));
  CK(cudaStreamSynchronize(st));
  if (*nfb >> 62) throw std::runtime_error("MLP inference: tensor-core wait timed out");
}

void set_err(chs_handle* H, const char* fmt, ...) {
  if (!H) return;
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  H->err = buf;
}

int guard(chs_handle* H, const std::function<void()>& f) {
  try {
    f();
    return CHS_OK;
  } catch (const CudaError& e) {
    set_err(H, "%s", e.what());
    return CHS_ERR_CUDA;
  } catch (const std::invalid_argument& e) {
    set_err(H, "%s", e.what());
    return CHS_ERR_ARG;
  } catch (const std::exception& e) {
    set_err(H, "%s", e.what());
    return CHS_ERR_ARG;
  }
}

double* field_ptr(chs_handle* H, int field, size_t* n) {
  switch (field) {
    case CHS_QX: *n = H->n_pcc; return H->qx;
    case CHS_QY: *n = H->n_cpc; return H->qy;
    case CHS_QZ: *n = H->n_ccp; return H->qz;
    case CHS_PRES: *n = H->n_ccc; return H->pres;
    case CHS_PCOR: *n = H->n_ccc; return H->pcor;
    case CHS_MX_RHS0: *n = H->n_pcc; return H->mx0;
    case CHS_MY_RHS0: *n = H->n_cpc; return H->my0;
    case CHS_MZ_RHS0: *n = H->n_ccp; return H->mz0;
    default: break;
  }
  if (!H->thermo) throw std::invalid_argument("unknown field id, or a thermal field without chs_thermo_init");
  switch (field) {
    case CHS_GX: *n = H->n_pcc; return H->gx;
    case CHS_GY: *n = H->n_cpc; return H->gy;
    case CHS_GZ: *n = H->n_ccp; return H->gz;
    case CHS_RHOH: *n = H->n_ccc; return H->rhoh;
    case CHS_HENTH: *n = H->n_ccc; return H->hEnth;
    case CHS_TTEMP: *n = H->n_ccc; return H->tTemp;
    case CHS_KCOND: *n = H->n_ccc; return H->kCond;
    case CHS_DDENS: *n = H->n_ccc; return H->dDens;
    case CHS_MVISC: *n = H->n_ccc; return H->mVisc;
    case CHS_ENE_RHS0: *n = H->n_ccc; return H->erhs0;
    default: throw std::invalid_argument("unknown field id");
  }
}

// host (double) -> device field, converting to float in the mixed form (stream-ordered)
// host <-> device copy of one field on stream st; the mixed form converts through an FP64
// staging buffer (one per stream that copies concurrently)
void h2d_field(chs_handle* H, double* dev, const double* host, size_t n, cudaStream_t st = nullptr,
               double* stage = nullptr) {
  if (!st) st = H->st;
  if (!stage) stage = H->stage;
  if (!H->mixed) {
    CK(cudaMemcpyAsync(dev, host, n * sizeof(double), cudaMemcpyHostToDevice, st));
    return;
  }
  CK(cudaMemcpyAsync(stage, host, n * sizeof(double), cudaMemcpyHostToDevice, st));
  launch_convert(reinterpret_cast<float*>(dev), stage, (int64_t)n, st);
  H->launches++;
}
void d2h_field(chs_handle* H, double* host, const double* dev, size_t n, cudaStream_t st = nullptr,
               double* stage = nullptr) {
  if (!st) st = H->st;
  if (!stage) stage = H->stage;
  if (!H->mixed) {
    CK(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    return;
  }
  launch_convert(stage, reinterpret_cast<const float*>(dev), (int64_t)n, st);
  H->launches++;
  CK(cudaMemcpyAsync(host, stage, n * sizeof(double), cudaMemcpyDeviceToHost, st));
}

// ---- restart files and running statistics (src/io_restart.f90:32-227, src/post_statistics.f90:152-300)
const char* const kStatKey[12] = {"time_averaged_pr", "time_averaged_ux", "time_averaged_uy", "time_averaged_uz",
                                  "time_averaged_uu", "time_averaged_vv", "time_averaged_ww", "time_averaged_uv",
                                  "time_averaged_uw", "time_averaged_vw", "time_averaged_t",  "time_averaged_tt"};

// generate_pathfile_name (src/io_tools.f90:44-61): <dir>/domain<idom>_<keyword>_<iter>.bin
std::string data_file(const char* dir, int idom, const char* key, int iter) {
  return std::string(dir) + "/domain" + std::to_string(idom) + "_" + key + "_" + std::to_string(iter) + ".bin";
}

// decomp_2d_write_one / _read_one of a full-domain x-pencil array on one rank: the raw FP64 values
// in Fortran order (x fastest), no header
void write_raw(const std::string& path, const double* a, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot open " + path + " for writing");
  const size_t w = std::fwrite(a, sizeof(double), n, f);
  const int rc = std::fclose(f);
  if (w != n || rc != 0) throw std::runtime_error("short write to " + path);
}
void read_raw(const std::string& path, double* a, size_t n) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + path);
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz != (long)(n * sizeof(double))) {
    std::fclose(f);
    throw std::runtime_error(path + ": " + std::to_string(sz) + " bytes, expected " + std::to_string(n * sizeof(double)));
  }
  const size_t r = std::fread(a, sizeof(double), n, f);
  std::fclose(f);
  if (r != n) throw std::runtime_error("short read from " + path);
}

void save_field(chs_handle* H, int field, const std::string& path) {
  size_t n = 0;
  double* d = field_ptr(H, field, &n);
  std::vector<double> h(n);
  d2h_field(H, h.data(), d, n);
  CK(cudaStreamSynchronize(H->st));
  write_raw(path, h.data(), n);
}
void load_field(chs_handle* H, int field, const std::string& path) {
  size_t n = 0;
  double* d = field_ptr(H, field, &n);
  std::vector<double> h(n);
  read_raw(path, h.data(), n);
  h2d_field(H, d, h.data(), n);
  CK(cudaStreamSynchronize(H->st));  // the host copy is released on return
}

// Update_thermal_properties (src/eq_energy.f90:14-146) from the current rho*h, wall states
// included, then g = q * rho_face (convert_primary_conservative IQ2G): the thermal part of
// restore_thermo_variables_from_restart (src/io_restart.f90:208-226)
template <typename T>
void thermo_refresh_t(chs_handle* H) {
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const int nc0 = H->nc[0], nc2 = H->nc[2], np1 = H->np[1];
  const int s_ccc[3] = {H->nc[0], H->nc[1], H->nc[2]};
  launch_property_update<T>(H->tab, A(H->rhoh), A(H->hEnth), A(H->tTemp), A(H->kCond), A(H->dDens), A(H->mVisc),
                            (int64_t)H->n_ccc, H->st);
  H->launches++;
  const auto& B = H->ibc;
  const int s0 = B[1][V_TM][0] == BC_NEUMANN, s1 = B[1][V_TM][1] == BC_NEUMANN;
  if (s0 || s1) {
    run_op(H, 1, M1C2P, H->ftpy, nullptr, src(A(H->rhoh)), s_ccc, A(H->dh_cpc), false, 1.0);
    launch_wall_props<T>(H->tab, A(H->dh_cpc), nc0, np1, nc2, s0, s1, A(H->fb_h), A(H->fb_k), A(H->fb_m), A(H->fb_d),
                         H->st);
    H->launches++;
  }
  const Pair per = P2(kPer2);
  const T* any = A(H->fb_maxp);
  run_op(H, 0, M1C2P, per, any, src(A(H->dDens)), s_ccc, A(H->gx), false, 1.0, O_MUL, A(H->qx));
  run_op(H, 1, M1C2P, H->ftpy, A(H->fb_d), src(A(H->dDens)), s_ccc, A(H->gy), false, 1.0, O_MUL, A(H->qy));
  run_op(H, 2, M1C2P, per, any, src(A(H->dDens)), s_ccc, A(H->gz), false, 1.0, O_MUL, A(H->qz));
}

// update_statistics_flow / _thermo (src/post_statistics.f90:152-283) for sample nstat
template <typename T>
void stats_update_t(chs_handle* H, int nstat) {
  auto A = [](double* p) { return reinterpret_cast<T*>(p); };
  const int nst = H->thermo ? 12 : 10;
  for (int k = 0; k < nst; ++k)
    if (!H->stat[k]) H->stat[k] = H->dalloc<double>(H->n_ccc);
  const auto& B = H->ibc;
  const int s_pcc[3] = {H->np[0], H->nc[1], H->nc[2]}, s_cpc[3] = {H->nc[0], H->np[1], H->nc[2]};
  const int s_ccp[3] = {H->nc[0], H->nc[1], H->np[2]};
  const T* any = A(H->fb_maxp);
  const T* fyqy = H->periodic_y ? nullptr : A(H->fb_qy);
  // cell-centre velocities: the P2C mid-point interpolations of the reference (the derived-quantity
  // buffers serve as scratch between steps)
  run_op(H, 0, M1P2C, P2(B[0][V_QX]), any, src(A(H->qx)), s_pcc, A(H->qxix), false, 1.0);
  run_op(H, 1, M1P2C, P2(B[1][V_QY]), fyqy, src(A(H->qy)), s_cpc, A(H->qyiy), false, 1.0);
  run_op(H, 2, M1P2C, P2(B[2][V_QZ]), any, src(A(H->qz)), s_ccp, A(H->qziz), false, 1.0);
  StatsIO<T> io{};
  io.p = A(H->pres);
  io.u[0] = A(H->qxix);
  io.u[1] = A(H->qyiy);
  io.u[2] = A(H->qziz);
  io.t = H->thermo ? A(H->tTemp) : nullptr;
  io.pm = H->stat[0];
  for (int k = 0; k < 3; ++k) io.um[k] = H->stat[1 + k];
  for (int k = 0; k < 6; ++k) io.uu[k] = H->stat[4 + k];
  io.tm = H->stat[10];
  io.ttm = H->stat[11];
  io.ac = 1.0 / (double)nstat;
  io.am = (double)(nstat - 1) / (double)nstat;
  io.n = (int64_t)H->n_ccc;
  launch_stats_update<T>(io, H->st);
  H->launches++;
}

// capture substep isub (parts PART_*) as one graph; returns its kernel count
long long capture_one(chs_handle* H, int isub, int parts, cudaGraphExec_t* out) {
  cudaGraph_t g;
  const long long before = H->launches;
  CK(cudaStreamBeginCapture(H->st, cudaStreamCaptureModeThreadLocal));
  H->capturing = true;
  try {
    H->dag_start();
    substep_body(H, isub, parts);
    H->dag_stop();
  } catch (...) {
    H->dag_stop();
    H->capturing = false;
    cudaStreamEndCapture(H->st, &g);
    throw;
  }
  H->capturing = false;
  CK(cudaStreamEndCapture(H->st, &g));
  const long long n = H->launches - before;
  H->launches = before;
  CK(cudaGraphInstantiate(out, g, 0));
  CK(cudaGraphDestroy(g));
  return n;
}

void capture_graphs(chs_handle* H) {
  for (int isub = 1; isub <= 3; ++isub) H->kernels_per_sub[isub] = capture_one(H, isub, PART_ALL, &H->gexec[isub]);
}

void capture_part_graphs(chs_handle* H) {
  for (int isub = 1; isub <= 3; ++isub) {
    H->kernels_per_part[0][isub] = capture_one(H, isub, PART_ENERGY, &H->gpart[0][isub]);
    H->kernels_per_part[1][isub] = capture_one(H, isub, PART_MOMENTUM, &H->gpart[1][isub]);
  }
}

}  // namespace

// Batched ensemble of independent handles: one captured graph per RK3 substep whose branches
// (one per member, on the member's stream) run concurrently, so one graph launch advances every
// member.  The members stay owned by the caller.
struct chs_ensemble {
  std::vector<chs_handle*> m;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t g[4] = {nullptr, nullptr, nullptr, nullptr};
  long long kps[4] = {0, 0, 0, 0};
  long long launches = 0;
  std::string err;
};

namespace {

void ensemble_capture(chs_ensemble* E) {
  for (int isub = 1; isub <= 3; ++isub) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(E->st, cudaStreamCaptureModeThreadLocal));
    long long kernels = 0;
    try {
      CK(cudaEventRecord(E->fork, E->st));
      for (size_t i = 0; i < E->m.size(); ++i) {
        chs_handle* H = E->m[i];
        CK(cudaStreamWaitEvent(H->st, E->fork, 0));
        const long long before = H->launches;
        H->capturing = true;
        substep_body(H, isub);
        H->capturing = false;
        kernels += H->launches - before;
        H->launches = before;
        CK(cudaEventRecord(E->join[i], H->st));
        CK(cudaStreamWaitEvent(E->st, E->join[i], 0));
      }
    } catch (...) {
      for (chs_handle* H : E->m) H->capturing = false;
      cudaStreamEndCapture(E->st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(E->st, &g));
    CK(cudaGraphInstantiate(&E->g[isub], g, 0));
    CK(cudaGraphDestroy(g));
    E->kps[isub] = kernels;
  }
}

// order the ensemble stream after each member's pending work, run, then order the members after it
void ensemble_run(chs_ensemble* E, int nsteps) {
  for (size_t i = 0; i < E->m.size(); ++i) {
    CK(cudaEventRecord(E->join[i], E->m[i]->st));
    CK(cudaStreamWaitEvent(E->st, E->join[i], 0));
  }
  for (int s = 0; s < nsteps; ++s)
    for (int isub = 1; isub <= 3; ++isub) {
      CK(cudaGraphLaunch(E->g[isub], E->st));
      E->launches += E->kps[isub];
    }
  CK(cudaEventRecord(E->done, E->st));
  for (chs_handle* H : E->m) CK(cudaStreamWaitEvent(H->st, E->done, 0));
}

int eguard(chs_ensemble* E, const std::function<void()>& f) {
  try {
    f();
    return CHS_OK;
  } catch (const CudaError& e) {
    E->err = e.what();
    return CHS_ERR_CUDA;
  } catch (const std::exception& e) {
    E->err = e.what();
    return CHS_ERR_ARG;
  }
}

// copy every device allocation of the handle into one buffer (or back), for trial runs
void snapshot(chs_handle* H, char* buf, bool save) {
  size_t off = 0;
  for (auto& a : H->allocs) {
    if (save) CK(cudaMemcpyAsync(buf + off, a.first, a.second, cudaMemcpyDeviceToDevice, H->st));
    else CK(cudaMemcpyAsync(a.first, buf + off, a.second, cudaMemcpyDeviceToDevice, H->st));
    off += a.second;
  }
}

float time_steps_ms(chs_handle* H, int nsteps) {
  if (!H->gexec[1]) capture_graphs(H);
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a, H->st));
  for (int s = 0; s < nsteps; ++s)
    for (int isub = 1; isub <= 3; ++isub) CK(cudaGraphLaunch(H->gexec[isub], H->st));
  CK(cudaEventRecord(b, H->st));
  CK(cudaEventSynchronize(b));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms;
}

}  // namespace

extern "C" {

int chs_autotune(chs_handle* H, int nsteps, int* block, int* lt_max, int* fused, float* best_ms) {
  if (!H || !block || !lt_max || !fused || !best_ms || nsteps < 1) return CHS_ERR_ARG;
  return guard(H, [&] {
    size_t total = 0;
    for (auto& a : H->allocs) total += a.second;
    char* snap = nullptr;
    CK(cudaMalloc(&snap, total));
    snapshot(H, snap, true);
    // 0: the specialised explicit-operator kernels; 128/256/512: the generic kernel's CTA size
    const int blocks[4] = {0, 128, 256, 512};
    const bool compact = H->iacc >= 3;
    const int lts[3] = {16, 32, 64};
    int bb = 0, bl = 64, bf = 0;
    float best = 1e30f;
    try {
      for (int fu = 0; fu <= 1; ++fu)
        for (int b : blocks)
          for (int l : lts) {
            if (!compact && l != 64) continue;
            H->tune_block = b;
            H->tune_lt = l;
            H->tune_fuse = fu;
            drop_graphs(H);
            time_steps_ms(H, 1);  // capture and warm up
            const float ms = time_steps_ms(H, nsteps);
            snapshot(H, snap, false);
            if (ms < best) { best = ms; bb = b; bl = l; bf = fu; }
          }
    } catch (...) {
      snapshot(H, snap, false);
      cudaStreamSynchronize(H->st);
      cudaFree(snap);
      throw;
    }
    CK(cudaStreamSynchronize(H->st));
    cudaFree(snap);
    H->tune_block = bb;
    H->tune_lt = bl;
    H->tune_fuse = bf;
    drop_graphs(H);
    *block = bb;
    *lt_max = bl;
    *fused = bf;
    *best_ms = best;
  });
}

int chs_set_launch_shape(chs_handle* H, int block, int lt_max, int fused) {
  if (!H || (block != 0 && block != 128 && block != 256 && block != 512) ||
      (lt_max != 0 && lt_max != 16 && lt_max != 32 && lt_max != 64) || (fused != 0 && fused != 1))
    return CHS_ERR_ARG;
  return guard(H, [&] {
    H->tune_block = block;
    H->tune_lt = lt_max;
    H->tune_fuse = fused;
    drop_graphs(H);
  });
}

int chs_set_fusion(chs_handle* H, int on) {
  if (!H || on < 0 || on > 1) return CHS_ERR_ARG;
  return guard(H, [&] {
    H->kfuse = on;
    drop_graphs(H);
  });
}

int chs_set_lanes(chs_handle* H, int lanes) {
  if (!H || lanes < 1 || lanes > chs_handle::kLanes) return CHS_ERR_ARG;
  return guard(H, [&] {
    H->dag_lanes = lanes;
    drop_graphs(H);
  });
}

int chs_ensemble_create(chs_handle* const* members, int n, chs_ensemble** out) {
  if (!members || n < 1 || !out) return CHS_ERR_ARG;
  auto* E = new chs_ensemble();
  const int rc = eguard(E, [&] {
    int dev0 = -1;
    for (int i = 0; i < n; ++i) {
      if (!members[i]) throw std::invalid_argument("null member");
      if (dev0 < 0) dev0 = members[i]->device;
      if (members[i]->device != dev0) throw std::invalid_argument("ensemble members must share one device");
      E->m.push_back(members[i]);
    }
    CK(cudaSetDevice(dev0));
    CK(cudaStreamCreateWithFlags(&E->st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&E->fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&E->done, cudaEventDisableTiming));
    E->join.resize(n);
    for (auto& e : E->join) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (chs_handle* H : E->m) CK(cudaStreamSynchronize(H->st));
    ensemble_capture(E);
  });
  if (rc != CHS_OK) {
    std::fprintf(stderr, "chs_ensemble_create: %s\n", E->err.c_str());
    chs_ensemble_destroy(E);
    *out = nullptr;
    return rc;
  }
  *out = E;
  return CHS_OK;
}

int chs_ensemble_step(chs_ensemble* E, int nsteps) {
  if (!E || nsteps < 0) return CHS_ERR_ARG;
  return eguard(E, [&] {
    ensemble_run(E, nsteps);
    CK(cudaGetLastError());
  });
}

int chs_ensemble_time_steps(chs_ensemble* E, int nsteps, float* ms) {
  if (!E || !ms || nsteps < 0) return CHS_ERR_ARG;
  return eguard(E, [&] {
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    for (size_t i = 0; i < E->m.size(); ++i) {
      CK(cudaEventRecord(E->join[i], E->m[i]->st));
      CK(cudaStreamWaitEvent(E->st, E->join[i], 0));
    }
    CK(cudaEventRecord(a, E->st));
    ensemble_run(E, nsteps);
    CK(cudaEventRecord(b, E->st));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

long long chs_ensemble_kernel_launches(const chs_ensemble* E) { return E ? E->launches : 0; }

int chs_ensemble_destroy(chs_ensemble* E) {
  if (!E) return CHS_OK;
  if (E->st) cudaStreamSynchronize(E->st);
  for (auto& g : E->g)
    if (g) cudaGraphExecDestroy(g);
  for (auto& e : E->join)
    if (e) cudaEventDestroy(e);
  if (E->fork) cudaEventDestroy(E->fork);
  if (E->done) cudaEventDestroy(E->done);
  if (E->st) cudaStreamDestroy(E->st);
  delete E;
  return CHS_OK;
}

int chs_create(const chs_config* cfg, int device, chs_handle** out) {
  if (!cfg || !out) return CHS_ERR_ARG;
  chs_handle* H = new chs_handle();
  int rc = guard(H, [&] {
    setup_host(H, cfg);  // validates the configuration before any device work
    if (device >= 0) CK(cudaSetDevice(device));
    CK(cudaGetDevice(&H->device));
    setup_device(H, cfg);
    prepare_plans(H);
    CK(cudaStreamSynchronize(H->st));
  });
  if (rc != CHS_OK) {
    std::fprintf(stderr, "chs_create: %s\n", H->err.c_str());
    chs_destroy(H);
    *out = nullptr;
    return rc;
  }
  *out = H;
  return CHS_OK;
}

int chs_destroy(chs_handle* H) {
  if (!H) return CHS_OK;
  if (H->st) cudaStreamSynchronize(H->st);
  drop_graphs(H);
  if (H->table) cudaFree(H->table);
  if (H->fz_rows) cudaFree(H->fz_rows);
  for (auto& a : H->allocs) cudaFree(a.first);
  for (int l = 1; l < chs_handle::kLanes; ++l)
    if (H->lane[l]) cudaStreamDestroy(H->lane[l]);
  for (cudaEvent_t e : H->evpool) cudaEventDestroy(e);
  if (H->st) cudaStreamDestroy(H->st);
  delete H;
  return CHS_OK;
}

int chs_upload_field(chs_handle* H, int field, const double* host, size_t n) {
  if (!H || !host) return CHS_ERR_ARG;
  return guard(H, [&] {
    size_t m;
    double* d = field_ptr(H, field, &m);
    if (n != m) throw std::invalid_argument("field size mismatch");
    h2d_field(H, d, host, n);
    CK(cudaStreamSynchronize(H->st));
  });
}

int chs_download_field(chs_handle* H, int field, double* host, size_t n) {
  if (!H || !host) return CHS_ERR_ARG;
  return guard(H, [&] {
    size_t m;
    double* d = field_ptr(H, field, &m);
    if (n != m) throw std::invalid_argument("field size mismatch");
    d2h_field(H, host, d, n);
    CK(cudaStreamSynchronize(H->st));
  });
}

int chs_thermo_init(chs_handle* H, const chs_thermo* th) {
  if (!H || !th) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (H->thermo) throw std::invalid_argument("chs_thermo_init was already called");
    thermo_init(H, th);
  });
}

int chs_mlp_train(chs_handle* H, const chs_mlp_train_cfg* cfg, chs_mlp_report* rep) {
  if (!H || !cfg || !rep) return CHS_ERR_ARG;
  return guard(H, [&] { mlp_train(H, cfg, rep); });
}

int chs_mlp_set_mode(chs_handle* H, int mode, double tol) {
  if (!H || mode < 0 || mode > 1) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (mode == 1 && !H->mlp_ready) throw std::invalid_argument("the MLP surrogate is not trained");
    if (tol > 0.0 && tol != H->mlp_check.tol) {
      set_mlp_tol(H->mlp_check, tol, H->tab.n);
      drop_graphs(H);  // the captured launches hold the check by value
    }
    if (mode != H->mlp_mode) drop_graphs(H);
    H->mlp_mode = mode;
    if (H->mlp_nfb) CK(cudaMemsetAsync(H->mlp_nfb, 0, sizeof(unsigned long long), H->st));
  });
}

int chs_mlp_fallbacks(chs_handle* H, unsigned long long* count) {
  if (!H || !count) return CHS_ERR_ARG;
  return guard(H, [&] {
    *count = 0;
    if (H->mlp_nfb) {
      CK(cudaMemcpyAsync(count, H->mlp_nfb, sizeof(unsigned long long), cudaMemcpyDeviceToHost, H->st));
      CK(cudaStreamSynchronize(H->st));
    }
  });
}

int chs_mlp_params(chs_handle* H, float* buf, int n, int set) {
  if (!H || !buf || n != MLP_NPARAM) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (set) {
      mlp_alloc_core(H);
      CK(cudaMemcpyAsync(H->mlp_params, buf, n * sizeof(float), cudaMemcpyHostToDevice, H->st));
      mlp_finalize(H);
      drop_graphs(H);
    } else {
      if (!H->mlp_params) throw std::invalid_argument("no MLP parameters");
      CK(cudaMemcpyAsync(buf, H->mlp_params, n * sizeof(float), cudaMemcpyDeviceToHost, H->st));
      CK(cudaStreamSynchronize(H->st));
    }
  });
}

int chs_mlp_grad(chs_handle* H, const float* params, int B, const float* x, const float* t, float* grad,
                 float* loss) {
  if (!H || !params || !x || !t || !grad || !loss || B < 1 || B > 65536) return CHS_ERR_ARG;
  return guard(H, [&] {
    cudaStream_t st = H->st;
    float* d = nullptr;
    const size_t need = (size_t)2 * MLP_NPARAM + B + (size_t)4 * B + (size_t)8 * B * MLP_H + 1;
    CK(cudaMallocAsync(&d, need * sizeof(float), st));
    float *P = d, *G = d + MLP_NPARAM, *X = G + MLP_NPARAM, *Tt = X + B, *W = Tt + (size_t)4 * B;
    float* L = W + (size_t)8 * B * MLP_H;
    CK(cudaMemcpyAsync(P, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(X, x, (size_t)B * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(Tt, t, (size_t)4 * B * sizeof(float), cudaMemcpyHostToDevice, st));
    mlp_grad(P, X, Tt, B, G, L, W, st);
    H->launches += 13;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(grad, G, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(loss, L, sizeof(float), cudaMemcpyDeviceToHost, st));
    CK(cudaFreeAsync(d, st));
    CK(cudaStreamSynchronize(st));
  });
}

int chs_mlp_eval(chs_handle* H, int n, const double* rhoh, double tol, double* out, unsigned long long* nfallback) {
  if (!H || n < 1 || !rhoh || !out || !nfallback) return CHS_ERR_ARG;
  return guard(H, [&] { mlp_eval(H, n, rhoh, tol, out, nfallback); });
}

int chs_mlp_norm(const chs_handle* H, double* out) {
  if (!H || !out || !H->thermo) return CHS_ERR_ARG;
  out[0] = H->mlp_norm.xa;
  out[1] = H->mlp_norm.xb;
  for (int j = 0; j < MLP_NOUT; ++j) {
    out[2 + j] = H->mlp_norm.ya[j];
    out[6 + j] = H->mlp_norm.yb[j];
  }
  return CHS_OK;
}

int chs_energy_substep(chs_handle* H, int isub) {
  if (!H) return CHS_ERR_ARG;
  if (isub < 1 || isub > 3) { set_err(H, "isub must be 1..3"); return CHS_ERR_ARG; }
  return guard(H, [&] {
    if (!H->thermo) throw std::invalid_argument("chs_energy_substep needs chs_thermo_init");
    substep_body(H, isub, PART_ENERGY);
    CK(cudaGetLastError());
  });
}

int chs_momentum_substep(chs_handle* H, int isub) {
  if (!H) return CHS_ERR_ARG;
  if (isub < 0 || isub > 3) { set_err(H, "isub must be 0..3"); return CHS_ERR_ARG; }
  return guard(H, [&] {
    if (H->thermo) {
      // the captured graphs hold the whole substep (energy + momentum)
      substep_body(H, isub, PART_MOMENTUM);
    } else if (isub >= 1 && H->gexec[isub]) {
      CK(cudaGraphLaunch(H->gexec[isub], H->st));
      H->launches += H->kernels_per_sub[isub];
    } else {
      substep_body(H, isub);
    }
    CK(cudaGetLastError());
  });
}

int chs_step(chs_handle* H, int nsteps) {
  if (!H) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (!H->gexec[1]) capture_graphs(H);
    for (int s = 0; s < nsteps; ++s)
      for (int isub = 1; isub <= 3; ++isub) {
        CK(cudaGraphLaunch(H->gexec[isub], H->st));
        H->launches += H->kernels_per_sub[isub];
      }
    CK(cudaGetLastError());
  });
}

int chs_momentum_substep_host(chs_handle* H, int isub, double* qx, double* qy, double* qz, double* pres) {
  if (!H || !qx || !qy || !qz || !pres) return CHS_ERR_ARG;
  if (isub < 0 || isub > 3) { set_err(H, "isub must be 0..3"); return CHS_ERR_ARG; }
  if (H->thermo) {
    set_err(H, "variable-property runs keep g and the thermal fields on the device: use chs_upload_field/"
               "chs_download_field around chs_energy_substep and chs_momentum_substep");
    return CHS_ERR_STATE;
  }
  return guard(H, [&] {
    h2d_field(H, H->qx, qx, H->n_pcc);
    h2d_field(H, H->qy, qy, H->n_cpc);
    h2d_field(H, H->qz, qz, H->n_ccp);
    h2d_field(H, H->pres, pres, H->n_ccc);
    if (isub >= 1) {
      if (!H->gexec[1]) capture_graphs(H);
      CK(cudaGraphLaunch(H->gexec[isub], H->st));
      H->launches += H->kernels_per_sub[isub];
    } else {
      substep_body(H, isub);
    }
    d2h_field(H, qx, H->qx, H->n_pcc);
    d2h_field(H, qy, H->qy, H->n_cpc);
    d2h_field(H, qz, H->qz, H->n_ccp);
    d2h_field(H, pres, H->pres, H->n_ccc);
    CK(cudaStreamSynchronize(H->st));
  });
}

int chs_time_steps(chs_handle* H, int nsteps, float* ms) {
  if (!H || !ms || nsteps < 0) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (!H->gexec[1]) capture_graphs(H);
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, H->st));
    for (int s = 0; s < nsteps; ++s)
      for (int isub = 1; isub <= 3; ++isub) {
        CK(cudaGraphLaunch(H->gexec[isub], H->st));
        H->launches += H->kernels_per_sub[isub];
      }
    CK(cudaEventRecord(b, H->st));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

int chs_time_steps_host(chs_handle* H, int nsteps, double* qx, double* qy, double* qz, double* pres, float* ms) {
  if (!H || !ms || !qx || !qy || !qz || !pres || nsteps < 0) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (!H->gexec[1]) capture_graphs(H);
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaEventRecord(a, H->st));
    for (int s = 0; s < nsteps; ++s)
      for (int isub = 1; isub <= 3; ++isub) {
        h2d_field(H, H->qx, qx, H->n_pcc);
        h2d_field(H, H->qy, qy, H->n_cpc);
        h2d_field(H, H->qz, qz, H->n_ccp);
        h2d_field(H, H->pres, pres, H->n_ccc);
        CK(cudaGraphLaunch(H->gexec[isub], H->st));
        H->launches += H->kernels_per_sub[isub];
        d2h_field(H, qx, H->qx, H->n_pcc);
        d2h_field(H, qy, H->qy, H->n_cpc);
        d2h_field(H, qz, H->qz, H->n_ccp);
        d2h_field(H, pres, H->pres, H->n_ccc);
      }
    CK(cudaEventRecord(b, H->st));
    CK(cudaEventSynchronize(b));
    CK(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  });
}

// nsteps RK3 steps on host-owned fields, copied in and out around every substep (per_substep) or
// around every RK3 step
static int time_host_fields(chs_handle* H, int nsteps, int nfields, const int* ids, double* const* bufs, float* ms,
                            bool per_substep) {
  if (!H || !ms || nsteps < 0 || nfields < 0 || (nfields > 0 && (!ids || !bufs))) return CHS_ERR_ARG;
  return guard(H, [&] {
    std::vector<double*> dev(nfields);
    std::vector<size_t> cnt(nfields);
    for (int f = 0; f < nfields; ++f) {
      if (!bufs[f]) throw std::invalid_argument("null host buffer");
      dev[f] = field_ptr(H, ids[f], &cnt[f]);
    }
    // Copies in and out of every substep on two copy streams, one per PCIe direction, ordered
    // per field: the copy-in of a field for substep k+1 waits only for that field's copy-out of
    // substep k (it reads the host array that copy wrote), so copy-out and copy-in of different
    // fields run at the same time.  With variable properties the substep runs as two graphs,
    // energy then momentum: the energy graph waits only for the fields it reads (g and the
    // thermal fields) while the rest are still coming in, and the fields final after it (rho*h,
    // h, T, kappa, the energy rhs) go out while the momentum graph runs.  Every copy-out waits
    // for the graph after which its field is final; rho and mu, which the momentum graph reads,
    // go out after it.
    const bool split = H->thermo;
    if (split) {
      if (!H->gpart[0][1]) capture_part_graphs(H);
    } else if (!H->gexec[1]) {
      capture_graphs(H);
    }
    auto energy_reads = [](int id) {
      return id == CHS_GX || id == CHS_GY || id == CHS_GZ || id == CHS_RHOH || id == CHS_HENTH || id == CHS_TTEMP ||
             id == CHS_KCOND || id == CHS_DDENS || id == CHS_MVISC || id == CHS_ENE_RHS0;
    };
    auto final_after_energy = [](int id) {
      return id == CHS_RHOH || id == CHS_HENTH || id == CHS_TTEMP || id == CHS_KCOND || id == CHS_ENE_RHS0;
    };
    const int nph = split ? 2 : 1;
    std::vector<int> in_ph(nfields), out_ph(nfields);
    for (int f = 0; f < nfields; ++f) {
      in_ph[f] = (split && !energy_reads(ids[f])) ? 1 : 0;
      out_ph[f] = (split && !final_after_energy(ids[f])) ? 1 : 0;
    }
    cudaStream_t sin = nullptr, sout = nullptr;
    CK(cudaStreamCreateWithFlags(&sin, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&sout, cudaStreamNonBlocking));
    std::vector<cudaEvent_t> out_done(nfields, nullptr);
    cudaEvent_t a = nullptr, b = nullptr, in_done[2] = {nullptr, nullptr}, graph_done[2] = {nullptr, nullptr};
    double* stage_out = nullptr;
    auto cleanup = [&] {
      for (auto& e : out_done)
        if (e) cudaEventDestroy(e);
      for (cudaEvent_t e : {a, b, in_done[0], in_done[1], graph_done[0], graph_done[1]})
        if (e) cudaEventDestroy(e);
      if (stage_out) cudaFree(stage_out);
      if (sin) cudaStreamDestroy(sin);
      if (sout) cudaStreamDestroy(sout);
    };
    try {
      for (auto& e : out_done) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      for (int p = 0; p < 2; ++p) {
        CK(cudaEventCreateWithFlags(&in_done[p], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&graph_done[p], cudaEventDisableTiming));
      }
      CK(cudaEventCreate(&a));
      CK(cudaEventCreate(&b));
      if (H->mixed) {
        size_t m = 0;
        for (size_t c : cnt) m = std::max(m, c);
        CK(cudaMalloc(&stage_out, std::max<size_t>(m, 1) * sizeof(double)));
      }
      CK(cudaEventRecord(a, H->st));
      CK(cudaStreamWaitEvent(sin, a, 0));
      bool first = true;
      for (int s = 0; s < nsteps; ++s)
        for (int isub = 1; isub <= 3; ++isub) {
          const bool cin = per_substep || isub == 1, cout = per_substep || isub == 3;
          for (int p = 0; p < nph && cin; ++p) {
            for (int f = 0; f < nfields; ++f) {
              if (in_ph[f] != p) continue;
              if (!first) CK(cudaStreamWaitEvent(sin, out_done[f], 0));
              h2d_field(H, dev[f], bufs[f], cnt[f], sin, H->stage);
            }
            CK(cudaEventRecord(in_done[p], sin));
          }
          first = false;
          for (int p = 0; p < nph; ++p) {
            if (cin) CK(cudaStreamWaitEvent(H->st, in_done[p], 0));
            CK(cudaGraphLaunch(split ? H->gpart[p][isub] : H->gexec[isub], H->st));
            H->launches += split ? H->kernels_per_part[p][isub] : H->kernels_per_sub[isub];
            CK(cudaEventRecord(graph_done[p], H->st));
          }
          for (int p = 0; p < nph && cout; ++p) {
            CK(cudaStreamWaitEvent(sout, graph_done[p], 0));
            // the fields the next substep copies in first go out first
            for (int q = 0; q < nph; ++q)
              for (int f = 0; f < nfields; ++f) {
                if (out_ph[f] != p || in_ph[f] != q) continue;
                d2h_field(H, bufs[f], dev[f], cnt[f], sout, stage_out);
                CK(cudaEventRecord(out_done[f], sout));
              }
          }
        }
      // the timed region ends when the last copy-out has landed
      CK(cudaEventRecord(graph_done[0], sout));
      CK(cudaStreamWaitEvent(H->st, graph_done[0], 0));
      CK(cudaEventRecord(b, H->st));
      CK(cudaEventSynchronize(b));
      CK(cudaEventElapsedTime(ms, a, b));
    } catch (...) {
      cudaStreamSynchronize(sin);
      cudaStreamSynchronize(sout);
      cudaStreamSynchronize(H->st);
      cleanup();
      throw;
    }
    cleanup();
  });
}

int chs_time_steps_host_fields(chs_handle* H, int nsteps, int nfields, const int* ids, double* const* bufs,
                               float* ms) {
  return time_host_fields(H, nsteps, nfields, ids, bufs, ms, true);
}

int chs_time_rk3_host_fields(chs_handle* H, int nsteps, int nfields, const int* ids, double* const* bufs,
                             float* ms) {
  return time_host_fields(H, nsteps, nfields, ids, bufs, ms, false);
}

void* chs_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
  return p;
}

void chs_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

int chs_profile_substep(chs_handle* H, int isub, chs_kprof* out, int max, int* n) {
  if (!H || !out || !n || isub < 0 || isub > 3) return CHS_ERR_ARG;
  return guard(H, [&] {
    H->recs.clear();
    H->profiling = true;
    try {
      substep_body(H, isub);
    } catch (...) {
      H->profiling = false;
      throw;
    }
    H->profiling = false;
    CK(cudaStreamSynchronize(H->st));
    int k = 0;
    for (auto& r : H->recs) {
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, r.e0, r.e1));
      if (k < max) out[k] = chs_kprof{r.kind, r.dir, r.bytes, ms};
      ++k;
      cudaEventDestroy(r.e0);
      cudaEventDestroy(r.e1);
    }
    H->recs.clear();
    *n = k;
  });
}

int chs_profile_class(chs_handle* H, int isub, int kind, int reps, float* ms) {
  if (!H || !ms || isub < 1 || isub > 3 || kind < -1 || kind > 4 || reps < 1) return CHS_ERR_ARG;
  return guard(H, [&] {
    // the partial substep leaves the state inconsistent: save it and put it back afterwards
    size_t tot = 0;
    for (const auto& a : H->allocs) tot += a.second;
    char* buf = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void**>(&buf), tot, H->st));
    snapshot(H, buf, true);
    cudaGraphExec_t ge = nullptr;
    H->only_kind = kind;
    try {
      capture_one(H, isub, PART_ALL, &ge);
    } catch (...) {
      H->only_kind = -1;
      throw;
    }
    H->only_kind = -1;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    CK(cudaGraphLaunch(ge, H->st));  // warm-up
    CK(cudaEventRecord(a, H->st));
    for (int r = 0; r < reps; ++r) CK(cudaGraphLaunch(ge, H->st));
    CK(cudaEventRecord(b, H->st));
    CK(cudaEventSynchronize(b));
    float t = 0.0f;
    CK(cudaEventElapsedTime(&t, a, b));
    *ms = t / reps;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaGraphExecDestroy(ge);
    snapshot(H, buf, false);
    CK(cudaFreeAsync(buf, H->st));
    CK(cudaStreamSynchronize(H->st));
  });
}

int chs_profile_substep_graph(chs_handle* H, int isub, chs_kprof* out, int max, int* n) {
  if (!H || !out || !n || isub < 1 || isub > 3) return CHS_ERR_ARG;
  return guard(H, [&] {
    for (auto& r : H->recs) { cudaEventDestroy(r.e0); cudaEventDestroy(r.e1); }
    H->recs.clear();
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamSynchronize(H->st));
    CK(cudaStreamBeginCapture(H->st, cudaStreamCaptureModeThreadLocal));
    H->capturing = true;
    H->profiling = true;
    const long long before = H->launches;
    try {
      substep_body(H, isub);
    } catch (...) {
      H->profiling = false;
      H->capturing = false;
      cudaStreamEndCapture(H->st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    H->profiling = false;
    H->capturing = false;
    CK(cudaStreamEndCapture(H->st, &g));
    const long long nk = H->launches - before;
    H->launches = before;
    const cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(ei);
    CK(cudaGraphUpload(ge, H->st));
    CK(cudaStreamSynchronize(H->st));
    CK(cudaGraphLaunch(ge, H->st));
    H->launches += nk;
    CK(cudaStreamSynchronize(H->st));
    cudaGraphExecDestroy(ge);
    int k = 0;
    for (auto& r : H->recs) {
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, r.e0, r.e1));
      if (k < max) out[k] = chs_kprof{r.kind, r.dir, r.bytes, ms};
      ++k;
      cudaEventDestroy(r.e0);
      cudaEventDestroy(r.e1);
    }
    H->recs.clear();
    *n = k;
  });
}

int chs_poisson_solve(chs_handle* H, double* rhs) {
  if (!H || !rhs) return CHS_ERR_ARG;
  return guard(H, [&] {
    // FP64 buffer: the correction field itself, or the staging array in the mixed form
    double* buf = H->mixed ? H->stage : H->pcor;
    CK(cudaMemcpyAsync(buf, rhs, H->n_ccc * sizeof(double), cudaMemcpyHostToDevice, H->st));
    poisson_device(H, buf);
    CK(cudaMemcpyAsync(rhs, buf, H->n_ccc * sizeof(double), cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
  });
}

int chs_poisson_solve_device(chs_handle* H, double* d_rhs) {
  if (!H || !d_rhs) return CHS_ERR_ARG;
  return guard(H, [&] {
    poisson_device(H, d_rhs);
    CK(cudaGetLastError());
  });
}

int chs_write_restart(chs_handle* H, const char* dir, int idom, int iter) {
  if (!H || !dir) return CHS_ERR_ARG;
  return guard(H, [&] {
    // write_instantanous_flow / _thermo (src/io_restart.f90:71-108)
    const int f[4] = {CHS_QX, CHS_QY, CHS_QZ, CHS_PRES};
    const char* k[4] = {"qx", "qy", "qz", "pr"};
    for (int i = 0; i < 4; ++i) save_field(H, f[i], data_file(dir, idom, k[i], iter));
    if (H->thermo) {
      save_field(H, CHS_RHOH, data_file(dir, idom, "rhoh", iter));
      save_field(H, CHS_TTEMP, data_file(dir, idom, "temp", iter));
    }
  });
}

int chs_read_restart(chs_handle* H, const char* dir, int idom, int iter) {
  if (!H || !dir) return CHS_ERR_ARG;
  return guard(H, [&] {
    // read_instantanous_flow (src/io_restart.f90:112-129), restore_flow_variables_from_restart
    // (:132-167: pcor = 0), read_instantanous_thermo (:170-204; T is recomputed from rho*h) and
    // restore_thermo_variables_from_restart (:208-226)
    const int f[4] = {CHS_QX, CHS_QY, CHS_QZ, CHS_PRES};
    const char* k[4] = {"qx", "qy", "qz", "pr"};
    for (int i = 0; i < 4; ++i) load_field(H, f[i], data_file(dir, idom, k[i], iter));
    if (H->mixed) launch_fill(reinterpret_cast<float*>(H->pcor), 0.0, (int64_t)H->n_ccc, H->st);
    else launch_fill(H->pcor, 0.0, (int64_t)H->n_ccc, H->st);
    H->launches++;
    if (H->thermo) {
      load_field(H, CHS_RHOH, data_file(dir, idom, "rhoh", iter));
      if (H->mixed) thermo_refresh_t<float>(H);
      else thermo_refresh_t<double>(H);
    }
    CK(cudaStreamSynchronize(H->st));
  });
}

int chs_stats_update(chs_handle* H, int nstat) {
  if (!H || nstat < 1) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (H->mixed) stats_update_t<float>(H, nstat);
    else stats_update_t<double>(H, nstat);
    CK(cudaGetLastError());
  });
}

int chs_stats_get(chs_handle* H, int which, double* host, size_t n) {
  if (!H || !host || which < 0 || which > 11) return CHS_ERR_ARG;
  return guard(H, [&] {
    if (!H->stat[which]) throw std::invalid_argument("no statistics of this kind yet (chs_stats_update)");
    if (n != H->n_ccc) throw std::invalid_argument("statistics size mismatch");
    CK(cudaMemcpyAsync(host, H->stat[which], n * sizeof(double), cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
  });
}

int chs_write_statistics(chs_handle* H, const char* dir, int idom, int iter) {
  if (!H || !dir) return CHS_ERR_ARG;
  return guard(H, [&] {
    // write_statistics_flow / _thermo (src/post_statistics.f90:217-239, :285-296)
    const int nst = H->thermo ? 12 : 10;
    std::vector<double> h(H->n_ccc);
    for (int k = 0; k < nst; ++k) {
      if (!H->stat[k]) throw std::invalid_argument("no statistics yet (chs_stats_update)");
      CK(cudaMemcpyAsync(h.data(), H->stat[k], H->n_ccc * sizeof(double), cudaMemcpyDeviceToHost, H->st));
      CK(cudaStreamSynchronize(H->st));
      write_raw(data_file(dir, idom, kStatKey[k], iter), h.data(), H->n_ccc);
    }
  });
}

int chs_read_statistics(chs_handle* H, const char* dir, int idom, int iter) {
  if (!H || !dir) return CHS_ERR_ARG;
  return guard(H, [&] {
    // read_statistics_flow / _thermo (src/post_statistics.f90:98-148)
    const int nst = H->thermo ? 12 : 10;
    std::vector<double> h(H->n_ccc);
    for (int k = 0; k < nst; ++k) {
      if (!H->stat[k]) H->stat[k] = H->dalloc<double>(H->n_ccc);
      read_raw(data_file(dir, idom, kStatKey[k], iter), h.data(), H->n_ccc);
      CK(cudaMemcpyAsync(H->stat[k], h.data(), H->n_ccc * sizeof(double), cudaMemcpyHostToDevice, H->st));
      CK(cudaStreamSynchronize(H->st));
    }
  });
}

int chs_data_file_name(const char* dir, int idom, const char* keyword, int iter, char* buf, size_t len) {
  if (!dir || !keyword || !buf || len == 0) return CHS_ERR_ARG;
  const std::string s = data_file(dir, idom, keyword, iter);
  if (s.size() + 1 > len) return CHS_ERR_ARG;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return CHS_OK;
}

int chs_diagnostics(chs_handle* H, chs_diag* out) {
  if (!H || !out) return CHS_ERR_ARG;
  return guard(H, [&] {
    const int nc0 = H->nc[0], nc1 = H->nc[1], nc2 = H->nc[2];
    const int s_pcc[3] = {H->np[0], nc1, nc2}, s_cpc[3] = {nc0, H->np[1], nc2}, s_ccp[3] = {nc0, nc1, H->np[2]};
    const Pair bx = P2(H->ibc[0][V_QX]), by = P2(H->ibc[1][V_QY]), bz = P2(H->ibc[2][V_QZ]);
    // The checks run in FP64.  In the mixed form the FP32 velocities are first widened into
    // the (FP64-sized) RHS work arrays, and FP64 wall planes are built in the spare planes.
    // the divergence is that of the advanced variable (g for variable properties)
    double *qx = H->qx, *qy = H->qy, *qz = H->qz, *fmaxp = H->fb_maxp, *fqy = H->fb_qy;
    double *ux = H->thermo ? H->gx : H->qx, *uy = H->thermo ? H->gy : H->qy, *uz = H->thermo ? H->gz : H->qz;
    if (H->mixed) {
      launch_convert(H->mx, reinterpret_cast<const float*>(H->qx), (int64_t)H->n_pcc, H->st);
      launch_convert(H->my, reinterpret_cast<const float*>(H->qy), (int64_t)H->n_cpc, H->st);
      launch_convert(H->mz, reinterpret_cast<const float*>(H->qz), (int64_t)H->n_ccp, H->st);
      if (H->thermo) {
        launch_convert(H->px, reinterpret_cast<const float*>(H->gx), (int64_t)H->n_pcc, H->st);
        launch_convert(H->py, reinterpret_cast<const float*>(H->gy), (int64_t)H->n_cpc, H->st);
        launch_convert(H->pz, reinterpret_cast<const float*>(H->gz), (int64_t)H->n_ccp, H->st);
        ux = H->px; uy = H->py; uz = H->pz;
        H->launches += 3;
      } else {
        ux = H->mx; uy = H->my; uz = H->mz;
      }
      launch_fbcy_const(H->fb_comb, nc0, nc2, kMaxp, kMaxp, H->st);
      launch_fbcy_const(H->fb_visc2, nc0, nc2, H->fbcy[V_QY][0], H->fbcy[V_QY][1], H->st);
      qx = H->mx; qy = H->my; qz = H->mz; fmaxp = H->fb_comb; fqy = H->fb_visc2;
      H->launches += 5;
    }
    // divergence (Get_divergence_flow, src/eq_continuity.f90:91-161) into `div`
    run_op(H, 0, D1P2C, bx, fmaxp, src(ux), s_pcc, H->div, false, 1.0);
    run_op(H, 1, D1P2C, by, nullptr, src(uy), s_cpc, H->div, true, 1.0);
    run_op(H, 2, D1P2C, bz, nullptr, src(uz), s_ccp, H->div, true, 1.0);
    launch_absmax(H->div, (int64_t)H->n_ccc, H->partial, H->npart, H->scal + 2, H->st);
    // the reference's three x-slab monitors of the same divergence (Check_element_mass_conservation,
    // src/eq_continuity.f90:379-389; its d(rho)/dt term is zero there, rho_m1 = rho after the
    // property update)
    launch_absmax_slabs(H->div, nc0, (int64_t)nc1 * nc2, reinterpret_cast<unsigned long long*>(H->scal + 8), H->st);
    // kinetic energy of the P2C-interpolated velocities (src/io_monitor.f90:209-241)
    run_op(H, 0, M1P2C, bx, fmaxp, src(qx), s_pcc, H->qxix, false, 1.0);
    run_op(H, 1, M1P2C, by, H->periodic_y ? nullptr : fqy, src(qy), s_cpc, H->qyiy, false, 1.0);
    run_op(H, 2, M1P2C, bz, fmaxp, src(qz), s_ccp, H->qziz, false, 1.0);
    launch_ke_density(H->qxdx, H->qxix, H->qyiy, H->qziz, (int64_t)H->n_ccc, H->st);
    launch_weighted_mean(H->qxdx, H->wy, nc0, nc1, nc2, H->partial, H->npart, H->scal + 4, H->vol, H->st);
    launch_weighted_mean(qx, H->wy, H->np[0], nc1, nc2, H->partial, H->npart, H->scal + 5, H->vol, H->st);
    H->launches += 8;
    double s[11];
    CK(cudaMemcpyAsync(s, H->scal, 11 * sizeof(double), cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    for (int m = 0; m < 3; ++m) out->mcon[m] = s[8 + m];
    out->max_div = s[2];
    out->nan_flag = s[3] != 0.0 ? 1 : 0;
    out->bulk_ke = s[4];
    out->bulk_u = s[5];
    out->last_bulk_rhs = s[0];
  });
}

int chs_op3d(chs_handle* H, int dir, int fam, int ibc1, int ibc2, const double* fbc2d, const double* in,
             const int nin3[3], double* out) {
  if (!H || !in || !out || !nin3 || dir < 0 || dir > 2 || fam < 0 || fam > 5) return CHS_ERR_ARG;
  return guard(H, [&] {
    const int n1 = nin3[0], n2 = nin3[1], n3 = nin3[2];
    const size_t nin = (size_t)n1 * n2 * n3;
    int o[3] = {n1, n2, n3};
    o[dir] = fam_p_output(fam) ? H->np[dir] : H->nc[dir];
    const size_t nout = (size_t)o[0] * o[1] * o[2];
    const int64_t nl = num_lines(dir, n1, n2, n3);
    Pair bc{{ibc1, ibc2}};
    const size_t before = H->book.table.size();
    H->plan(dir, fam, bc, fbc2d != nullptr);
    if (H->book.table.size() != before) upload_table(H);
    double *din, *dout, *dfbc = nullptr;
    CK(cudaMallocAsync(&din, nin * sizeof(double), H->st));
    CK(cudaMallocAsync(&dout, nout * sizeof(double), H->st));
    CK(cudaMemcpyAsync(din, in, nin * sizeof(double), cudaMemcpyHostToDevice, H->st));
    std::vector<double> fb;
    if (fbc2d) {
      // reference layouts fbcx(4,n2,n3) / fbcy(n1,4,n3) / fbcz(n1,n2,4) -> [4][lines]
      fb.resize(4 * nl);
      for (int64_t L = 0; L < nl; ++L)
        for (int u = 0; u < 4; ++u) {
          size_t src_i;
          if (dir == 0) src_i = (size_t)L * 4 + u;
          else if (dir == 1) { int64_t k = L / n1, i = L - k * n1; src_i = (size_t)(k * 4 + u) * n1 + i; }
          else { int64_t j = L / n1, i = L - j * n1; src_i = (size_t)(u * n2 + j) * n1 + i; }
          fb[u * nl + L] = fbc2d[src_i];
        }
      CK(cudaMallocAsync(&dfbc, fb.size() * sizeof(double), H->st));
      CK(cudaMemcpyAsync(dfbc, fb.data(), fb.size() * sizeof(double), cudaMemcpyHostToDevice, H->st));
    }
    run_op(H, dir, fam, bc, dfbc, src(din), nin3, dout, false, 1.0);
    CK(cudaMemcpyAsync(out, dout, nout * sizeof(double), cudaMemcpyDeviceToHost, H->st));
    CK(cudaStreamSynchronize(H->st));
    cudaFreeAsync(din, H->st);
    cudaFreeAsync(dout, H->st);
    if (dfbc) cudaFreeAsync(dfbc, H->st);
    CK(cudaStreamSynchronize(H->st));
  });
}

// Host-only inspection of one operator plan (no device work).  Layout of buf:
// [0..15] fam nin nout b_lo b_hi off0..3 sgn r1 r2 dd nspec tdma b1
// [16..19] an cn inv_den neu1*2+neu2
// [20 + 26*s ..] special row s: row nt idx[10] w[10] wb[4]  (s < 4)
// [128 ..] a c' d x1 map (nout each; zeros when absent)
int chs_plan_inspect(const chs_config* cfg, int dir, int fam, int ibc1, int ibc2, int has_fbc, double* buf,
                     size_t len) {
  if (!cfg || !buf || dir < 0 || dir > 2 || fam < 0 || fam > 5) return CHS_ERR_ARG;
  chs_handle H;
  try {
    setup_host(&H, cfg);
    int bc[2] = {ibc1, ibc2};
    OpPlan P = H.book.make(dir, fam, bc, has_fbc != 0);
    const int n = P.nout;
    if (len < (size_t)(128 + 5 * n)) return CHS_ERR_ARG;
    for (size_t i = 0; i < len; ++i) buf[i] = 0.0;
    double hd[20] = {(double)P.fam, (double)P.nin, (double)P.nout, (double)P.b_lo, (double)P.b_hi,
                     (double)P.off[0], (double)P.off[1], (double)P.off[2], (double)P.off[3], P.sgn, P.r1, P.r2,
                     P.dd, (double)P.nspec, (double)P.tdma, P.b1, P.an, P.cn, P.inv_den,
                     (double)(P.neu1 * 2 + P.neu2 + 4 * P.wrap)};
    for (int i = 0; i < 20; ++i) buf[i] = hd[i];
    for (int k = 0; k < P.nspec; ++k) {
      double* o = buf + 20 + 26 * k;
      o[0] = P.sp[k].row;
      o[1] = P.sp[k].nt;
      for (int t = 0; t < P.sp[k].nt; ++t) { o[2 + t] = P.sp[k].idx[t]; o[12 + t] = P.sp[k].w[t]; }
      for (int u = 0; u < 4; ++u) o[22 + u] = P.sp[k].wb[u];
    }
    const std::vector<double>& T = H.book.table;
    double* arr = buf + 128;
    for (int i = 0; i < n; ++i) {
      if (P.tdma) {
        arr[i] = T[P.la + i];
        arr[n + i] = T[P.lc + i];
        arr[2 * n + i] = T[P.ld + i];
        arr[3 * n + i] = T[P.lx1 + i];
      }
      if (P.lmap >= 0) arr[4 * n + i] = T[P.lmap + i];
    }
    return CHS_OK;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "chs_plan_inspect: %s\n", e.what());
    return CHS_ERR_ARG;
  }
}

int chs_sync(chs_handle* H) {
  if (!H) return CHS_ERR_ARG;
  return guard(H, [&] { CK(cudaStreamSynchronize(H->st)); });
}

long long chs_kernel_launches(const chs_handle* H) { return H ? H->launches : 0; }

int chs_last_error(const chs_handle* H, char* buf, size_t len) {
  if (!H || !buf || len == 0) return CHS_ERR_ARG;
  std::snprintf(buf, len, "%s", H->err.c_str());
  return CHS_OK;
}

}  // extern "C"
