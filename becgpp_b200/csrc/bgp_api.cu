// Host side of libbgp.so: plans, twiddle and kernel tables, team scheduling,
// cooperative launches and the C ABI declared in include/bgp.h.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bgp.h"
#include "bgp_programs.cuh"
#include "bgp_sizes_gen.h"
#include "bgp_table.cuh"
#include "bgp_tf.cuh"
#include "bgp_stream.cuh"

using namespace bgp;

namespace {

constexpr int kProfSlots = 20 * 5;   // phase profiler: 20 phase kinds x 5 counters
constexpr int kYieldDiv = 4;         // a solve launch yields once 1/kYieldDiv of it has finished
constexpr int kTuneYield[3] = {2, 4, 8};  // relaunch schedules the autotuner tries
constexpr int kMaxSegments = 256;    // relaunch limit of one solve

thread_local std::string g_err;
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(e_ == cudaErrorMemoryAllocation ? BGP_ERR_OOM : BGP_ERR_CUDA,       \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

bool size_ok(int N, int M) {
#define X(n, m) if (N == n && M == m) return true;
  BGP_FOR_SIZES(X)
#undef X
  return false;
}

// kernel entry for a size pair, or for two pairs (mixed: the build with FP32
// transforms); null if not compiled
void* kernel_for(int N, int M, int ndim, bool mixed = false) {
#define X(n, m)                                                                              \
  if (N == n && M == m) {                                                                    \
    if (ndim == 3) return mixed ? bgp_kptr_##n##_##m##_d3_mx() : bgp_kptr_##n##_##m##_d3(); \
    return mixed ? bgp_kptr_##n##_##m##_d2_mx() : bgp_kptr_##n##_##m##_d2();               \
  }
  BGP_FOR_SIZES(X)
#undef X
  return nullptr;
}
// two-size kernels (2D only)
void* kernel_for2(int N1, int M1, int N2, int M2, int ndim, bool mixed = false) {
  if (ndim != 2) return nullptr;
#define X(a, b, c, d)                                                                      \
  if ((N1 == a && M1 == b && N2 == c && M2 == d) ||                                      \
      (N1 == c && M1 == d && N2 == a && M2 == b))                                        \
    return mixed ? bgp_kptr2_##a##_##b##_##c##_##d##_d2_mx() : bgp_kptr2_##a##_##b##_##c##_##d##_d2();
  BGP_FOR_COMBOS(X)
#undef X
  return nullptr;
}

}  // namespace

// Forward FFT of every line along axis `ax` of an L^d complex cube (table build).
template <int L>
struct OpCube {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = false;
  BGP_NO_OUT(64)
  const Inst& I;
  int ax;
  double2* A;
  BGP_D Pre fetch(int t, int r, int c) {
    int i, j, k;
    Pre P;
    P.a = A[nline_elem(I, ax, t, r, c, i, j, k)];
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int, int) { return P.a; }
  BGP_D void line(double2* b, int lane, int, int) { warp_fft<L, false>(b, I.twN, lane); }
  BGP_D void leave(const Pre&, int t, int r, int c, double2 v) {
    int i, j, k;
    A[nline_elem(I, ax, t, r, c, i, j, k)] = v;
  }
};

template <int L>
__global__ void __launch_bounds__(kThreads) k_cube_fft(Inst I, int ax, double2* A) {
  extern __shared__ double2 dyn_sm[];
  OpCube<L> op{I, ax, A};
  const int nt = ntiles_axis(I);
  for (int t = blockIdx.x; t < nt; t += gridDim.x) {
    if (ax == I.ndim - 1) tile_run<L, true>(op, dyn_sm, t);
    else tile_run<L, false>(op, dyn_sm, t);
  }
}

__global__ void k_scale_c(double2* a, long long n, double s) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    a[q] = cscale(a[q], s);
}

// ---------------------------------------------------------------- host state
namespace {

struct DevCtx {
  int device = -1, sms = 0, max_grid = 0;
  size_t max_smem_optin = 0;
  std::map<int, double2*> tw;   // twiddle tables by length
  std::map<int, float2*> tw32;  // the same rounded to FP32
};
std::mutex g_mu;
std::map<int, DevCtx> g_dev;

int ensure_device(DevCtx** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  DevCtx& d = g_dev[dev];
  if (d.device < 0) {
    cudaDeviceProp p;
    CK(cudaGetDeviceProperties(&p, dev));
    d.device = dev;
    d.sms = p.multiProcessorCount;
    d.max_smem_optin = p.sharedMemPerBlockOptin;
  }
  *out = &d;
  return BGP_OK;
}

// exp(-2 pi i t / L), t = 0..L-1, from long-double sin/cos of the reduced angle
int twiddles(DevCtx* d, int L, const double2** out) {
  auto it = d->tw.find(L);
  if (it != d->tw.end()) { *out = it->second; return BGP_OK; }
  std::vector<double2> h(L);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int t = 0; t < L; ++t) {
    // reduce to the first octant by symmetry so the table is exactly symmetric
    const long double ang = 2.0L * pi * (long double)t / (long double)L;
    long double c = cosl(ang), s = sinl(ang);
    if (8LL * t % L == 0) {
      const int oct = (int)(8LL * t / L);
      const double cs[8] = {1, M_SQRT1_2, 0, -M_SQRT1_2, -1, -M_SQRT1_2, 0, M_SQRT1_2};
      const double sn[8] = {0, M_SQRT1_2, 1, M_SQRT1_2, 0, -M_SQRT1_2, -1, -M_SQRT1_2};
      c = cs[oct]; s = sn[oct];
    }
    h[t] = cmk((double)c, -(double)s);
  }
  double2* dp = nullptr;
  CK(cudaMalloc(&dp, sizeof(double2) * L));
  CK(cudaMemcpy(dp, h.data(), sizeof(double2) * L, cudaMemcpyHostToDevice));
  d->tw[L] = dp;
  std::vector<float2> hf(L);
  for (int t = 0; t < L; ++t) hf[t] = cmake<float2>((float)h[t].x, (float)h[t].y);
  float2* fp = nullptr;
  CK(cudaMalloc(&fp, sizeof(float2) * L));
  CK(cudaMemcpy(fp, hf.data(), sizeof(float2) * L, cudaMemcpyHostToDevice));
  d->tw32[L] = fp;
  *out = dp;
  return BGP_OK;
}

int twiddles32(DevCtx* d, int L, const float2** out) {
  const double2* dp = nullptr;
  int rc = twiddles(d, L, &dp);
  if (rc) return rc;
  *out = d->tw32[L];
  return BGP_OK;
}

}  // namespace

struct bgp_plan {
  DevCtx* dev = nullptr;
  std::vector<bgp_instance_desc> desc;
  std::vector<Inst> inst;                 // host copies with device pointers
  std::vector<void*> allocs;
  long long bytes = 0;
  Inst* d_inst = nullptr;
  int* d_cta_inst = nullptr;
  int* d_abort = nullptr;
  int* d_finished = nullptr;               // finished-instance counter of a solve launch
  long long launches = 0;                  // kernel launches issued by this plan
  SolveOut* d_out = nullptr;
  double* d_res = nullptr;                // n_inst x (kNRec + 1)
  int max_team = 0;
  int lmax = 0;
  size_t smem = 0;
  int grid_cap = 0;
  std::vector<int> cta_inst;
  // relaunch schedule and its autotuner: 0 off, 1 trying candidates, 2 done
  int yield_div = kYieldDiv;
  int tune = 0, tune_next = 0;
  float tune_ms[3] = {0.f, 0.f, 0.f};
  // stream-pass schedules by line length N (autotuned on first use unless fixed)
  struct StreamSched {
    int ln = 0, v = 0;            // H psi lines per tile, radix order
    int cln = 8, csln = 8, cv = 0;   // convolution: lines of contiguous / strided tiles, radix order
    int tuned = 0;                // 0: tune on first use, 1: tuned, 2: fixed by the caller
    std::vector<std::array<float, 4>> cand;   // (ln, v, strided ln, ms) of every timed candidate
  };
  std::map<int, StreamSched> ssched;
  // batched apply: one stream per further size group (forked from and joined to the
  // caller's stream by events), so groups of different sizes overlap on the GPU
  std::vector<cudaStream_t> side_st;
  std::vector<cudaEvent_t> side_ev;   // [0] the fork, [1 + g] the join of side group g
  // per size group: the stream of the H psi passes that run beside its convolution,
  // and that overlap's fork and join events
  std::vector<cudaStream_t> ovl_st;
  std::vector<cudaEvent_t> ovl_ev;
};

namespace {

int palloc(bgp_plan* p, size_t bytes, void** out) {
  void* q = nullptr;
  if (bytes == 0) { *out = nullptr; return BGP_OK; }
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) return fail(BGP_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  p->allocs.push_back(q);
  p->bytes += (long long)bytes;
  CK(cudaMemset(q, 0, bytes));
  *out = q;
  return BGP_OK;
}

template <class T>
int palloc_t(bgp_plan* p, size_t count, T** out) {
  void* q = nullptr;
  int rc = palloc(p, count * sizeof(T), &q);
  *out = (T*)q;
  return rc;
}

template <int L>
int cube_fft_len(const Inst& I, double2* A, int ax) {
  const size_t smem = tile_smem_bytes(L);
  CK(cudaFuncSetAttribute(k_cube_fft<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int nt = ntiles_axis(I);
  k_cube_fft<L><<<nt < 4096 ? nt : 4096, kThreads, smem>>>(I, ax, A);
  CK(cudaGetLastError());
  return BGP_OK;
}

int cube_fft(const Inst& I, double2* A, int ax) {
  switch (I.N) {
#define X(l) case l: return cube_fft_len<l>(I, A, ax);
    BGP_FOR_TABLE_LENGTHS(X)
#undef X
    default: return fail(BGP_ERR_UNSUPPORTED, "kernel table length not compiled in");
  }
}

// Build the real quadrant of the transformed cell-averaged kernel table.
int build_table(bgp_plan* p, const bgp_instance_desc& d, const Inst& I, int which, double** out) {
  const int M = I.M, ndim = I.ndim;
  const size_t tot = (ndim == 2) ? (size_t)M * M : (size_t)M * M * M;
  double2* F = nullptr;
  CK(cudaMalloc(&F, tot * sizeof(double2)));
  k_table_fill<<<1184, 256>>>(F, ndim, M, I.dx, I.kind, which, d.l_z);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { cudaFree(F); return fail(BGP_ERR_CUDA, cudaGetErrorString(e)); }
  // exact self cell at the origin (interactions.py:128-135, 146)
  double self;
  if (which == 1) self = polar_self_cell_2d(I.kind, 1, d.l_z, I.dx);
  else if (ndim == 3) self = kSelfNewton3D / I.dx;
  else if (I.kind == kNewton) self = 4.0 * asinh(1.0) / I.dx;
  else if (I.kind == kLog) self = -log(I.dx) + (1.5 + 0.5 * log(2.0) - 0.25 * M_PI);
  else self = polar_self_cell_2d(I.kind, 0, d.l_z, I.dx);
  const double2 sc = cmk(self, 0.0);
  CK(cudaMemcpy(F, &sc, sizeof(double2), cudaMemcpyHostToDevice));
  Inst C = I;
  C.N = M;  // transform the M-cube with the M twiddles
  C.twN = I.twM;
  for (int ax = 0; ax < ndim; ++ax) {
    int rc = cube_fft(C, F, ax);
    if (rc) { cudaFree(F); return rc; }
  }
  const int Mh = M / 2 + 1;
  const size_t qn = (ndim == 2) ? (size_t)Mh * Mh : (size_t)Mh * Mh * Mh;
  double* Kq = nullptr;
  int rc = palloc_t(p, qn, &Kq);
  if (rc) { cudaFree(F); return rc; }
  k_table_quadrant<<<1184, 256>>>(F, Kq, ndim, M);
  e = cudaDeviceSynchronize();
  cudaFree(F);
  if (e != cudaSuccess) return fail(BGP_ERR_CUDA, std::string("kernel table: ") + cudaGetErrorString(e));
  *out = Kq;
  return BGP_OK;
}

int grid_cap_for(bgp_plan* p, void* kern, int* cap) {
  int nb = 0;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kThreads, p->smem));
  if (nb < 1) return fail(BGP_ERR_CUDA, "solver kernel does not fit on an SM");
  *cap = nb * p->dev->sms;
  return BGP_OK;
}

int max_grid(bgp_plan* p) {
  int cap = 1 << 30;
  for (const Inst& I : p->inst) {
    for (bool mixed : {false, true}) {
      void* k = kernel_for(I.N, I.M, I.ndim, mixed);
      if (!k) return fail(BGP_ERR_UNSUPPORTED, "grid size not compiled in");
      int c = 0;
      int rc = grid_cap_for(p, k, &c);
      if (rc) return rc;
      cap = c < cap ? c : cap;
    }
  }
  p->grid_cap = cap;
  return BGP_OK;
}

// CTAs an instance can keep busy in its widest phase
int useful_ctas(const Inst& I) {
  const int nt = ntiles_axis(I);
  if (I.kind == kNone || I.M == 0) return nt;
  const int tpl = (I.Mh + kLines - 1) / kLines;
  return nt + (I.ndim == 2 ? tpl : I.M * tpl);
}

int launch_group(bgp_plan* p, const std::vector<int>& active, void* kern, cudaStream_t st);

// Launch the active instances: one kernel when they share a size (or form a
// compiled two-size combination), otherwise one launch per size group.
int launch(bgp_plan* p, const std::vector<int>& active, cudaStream_t st) {
  // kinds of kernel: (ndim, N, M)
  std::vector<std::array<int, 3>> kinds;
  auto kind_of = [&](int a) {
    const Inst& I = p->inst[a];
    return std::array<int, 3>{I.ndim, I.N, I.M};
  };
  for (int a : active) {
    const auto k = kind_of(a);
    bool seen = false;
    for (auto& q : kinds) seen = seen || q == k;
    if (!seen) kinds.push_back(k);
  }
  // a mixed-precision solve runs in the kernels built with FP32 transforms while
  // one of its instances still uses them
  bool mixed = false;
  for (int a : active) mixed = mixed || (p->inst[a].prog == kProgSolve && p->inst[a].sp.mixed);
  if (kinds.size() == 1)
    return launch_group(p, active, kernel_for(kinds[0][1], kinds[0][2], kinds[0][0], mixed), st);
  if (kinds.size() == 2 && kinds[0][0] == kinds[1][0]) {
    void* k2 = kernel_for2(kinds[0][1], kinds[0][2], kinds[1][1], kinds[1][2], kinds[0][0], mixed);
    if (k2) return launch_group(p, active, k2, st);
  }
  for (auto& k : kinds) {
    std::vector<int> grp;
    for (int a : active) if (kind_of(a) == k) grp.push_back(a);
    int rc = launch_group(p, grp, kernel_for(k[1], k[2], k[0], mixed), st);
    if (rc) return rc;
  }
  return BGP_OK;
}

// Assign teams to the active instances and launch the persistent kernel.
int launch_group(bgp_plan* p, const std::vector<int>& active, void* kern, cudaStream_t st) {
  if (!kern) return fail(BGP_ERR_UNSUPPORTED, "grid size not compiled in");
  const int na = (int)active.size();
  std::vector<int> team(na, 1);
  std::vector<double> w(na);
  double wsum = 0.0;
  for (int a = 0; a < na; ++a) { w[a] = (double)p->inst[active[a]].n; wsum += w[a]; }
  if (na > p->grid_cap) return fail(BGP_ERR_ARG, "more instances than resident CTAs in one batch");
  int cap = p->grid_cap;
  int used = 0;
  for (int a = 0; a < na; ++a) {
    const int want = useful_ctas(p->inst[active[a]]);
    int t = (int)floor(cap * w[a] / wsum);
    t = t < 1 ? 1 : t;
    t = t > want ? want : t;
    t = t > p->max_team ? p->max_team : t;
    team[a] = t;
    used += t;
  }
  // hand out what is left, largest instances first
  for (bool grew = true; used < cap && grew;) {
    grew = false;
    for (int a = 0; a < na && used < cap; ++a) {
      const int want = useful_ctas(p->inst[active[a]]);
      if (team[a] < want && team[a] < p->max_team) { team[a]++; used++; grew = true; }
    }
  }
  while (used > cap) {  // only if the floor-1 clamps overflowed
    int big = 0;
    for (int a = 1; a < na; ++a) if (team[a] > team[big]) big = a;
    if (team[big] <= 1) return fail(BGP_ERR_ARG, "batch too large for one launch");
    team[big]--; used--;
  }
  std::vector<Inst> hi(na);
  p->cta_inst.assign(used, 0);
  int first = 0;
  for (int a = 0; a < na; ++a) {
    hi[a] = p->inst[active[a]];
    hi[a].team_first = first;
    hi[a].team_size = team[a];
    for (int q = 0; q < team[a]; ++q) p->cta_inst[first + q] = a;
    first += team[a];
  }
  CK(cudaMemcpyAsync(p->d_inst, hi.data(), sizeof(Inst) * na, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(p->d_cta_inst, p->cta_inst.data(), sizeof(int) * used, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(p->d_abort, 0, (4 + (size_t)used) * sizeof(int), st));
  for (int a = 0; a < na; ++a) CK(cudaMemsetAsync(hi[a].bar, 0, sizeof(unsigned long long), st));
  Launch L{p->d_inst, p->d_cta_inst, p->d_abort};
  void* args[] = {&L};
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->smem));
  CK(cudaLaunchCooperativeKernel(kern, dim3(used), dim3(kThreads), args, p->smem, st));
  p->launches++;
  CK(cudaGetLastError());
  int ab[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(ab, p->d_abort, sizeof(ab), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (ab[0] != 0) {
    // last barrier arrival of every CTA of the team that timed out
    std::vector<int> arr(used);
    CK(cudaMemcpy(arr.data(), p->d_abort + 4, sizeof(int) * used, cudaMemcpyDeviceToHost));
    std::string team;
    const int a0 = ab[1] >= 0 && ab[1] < used ? p->cta_inst[ab[1]] : -1;
    for (int b = 0; b < used; ++b)
      if (p->cta_inst[b] == a0) team += std::to_string(b) + ":" + std::to_string(arr[b]) + " ";
    char buf[200];
    snprintf(buf, sizeof buf,
             "device status %d (1 = team barrier timeout, 2 = size not compiled); block %d waited "
             "for barrier count %d and saw %d; last arrivals (block:count) ", ab[0], ab[1], ab[2], ab[3]);
    return fail(BGP_ERR_DEVICE, std::string(buf) + team);
  }
  return BGP_OK;
}

int check_inst(const bgp_plan* p, int i) {
  if (!p) return fail(BGP_ERR_ARG, "null plan");
  if (i < 0 || i >= (int)p->inst.size()) return fail(BGP_ERR_ARG, "instance index out of range");
  return BGP_OK;
}

}  // namespace

// error reporting for the other translation units of the library
int bgp_report_error(int code, const char* msg) { return fail(code, msg); }

// ======================================================================= C ABI
extern "C" {

int bgp_version(void) { return 100; }
const char* bgp_last_error(void) { return g_err.c_str(); }

double bgp_k0e(double x) { double a, b; k01e(x, a, b); return a; }
double bgp_k1e(double x) { double a, b; k01e(x, a, b); return b; }

int bgp_size_supported(int ndim, int N, int pad, int kernel) {
  if (ndim != 2 && ndim != 3) return 0;
  if (kernel != BGP_KERNEL_NONE && pad != 2) return 0;
  return size_ok(N, kernel == BGP_KERNEL_NONE ? 0 : 2 * N) ? 1 : 0;
}

int bgp_plan_create(const bgp_instance_desc* desc, int n_inst, bgp_plan** plan) {
  if (!desc || n_inst < 1 || !plan) return fail(BGP_ERR_ARG, "bad arguments");
  std::lock_guard<std::mutex> lk(g_mu);
  DevCtx* dev = nullptr;
  int rc = ensure_device(&dev);
  if (rc) return rc;
  bgp_plan* p = new bgp_plan();
  p->dev = dev;
  p->desc.assign(desc, desc + n_inst);
  p->inst.resize(n_inst);
  auto bail = [&](int code) { bgp_plan_destroy(p); return code; };
  // first pass: sizes
  for (int i = 0; i < n_inst; ++i) {
    const bgp_instance_desc& d = desc[i];
    if (d.ndim != 2 && d.ndim != 3) return bail(fail(BGP_ERR_ARG, "ndim must be 2 or 3"));
    if (d.kernel < 0 || d.kernel > 3) return bail(fail(BGP_ERR_ARG, "unknown kernel"));
    if (d.kernel == BGP_KERNEL_LOG && d.ndim != 2) return bail(fail(BGP_ERR_ARG, "kernel 'log' is 2D only"));
    if (d.kernel == BGP_KERNEL_Q2D && (d.ndim != 2 || !(d.l_z > 0))) return bail(fail(BGP_ERR_ARG, "kernel 'q2d' needs 2D and l_z > 0"));
    if (d.kernel == BGP_KERNEL_NEWTON && false) {}
    if (!(d.L > 0)) return bail(fail(BGP_ERR_ARG, "L must be positive"));
    if (d.kernel != BGP_KERNEL_NONE && d.pad != 2)
      return bail(fail(BGP_ERR_UNSUPPORTED, "only pad = 2 is compiled in for the long-range term"));
    const int M = d.kernel == BGP_KERNEL_NONE ? 0 : 2 * d.N;
    if (!size_ok(d.N, M)) {
      char buf[160];
      snprintf(buf, sizeof buf, "grid N=%d%s is not compiled in (supported: 16 24 32 48 64 96 128 192 256 384 512; "
               "up to 384 with a long-range kernel)", d.N, M ? " with a long-range kernel" : "");
      return bail(fail(BGP_ERR_UNSUPPORTED, buf));
    }
    Inst& I = p->inst[i];
    memset(&I, 0, sizeof(Inst));
    I.ndim = d.ndim; I.N = d.N; I.M = M; I.kind = d.kernel;
    I.n = d.ndim == 2 ? d.N * d.N : d.N * d.N * d.N;
    I.Mh = M ? M / 2 + 1 : 0;
    I.i0 = M ? (M - d.N) / 2 : 0;
    I.dx = 2.0 * d.L / d.N;
    I.dv = d.ndim == 2 ? I.dx * I.dx : I.dx * I.dx * I.dx;
    I.kfac = 1.0 / (d.N * I.dx);
    I.s = d.s; I.tc = d.trap_coeff;
    I.beta2 = d.beta2; I.beta3 = d.beta3; I.Omega = d.Omega; I.G_C = d.G_C;
    I.inv_n = 1.0 / (double)I.n;
    const double Md = M ? (d.ndim == 2 ? (double)M * M : (double)M * M * M) : 1.0;
    I.conv_scale = M ? -d.G_C * I.dv / Md : 0.0;
    p->lmax = std::max(p->lmax, std::max(d.N, M));
  }
  // the tile buffer; the median's rank selection reuses it for kSelCap keys
  p->smem = std::max(tile_smem_bytes(p->lmax), (size_t)kSelCap * sizeof(unsigned long long));
  if (p->smem > dev->max_smem_optin) return bail(fail(BGP_ERR_UNSUPPORTED, "tile does not fit in shared memory"));
  rc = max_grid(p);
  if (rc) return bail(rc);
  p->max_team = p->grid_cap;
  for (int i = 0; i < n_inst; ++i) {
    Inst& I = p->inst[i];
    const bgp_instance_desc& d = desc[i];
    const size_t n = (size_t)I.n;
    if ((rc = twiddles(dev, I.N, &I.twN))) return bail(rc);
    if ((rc = twiddles32(dev, I.N, &I.twN32))) return bail(rc);
    if (I.M && (rc = twiddles(dev, I.M, &I.twM))) return bail(rc);
    if (I.M && (rc = twiddles32(dev, I.M, &I.twM32))) return bail(rc);
    if ((rc = palloc_t(p, (size_t)kNB * n, &I.pool))) return bail(rc);
    // potentials: current and trial; 3D with a kernel also the potentials of the
    // density's linear and quadratic parts in the step (the line search's quartic)
    if ((rc = palloc_t(p, (I.M && I.ndim == 3 ? 4 : 2) * n, &I.phi2))) return bail(rc);
    if ((rc = palloc_t(p, n, &I.keys))) return bail(rc);
    if ((rc = palloc_t(p, (size_t)8 * 256 + 2, &I.hist))) return bail(rc);
    if ((rc = palloc_t(p, (size_t)kSelCap, &I.cand))) return bail(rc);
    if ((rc = palloc_t(p, (size_t)kSelCap, &I.wcand))) return bail(rc);
    // reduction partials: the solver's (2 x kNRec per team CTA) and the stream H psi
    // passes' (one per tile of the last pass: up to N^(d-1) with one-line tiles)
    const size_t stream_tiles = I.ndim == 2 ? (size_t)I.N : (size_t)I.N * I.N;
    if ((rc = palloc_t(p, std::max((size_t)2 * kNRec * p->max_team, stream_tiles), &I.part))) return bail(rc);
    if ((rc = palloc_t(p, (size_t)1, &I.bar))) return bail(rc);
    if ((rc = palloc(p, sizeof(Ctl), &I.save))) return bail(rc);
    if (I.M) {
      const size_t c1 = I.ndim == 2 ? (size_t)I.N * I.Mh : (size_t)I.N * I.N * I.Mh;
      if ((rc = palloc_t(p, c1, &I.cb1))) return bail(rc);
      if (I.ndim == 3 && (rc = palloc_t(p, (size_t)I.N * I.M * I.Mh, &I.cb2))) return bail(rc);
      double* Kq = nullptr;
      if ((rc = build_table(p, d, I, 0, &Kq))) return bail(rc);
      I.Kq = Kq;
      if (I.kind == kQ2d) {
        double* Wq = nullptr;
        if ((rc = build_table(p, d, I, 1, &Wq))) return bail(rc);
        I.Wq = Wq;
      }
    }
  }
  if ((rc = palloc_t(p, (size_t)n_inst, &p->d_inst))) return bail(rc);
  if ((rc = palloc_t(p, (size_t)p->grid_cap, &p->d_cta_inst))) return bail(rc);
  if ((rc = palloc_t(p, (size_t)4 + p->grid_cap, &p->d_abort))) return bail(rc);
  if ((rc = palloc_t(p, (size_t)1, &p->d_finished))) return bail(rc);
  if ((rc = palloc_t(p, (size_t)n_inst, &p->d_out))) return bail(rc);
  if ((rc = palloc_t(p, (size_t)n_inst * (kNRec + 1), &p->d_res))) return bail(rc);
  for (int i = 0; i < n_inst; ++i) {
    p->inst[i].out = p->d_out + i;
    p->inst[i].res = p->d_res + (size_t)i * (kNRec + 1);
  }
#if defined(BGP_PROF)
  unsigned long long* prof = nullptr;
  if ((rc = palloc_t(p, (size_t)n_inst * kProfSlots, &prof))) return bail(rc);
  for (int i = 0; i < n_inst; ++i) p->inst[i].prof = prof + (size_t)i * kProfSlots;
#endif
  *plan = p;
  return BGP_OK;
}

int bgp_plan_destroy(bgp_plan* p) {
  if (!p) return BGP_OK;
  for (cudaStream_t q : p->side_st) cudaStreamDestroy(q);
  for (cudaStream_t q : p->ovl_st) cudaStreamDestroy(q);
  for (cudaEvent_t q : p->ovl_ev) cudaEventDestroy(q);
  for (cudaEvent_t q : p->side_ev) cudaEventDestroy(q);
  for (void* q : p->allocs) cudaFree(q);
  delete p;
  return BGP_OK;
}

long long bgp_plan_bytes(const bgp_plan* p) { return p ? p->bytes : 0; }

int bgp_plan_autotune(bgp_plan* p, int enable) {
  if (!p) return fail(BGP_ERR_ARG, "null plan");
  if (enable) { p->tune = 1; p->tune_next = 0; }
  else if (p->tune == 1) { p->tune = 0; }
  return BGP_OK;
}

int bgp_plan_schedule(const bgp_plan* p, int* yield_div, int* tuned, float* ms3) {
  if (!p) return fail(BGP_ERR_ARG, "null plan");
  if (yield_div) *yield_div = p->yield_div;
  if (tuned) *tuned = p->tune == 2;
  if (ms3) for (int c = 0; c < 3; ++c) ms3[c] = p->tune_ms[c];
  return BGP_OK;
}

#if defined(BGP_PROF)
// Phase profiler counters of instance i (kProfSlots values), profiling builds only.
int bgp_prof_read(bgp_plan* p, int i, unsigned long long* out, int reset) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(out, p->inst[i].prof, sizeof(unsigned long long) * kProfSlots, cudaMemcpyDeviceToHost));
  if (reset) CK(cudaMemset(p->inst[i].prof, 0, sizeof(unsigned long long) * kProfSlots));
  return BGP_OK;
}
#endif
long long bgp_plan_launches(const bgp_plan* p) { return p ? p->launches : 0; }

namespace {
int run_api(bgp_plan* p, int i, Inst& I, cudaStream_t st, double* res_host) {
  Inst save = p->inst[i];
  p->inst[i] = I;
  std::vector<int> act{i};
  int rc = launch(p, act, st);
  p->inst[i] = save;
  if (rc) return rc;
  CK(cudaMemcpyAsync(res_host, p->d_res + (size_t)i * (kNRec + 1), sizeof(double) * (kNRec + 1),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (res_host[kNRec] != 0.0) return fail(BGP_ERR_DEVICE, "device program failed");
  return BGP_OK;
}
}  // namespace

int bgp_apply_H(bgp_plan* p, int i, const void* psi, void* hpsi, const double* phi, int phi_mode,
                double* mu_out, void* stream) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  if (!psi || !hpsi) return fail(BGP_ERR_ARG, "null field pointer");
  if (phi_mode == 1 && !phi) return fail(BGP_ERR_ARG, "phi_mode 1 needs phi");
  Inst I = p->inst[i];
  I.prog = kProgApplyH;
  I.in_psi = (const double2*)psi;
  I.out_c = (double2*)hpsi;
  I.in_phi = phi;
  I.use_phi = (I.kind == kNone || I.M == 0) ? (phi_mode == 1 ? 1 : 0) : phi_mode;
  double res[kNRec + 1] = {0};
  CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), (cudaStream_t)stream));
  rc = run_api(p, i, I, (cudaStream_t)stream, res);
  if (rc) return rc;
  if (mu_out) *mu_out = res[0];
  return BGP_OK;
}

int bgp_energy(bgp_plan* p, int i, const void* psi, double* phi_out, bgp_energy_terms* terms,
               void* stream) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  if (!psi || !terms) return fail(BGP_ERR_ARG, "null pointer");
  Inst I = p->inst[i];
  I.prog = kProgEnergy;
  I.in_psi = (const double2*)psi;
  I.out_r = phi_out;
  double res[kNRec + 1] = {0};
  CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), (cudaStream_t)stream));
  rc = run_api(p, i, I, (cudaStream_t)stream, res);
  if (rc) return rc;
  double comp[8];
  energy_assemble(I, res, 1.0, comp);
  terms->E = comp[0]; terms->Ekin = comp[1]; terms->Etrap = comp[2]; terms->Econtact = comp[3];
  terms->Ethree = comp[4]; terms->Erot = comp[5]; terms->Egrav = comp[6]; terms->Lz = comp[7];
  terms->mass = res[S_N0] * I.dv;
  terms->r2mean = res[S_R2] * I.dv;
  terms->peak = res[kNSum];
  terms->rperp2 = res[S_PERP] * I.dv;
  terms->z2 = res[S_Z2] * I.dv;
  return BGP_OK;
}

int bgp_energy_grad(bgp_plan* p, int i, const void* psi, bgp_energy_terms* terms, void* dE_dpsi,
                    double* dparams, void* stream) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  if (!psi || !terms || !dparams) return fail(BGP_ERR_ARG, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const Inst base = p->inst[i];
  const bool kern = base.kind != kNone && base.M > 0;
  // energy terms and the raw sums; the potential goes to the plan's phi buffer 0
  Inst I = base;
  I.prog = kProgEnergy;
  I.in_psi = (const double2*)psi;
  I.out_r = nullptr;
  double res[kNRec + 1] = {0};
  CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), st));
  rc = run_api(p, i, I, st, res);
  if (rc) return rc;
  double comp[8];
  energy_assemble(I, res, 1.0, comp);
  terms->E = comp[0]; terms->Ekin = comp[1]; terms->Etrap = comp[2]; terms->Econtact = comp[3];
  terms->Ethree = comp[4]; terms->Erot = comp[5]; terms->Egrav = comp[6]; terms->Lz = comp[7];
  terms->mass = res[S_N0] * I.dv;
  terms->r2mean = res[S_R2] * I.dv;
  terms->peak = res[kNSum];
  terms->rperp2 = res[S_PERP] * I.dv;
  terms->z2 = res[S_Z2] * I.dv;
  dparams[0] = 0.5 * res[S_2] * I.dv;                                  // dE/dbeta2
  dparams[1] = res[S_3] * I.dv / 3.0;                                  // dE/dbeta3
  dparams[2] = (kern && base.G_C != 0.0) ? comp[6] / base.G_C : 0.0;   // dE/dG_C
  dparams[3] = -comp[7];                                               // dE/dOmega
  dparams[4] = 0.0;                                                    // dE/dl_z
  if (dE_dpsi) {
    // dE/dpsi* = H psi dV, with the potential of this psi
    Inst J = base;
    J.prog = kProgApplyH;
    J.in_psi = (const double2*)psi;
    J.out_c = (double2*)dE_dpsi;
    J.in_phi = base.phi2;
    J.use_phi = kern ? 1 : 0;
    CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), st));
    rc = run_api(p, i, J, st, res);
    if (rc) return rc;
    k_scale_c<<<296, 256, 0, st>>>((double2*)dE_dpsi, (long long)base.n, base.dv);
    CK(cudaGetLastError());
  }
  if (kern && base.kind == kQ2d && base.Wq) {
    // dK/dl_z = -(K + W)/l_z, so dE/dl_z = -(Egrav + E_W)/l_z with E_W the energy of
    // the virial kernel's potential
    Inst J = base;
    J.prog = kProgConvW;
    J.in_psi = (const double2*)psi;
    CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), st));
    rc = run_api(p, i, J, st, res);
    if (rc) return rc;
    const double EW = 0.5 * res[0] * base.dv;
    const double lz = p->desc[i].l_z;
    dparams[4] = -(comp[6] + EW) / lz;
  }
  CK(cudaStreamSynchronize(st));
  return BGP_OK;
}

int bgp_residual(bgp_plan* p, int i, const void* psi, double* out3, void* stream) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  if (!psi || !out3) return fail(BGP_ERR_ARG, "null pointer");
  Inst I = p->inst[i];
  I.prog = kProgResidual;
  I.in_psi = (const double2*)psi;
  I.use_phi = 2;
  double res[kNRec + 1] = {0};
  CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), (cudaStream_t)stream));
  rc = run_api(p, i, I, (cudaStream_t)stream, res);
  if (rc) return rc;
  const double mu = res[0];
  const double r = sqrt(res[1] * I.dv);
  out3[0] = r;
  out3[1] = mu;
  out3[2] = r / fmax(1.0, fabs(mu));
  return BGP_OK;
}

int bgp_convolve(bgp_plan* p, int i, const double* rho, double* out, int which, void* stream) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  Inst I = p->inst[i];
  if (I.M == 0) return fail(BGP_ERR_ARG, "instance has no long-range kernel");
  if (which == 1 && !I.Wq) return fail(BGP_ERR_ARG, "virial kernel exists for q2d only");
  if (!rho || !out) return fail(BGP_ERR_ARG, "null pointer");
  I.prog = kProgConv;
  I.in_phi = rho;
  I.out_r = out;
  I.which_w = which;
  double res[kNRec + 1] = {0};
  CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), (cudaStream_t)stream));
  return run_api(p, i, I, (cudaStream_t)stream, res);
}

int bgp_precondition(bgp_plan* p, int i, const void* grad, const void* psi, const double* phi,
                     double shift_min, void* z, double* sigma_out, void* stream) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  if (!grad || !psi || !z) return fail(BGP_ERR_ARG, "null pointer");
  Inst I = p->inst[i];
  I.prog = kProgPrecond;
  I.in_grad = (const double2*)grad;
  I.in_psi = (const double2*)psi;
  I.in_phi = phi;
  I.use_phi = phi ? 1 : 0;
  I.out_c = (double2*)z;
  I.sp.shift_min = shift_min;
  double res[kNRec + 1] = {0};
  CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), (cudaStream_t)stream));
  rc = run_api(p, i, I, (cudaStream_t)stream, res);
  if (rc) return rc;
  if (sigma_out) *sigma_out = res[0];
  return BGP_OK;
}

namespace {
// ------------------------------------------------------------ stream passes
void* stream_h_kernel(int N, int ln, int v) {
  switch (N) {
#define X(n) case n: return bgp_sptr_##n(ln, v);
    BGP_FOR_STREAM_N(X)
#undef X
    default: return nullptr;
  }
}
void* stream_conv_kernel(int M, int ln, int v) {
  switch (M) {
#define X(m) case m: return bgp_scptr_##m(ln, v);
    BGP_FOR_STREAM_M(X)
#undef X
    default: return nullptr;
  }
}

// per-instance total of the tiles' partial sums, in tile order: mu = sum dV
__global__ void k_stream_mu(SLaunch SL, int tiles, double* mu, int offset) {
  const int a = blockIdx.x;
  if (a >= SL.ninst) return;
  const SInst& I = SL.insts[a];
  double s = 0.0;
  for (int t = threadIdx.x; t < tiles; t += blockDim.x) s += I.part[t];
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) tot += red[q];
    mu[offset + a] = tot * I.dv;
  }
}

int stream_launch(void* kern, int tiles, int threads, size_t smem, SLaunch& SL, cudaStream_t st, void** args) {
  SL.tiles = tiles;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaLaunchKernel(kern, dim3(tiles * SL.ninst), dim3(threads), args, smem, st));
  return BGP_OK;
}

// The passes of one group (same N, ndim, kernel): optional convolution (phi from
// |psi|^2), then the H psi axis passes, then mu.
int stream_run(SLaunch& SL, int ln, int v, int cln, int csln, int cv, bool conv, double* mu_dev, int mu_off,
               cudaStream_t st, cudaStream_t side = nullptr, cudaEvent_t ev_fork = nullptr,
               cudaEvent_t ev_join = nullptr) {
  const SInst& I0 = SL.insts[0];
  const int N = I0.N, ndim = I0.ndim, n = I0.n;
  void* k = stream_h_kernel(N, ln, v);
  if (!k) return fail(BGP_ERR_UNSUPPORTED, "stream H psi pass not compiled for this size / schedule");
  const size_t smem = s_smem(N, ln);
  const int tiles = n / (N * ln);
  auto hstage = [&](int st_, cudaStream_t q) -> int {
    int ax = ndim - 1 - st_;
    int stage = (st_ == 0) ? 0 : (ax == 0 ? 2 : 1);
    void* args[] = {&SL, &ax, &stage};
    return stream_launch(k, tiles, ln * 32, smem, SL, q, args);
  };
  // with the potential computed and a side stream given, the H psi passes before the
  // last (which reads phi) run on the side stream beside the convolution: they write
  // only the accumulator, the convolution only its scratch and phi
  const bool overlap = conv && side && ev_fork && ev_join;
  if (overlap) {
    CK(cudaEventRecord(ev_fork, st));
    CK(cudaStreamWaitEvent(side, ev_fork, 0));
    for (int st_ = 0; st_ < ndim - 1; ++st_) {
      int rc = hstage(st_, side);
      if (rc) return rc;
    }
    CK(cudaEventRecord(ev_join, side));
  }
  if (conv) {
    const int M = I0.M, Mh = I0.Mh;
    // contiguous passes (ops 0, 5) in tiles of cln lines, strided passes in tiles
    // of csln lines (wider rows of the strided loads and stores)
    void* kc = stream_conv_kernel(M, cln, cv);
    void* ks = stream_conv_kernel(M, csln, cv);
    if (!kc || !ks) return fail(BGP_ERR_UNSUPPORTED, "stream convolution not compiled for this size");
    const int lines = ndim == 2 ? N : N * N, tpl = (Mh + csln - 1) / csln;
    const int ops2[3] = {0, 1, 5}, ops3[5] = {0, 2, 3, 4, 5};
    const int* ops = ndim == 2 ? ops2 : ops3;
    const int nops = ndim == 2 ? 3 : 5;
    for (int q = 0; q < nops; ++q) {
      int op = ops[q];
      const bool contig = (op == 0 || op == 5);
      const int lw = contig ? cln : csln;
      int ctiles;
      if (contig) ctiles = (lines + cln - 1) / cln;
      else if (op == 1) ctiles = tpl;
      else if (op == 3) ctiles = M * tpl;
      else ctiles = N * tpl;
      void* args[] = {&SL, &op};
      int rc = stream_launch(contig ? kc : ks, ctiles, lw * 32, s_conv_smem(M, lw), SL, st, args);
      if (rc) return rc;
    }
  }
  if (overlap) CK(cudaStreamWaitEvent(st, ev_join, 0));
  for (int st_ = overlap ? ndim - 1 : 0; st_ < ndim; ++st_) {
    int rc = hstage(st_, st);
    if (rc) return rc;
  }
  if (mu_dev) {
    k_stream_mu<<<SL.ninst, 256, 0, st>>>(SL, tiles, mu_dev, mu_off);
  }
  CK(cudaGetLastError());
  return BGP_OK;
}

// Time every compiled (lines, radix order) candidate of line length N on this
// group, then the convolution's lines per tile; keep the fastest (median of 3).
int stream_autotune(bgp_plan* p, bgp_plan::StreamSched& sc, SLaunch& SL, bool conv, cudaStream_t st) {
  const int N = SL.insts[0].N;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto timed = [&](int ln, int v, int cln, int csln, int cv, bool with_conv, float* ms) -> int {
    float t[3];
    int rc = stream_run(SL, ln, v, cln, csln, cv, with_conv, nullptr, 0, st);   // warm-up
    if (rc) return rc;
    for (int r = 0; r < 3; ++r) {
      CK(cudaEventRecord(e0, st));
      if ((rc = stream_run(SL, ln, v, cln, csln, cv, with_conv, nullptr, 0, st))) return rc;
      CK(cudaEventRecord(e1, st));
      CK(cudaEventSynchronize(e1));
      CK(cudaEventElapsedTime(&t[r], e0, e1));
    }
    std::sort(t, t + 3);
    *ms = t[1];
    return BGP_OK;
  };
  float best = 1e30f;
  sc.cand.clear();
  for (int ln : {1, 2, 4, 8, 16}) {
    for (int v = 0; v < 8; ++v) {
      if (!stream_h_kernel(N, ln, v)) continue;
      float ms = 0.f;
      int rc = timed(ln, v, 8, 8, 0, false, &ms);
      if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
      sc.cand.push_back({(float)ln, (float)v, 0.f, ms});
      if (ms < best) { best = ms; sc.ln = ln; sc.v = v; }
    }
  }
  if (conv) {
    float bc = 1e30f;
    for (int cln : {1, 2, 4, 8}) {
      for (int csln : {1, 2, 4, 8, 16}) {
        for (int cv : {0, 3}) {
          if (!stream_conv_kernel(SL.insts[0].M, cln, cv) || !stream_conv_kernel(SL.insts[0].M, csln, cv)) continue;
          float ms = 0.f;
          int rc = timed(sc.ln, sc.v, cln, csln, cv, true, &ms);
          if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
          // negative lines: a convolution candidate
          sc.cand.push_back({(float)(-cln), (float)cv, (float)csln, ms});
          if (ms < bc) { bc = ms; sc.cln = cln; sc.csln = csln; sc.cv = cv; }
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  sc.tuned = 1;
  (void)p;
  return BGP_OK;
}
}  // namespace

// H psi of several instances of a plan, enqueued without host synchronisation
int bgp_apply_H_batch(bgp_plan* p, int n, const int* idx, const void* const* psi, void* const* hpsi,
                      const double* const* phi, int phi_mode, double* mu_dev, void* stream) {
  if (!p || n < 1 || !idx || !psi || !hpsi) return fail(BGP_ERR_ARG, "bad arguments");
  if (phi_mode < 0 || phi_mode > 2) return fail(BGP_ERR_ARG, "phi_mode must be 0, 1 or 2");
  if (phi_mode == 1 && !phi) return fail(BGP_ERR_ARG, "phi_mode 1 needs phi");
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<int> seen(p->inst.size(), 0);
  for (int a = 0; a < n; ++a) {
    int rc = check_inst(p, idx[a]);
    if (rc) return rc;
    if (seen[idx[a]]++) return fail(BGP_ERR_ARG, "an instance appears twice in one batched apply");
    if (!psi[a] || !hpsi[a]) return fail(BGP_ERR_ARG, "null field pointer");
    if (psi[a] == hpsi[a]) return fail(BGP_ERR_ARG, "hpsi must not alias psi");
    if (phi_mode == 1 && !phi[a]) return fail(BGP_ERR_ARG, "phi_mode 1 needs phi for every instance");
  }
  // groups of equal (ndim, N, convolution on), in call order, at most kStreamBatch each;
  // the first runs on the caller's stream, each further one on a side stream that
  // waits for the work enqueued before the call and that the caller's stream waits for
  std::vector<char> done(n, 0);
  if (p->side_ev.empty()) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p->side_ev.push_back(e);
  }
  CK(cudaEventRecord(p->side_ev[0], st));   // the fork: the work enqueued before this call
  int ngroup = 0;
  for (int a = 0; a < n; ++a) {
    if (done[a]) continue;
    const int gi = ngroup++;
    const Inst& A0 = p->inst[idx[a]];
    const bool conv = phi_mode == 2 && A0.kind != kNone && A0.M > 0;
    std::vector<int> grp;
    for (int b = a; b < n && (int)grp.size() < kStreamBatch; ++b) {
      const Inst& B = p->inst[idx[b]];
      const bool cb = phi_mode == 2 && B.kind != kNone && B.M > 0;
      if (!done[b] && B.ndim == A0.ndim && B.N == A0.N && cb == conv && (!conv || B.M == A0.M)) {
        grp.push_back(b);
        done[b] = 1;
      }
    }
    SLaunch SL;
    memset(&SL, 0, sizeof(SL));
    SL.ninst = (int)grp.size();
    for (int g = 0; g < SL.ninst; ++g) {
      const int b = grp[g];
      const Inst& I = p->inst[idx[b]];
      SInst& S = SL.insts[g];
      S.ndim = I.ndim; S.N = I.N; S.n = I.n; S.M = I.M; S.Mh = I.Mh; S.i0 = I.i0;
      S.dx = I.dx; S.kfac = I.kfac; S.s = I.s; S.tc = I.tc; S.beta2 = I.beta2; S.beta3 = I.beta3;
      S.Omega = I.Omega; S.dv = I.dv;
      S.psi = (const double2*)psi[b];
      S.H = (double2*)hpsi[b];
      S.A = I.pool;                 // pool field 0 of the instance as the accumulator
      S.part = I.part;
      S.cb1 = I.cb1; S.cb2 = I.cb2; S.Kq = I.Kq; S.conv_scale = I.conv_scale;
      S.phi_out = I.phi2;           // computed potential: the instance's first potential field
      S.phi = conv ? I.phi2 : (phi_mode == 1 ? phi[b] : nullptr);
      if (I.kind == kNone || I.M == 0) S.phi = (phi_mode == 1) ? phi[b] : nullptr;
      S.twN = I.twN; S.twM = I.twM;
    }
    bgp_plan::StreamSched& sc = p->ssched[A0.N];
    if (sc.tuned == 0) {
      int rc = stream_autotune(p, sc, SL, conv, st);
      if (rc) return rc;
    }
    cudaStream_t gs = st;
    if (gi > 0) {
      while ((int)p->side_st.size() < gi) {
        cudaStream_t q;
        CK(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
        p->side_st.push_back(q);
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        p->side_ev.push_back(e);
      }
      gs = p->side_st[gi - 1];
      CK(cudaStreamWaitEvent(gs, p->side_ev[0], 0));
    }
    cudaStream_t os = nullptr;
    cudaEvent_t oe0 = nullptr, oe1 = nullptr;
    if (conv) {
      while ((int)p->ovl_st.size() <= gi) {
        cudaStream_t q;
        CK(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
        p->ovl_st.push_back(q);
        for (int e = 0; e < 2; ++e) {
          cudaEvent_t ev;
          CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
          p->ovl_ev.push_back(ev);
        }
      }
      os = p->ovl_st[gi]; oe0 = p->ovl_ev[2 * gi]; oe1 = p->ovl_ev[2 * gi + 1];
    }
    // mu of the group, written in call order
    int rc = BGP_OK;
    if (mu_dev) {
      // the mu kernel writes SL order; the group's members are consecutive in the
      // output only when the caller passed them so: write each one at its own index
      double* tmp = nullptr;
      if (!(grp.back() - grp.front() == (int)grp.size() - 1)) {
        CK(cudaMallocAsync((void**)&tmp, sizeof(double) * grp.size(), gs));
      }
      rc = stream_run(SL, sc.ln, sc.v, sc.cln, sc.csln, sc.cv, conv, tmp ? tmp : mu_dev, tmp ? 0 : grp.front(), gs,
                      os, oe0, oe1);
      if (!rc && tmp) {
        for (int g = 0; g < SL.ninst; ++g)
          CK(cudaMemcpyAsync(mu_dev + grp[g], tmp + g, sizeof(double), cudaMemcpyDeviceToDevice, gs));
      }
      if (tmp) cudaFreeAsync(tmp, gs);
    } else {
      rc = stream_run(SL, sc.ln, sc.v, sc.cln, sc.csln, sc.cv, conv, nullptr, 0, gs, os, oe0, oe1);
    }
    if (rc) return rc;
    if (gi > 0) CK(cudaEventRecord(p->side_ev[gi], gs));
    p->launches += conv ? (A0.ndim == 2 ? 3 : 5) + A0.ndim : A0.ndim;
  }
  // the join: the caller's stream waits for every side group
  for (int g = 1; g < ngroup; ++g) CK(cudaStreamWaitEvent(st, p->side_ev[g], 0));
  return BGP_OK;
}

int bgp_plan_stream_schedule(bgp_plan* p, int N, int* lines, int* radix_order, int* conv_lines,
                             int* conv_strided_lines, int* conv_order, int* tuned, float* cand, int* ncand) {
  if (!p) return fail(BGP_ERR_ARG, "null plan");
  auto it = p->ssched.find(N);
  const bgp_plan::StreamSched none;
  const bgp_plan::StreamSched& sc = it == p->ssched.end() ? none : it->second;
  if (lines) *lines = sc.ln;
  if (radix_order) *radix_order = sc.v;
  if (conv_lines) *conv_lines = sc.cln;
  if (conv_strided_lines) *conv_strided_lines = sc.csln;
  if (conv_order) *conv_order = sc.cv;
  if (tuned) *tuned = sc.tuned;
  if (ncand) {
    const int cap = *ncand;
    *ncand = (int)sc.cand.size();
    if (cand)
      for (int q = 0; q < (int)sc.cand.size() && q < cap; ++q)
        for (int c = 0; c < 4; ++c) cand[4 * q + c] = sc.cand[q][c];
  }
  return BGP_OK;
}

int bgp_plan_stream_set(bgp_plan* p, int N, int lines, int radix_order, int conv_lines, int conv_strided_lines,
                        int conv_order) {
  if (!p) return fail(BGP_ERR_ARG, "null plan");
  bgp_plan::StreamSched& sc = p->ssched[N];
  if (lines == 0) { sc.tuned = 0; sc.cand.clear(); return BGP_OK; }   // tune again on next use
  if (!stream_h_kernel(N, lines, radix_order)) return fail(BGP_ERR_UNSUPPORTED, "schedule not compiled for this N");
  if (conv_lines != 1 && conv_lines != 2 && conv_lines != 4 && conv_lines != 8)
    return fail(BGP_ERR_ARG, "contiguous convolution lines per tile: 1, 2, 4 or 8");
  if (conv_strided_lines != 1 && conv_strided_lines != 2 && conv_strided_lines != 4 && conv_strided_lines != 8 &&
      conv_strided_lines != 16)
    return fail(BGP_ERR_ARG, "strided convolution lines per tile: 1, 2, 4, 8 or 16");
  if (conv_order != 0 && conv_order != 3) return fail(BGP_ERR_ARG, "convolution radix order: 0 or 3");
  if (conv_order == 3 && (2 * N) % 32 != 0) return fail(BGP_ERR_UNSUPPORTED, "register transform needs 2N = 32 R");
  // where the convolution is compiled for this N, both of its tile widths must be
  if (stream_conv_kernel(2 * N, 4, 0) &&
      (!stream_conv_kernel(2 * N, conv_lines, conv_order) || !stream_conv_kernel(2 * N, conv_strided_lines, conv_order)))
    return fail(BGP_ERR_UNSUPPORTED, "convolution tile width not compiled for this N");
  sc.ln = lines; sc.v = radix_order; sc.cln = conv_lines; sc.csln = conv_strided_lines; sc.cv = conv_order;
  sc.tuned = 2;
  return BGP_OK;
}

namespace {
// Cooperative launch of a Thomas-Fermi kernel over `grid` CTAs (one team).
int tf_launch(void* kern, int grid, void** args, bgp_plan* p, const Inst& I, cudaStream_t st) {
  CK(cudaMemsetAsync(I.bar, 0, sizeof(unsigned long long), st));
  CK(cudaMemsetAsync(p->d_abort, 0, (4 + (size_t)grid) * sizeof(int), st));
  CK(cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kThreads), args, 0, st));
  CK(cudaGetLastError());
  p->launches++;
  return BGP_OK;
}
}  // namespace

int bgp_tf_density(bgp_plan* p, int i, int nonlocal, double Omega, int iters, double relax, double* n_out,
                   double* info, void* stream) {
  int rc = check_inst(p, i);
  if (rc) return rc;
  if (!n_out || !info) return fail(BGP_ERR_ARG, "null pointer");
  const Inst I = p->inst[i];
  if (nonlocal && (I.M == 0 || I.kind == kNone)) return fail(BGP_ERR_ARG, "nonlocal Thomas-Fermi needs a long-range kernel");
  if (iters < 1) return fail(BGP_ERR_ARG, "iters must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  // one team over the resident CTAs, at most the plan's grid (its partial-sum and
  // status buffers are sized for it)
  int nb = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_tf_iter, kThreads, 0));
  int grid = std::min(nb * p->dev->sms, p->grid_cap);
  if (grid < 1) return fail(BGP_ERR_CUDA, "Thomas-Fermi kernel does not fit on an SM");
  double* state = p->d_res + (size_t)i * (kNRec + 1);
  double* conv = I.phi2 + I.n;   // the plan's second potential field as the convolution output
  TfArgs A;
  memset(&A, 0, sizeof(A));
  A.ndim = I.ndim; A.N = I.N; A.n = I.n; A.mode = nonlocal ? 1 : 0;
  A.dx = I.dx; A.dv = I.dv; A.tc = I.tc; A.s = I.s; A.Omega = Omega;
  A.b2 = I.beta2; A.b3 = I.beta3; A.gc = I.G_C; A.relax = relax;
  A.conv = nonlocal ? conv : nullptr;
  A.nf = n_out; A.part = I.part; A.bar = I.bar; A.abort_flag = p->d_abort; A.state = state;
  double h[4] = {NAN, INFINITY, 0.0, 0.0};
  int done = 0;
  auto read_state = [&]() -> int {
    int ab = 0;
    CK(cudaMemcpyAsync(h, state, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&ab, p->d_abort, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ab != 0 || h[2] == (double)kTfBarrier) return fail(BGP_ERR_DEVICE, "Thomas-Fermi kernel: team barrier timeout");
    return BGP_OK;
  };
  CK(cudaMemcpyAsync(state, h, sizeof(h), cudaMemcpyHostToDevice, st));
  if (!nonlocal) {
    void* args[] = {&A};
    if ((rc = tf_launch((void*)k_tf_iter, grid, args, p, I, st))) return rc;
    if ((rc = read_state())) return rc;
    done = 1;
  } else {
    const double sigma = 0.15 * (I.dx * I.N / 2.0);   // 0.15 L
    double two_s2 = 2.0 * (sigma * sigma);
    void* sargs[] = {&A, &two_s2};
    if ((rc = tf_launch((void*)k_tf_seed, grid, sargs, p, I, st))) return rc;
    for (int it = 0; it < iters; ++it) {
      Inst J = I;
      J.prog = kProgConv;
      J.in_phi = n_out;
      J.out_r = conv;
      J.which_w = 0;
      double res[kNRec + 1] = {0};
      CK(cudaMemsetAsync(p->d_res + (size_t)i * (kNRec + 1), 0, sizeof(double) * (kNRec + 1), st));
      if ((rc = run_api(p, i, J, st, res))) return rc;
      void* args[] = {&A};
      if ((rc = tf_launch((void*)k_tf_iter, grid, args, p, I, st))) return rc;
      if ((rc = read_state())) return rc;
      done = it + 1;
      if (h[2] != (double)kTfOk || h[3] != 0.0) break;
    }
  }
  info[0] = (h[2] == (double)kTfNoBracket) ? NAN : h[0];   // mu
  info[1] = h[3];                                          // converged
  info[2] = h[1];                                          // final dn
  info[3] = (double)done;                                  // steps taken
  info[4] = h[2];                                          // status
  return BGP_OK;
}

int bgp_solve(bgp_plan* p, const void* const* psi0, void* const* psi_out, const bgp_solver_params* sp,
              bgp_solve_result* results, double* trace, void* stream) {
  if (!p || !psi0 || !psi_out || !sp || !results) return fail(BGP_ERR_ARG, "null pointer");
  static_assert(sizeof(SolveOut) == sizeof(bgp_solve_result), "result layout");
  const int n = (int)p->inst.size();
  cudaStream_t st = (cudaStream_t)stream;
  SolverParams P{};
  P.maxit = sp->maxit; P.ls_max = sp->linesearch_max; P.stall_max = sp->linesearch_stall < 1 ? 1 : sp->linesearch_stall;
  P.restart = sp->cg_restart; P.cg_beta = sp->cg_beta; P.window = sp->conv_window;
  P.record_trace = sp->record_trace; P.trace_cap = sp->trace_cap;
  P.res_tol = sp->res_tol; P.etol = sp->energy_tol; P.alpha0 = sp->step; P.alpha_min = 1e-8;
  P.alpha_max = sp->step_max; P.shift_min = sp->precond_shift_min; P.c1 = 1e-4; P.shrink = 0.5;
  P.growth = 1.1; P.bb_min = 0.05; P.bb_max = sp->step_max; P.bb_mix = 0.5;
  P.mixed = sp->mixed ? 1 : 0; P.mixed_tol = sp->mixed_switch_res;
  if (P.cg_beta < 0 || P.cg_beta > 2) return fail(BGP_ERR_ARG, "cg_beta must be 0, 1 or 2");
  if (P.maxit < 0) return fail(BGP_ERR_ARG, "maxit must be >= 0");
  double* d_trace = nullptr;
  if (P.record_trace && P.trace_cap > 0) {
    CK(cudaMallocAsync((void**)&d_trace, sizeof(double) * 3 * (size_t)P.trace_cap * n, st));
  } else {
    P.record_trace = 0;
  }
  std::vector<Inst> save = p->inst;
  std::vector<int> act(n);
  for (int i = 0; i < n; ++i) {
    if (!psi0[i] || !psi_out[i]) return fail(BGP_ERR_ARG, "null field pointer");
    Inst& I = p->inst[i];
    I.prog = kProgSolve;
    I.in_psi = (const double2*)psi0[i];
    I.out_c = (double2*)psi_out[i];
    I.sp = P;
    I.trace = d_trace ? d_trace + (size_t)3 * P.trace_cap * i : nullptr;
    I.resume = 0;
    I.finished = p->d_finished;
    act[i] = i;
  }
  CK(cudaMemsetAsync(p->d_out, 0, sizeof(SolveOut) * n, st));
  // Segmented solve: each launch runs until a quarter of its instances have
  // finished; the others save their state and are relaunched with larger teams,
  // so the instances that need the most iterations soon get the whole GPU.
  int rc = BGP_OK;
  std::vector<SolveOut> outs(n);
  const bool tuning = p->tune == 1 && n > 1;
  const int ydiv = tuning ? kTuneYield[p->tune_next] : p->yield_div;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (tuning) {
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    CK(cudaEventRecord(ev0, st));
  }
  for (int seg = 0; !act.empty() && seg < kMaxSegments; ++seg) {
    const int na = (int)act.size();
    const int yield_at = na > 1 ? std::max(1, na / ydiv) : (1 << 30);
    for (int a : act) p->inst[a].yield_at = yield_at;
    CK(cudaMemsetAsync(p->d_finished, 0, sizeof(int), st));
    rc = launch(p, act, st);
    if (rc) break;
    CK(cudaMemcpyAsync(outs.data(), p->d_out, sizeof(SolveOut) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<int> next;
    for (int a : act) {
      if (outs[a].status == 2) {
        next.push_back(a);
        p->inst[a].resume = 1;
        // handed over to FP64: later segments run in the smaller FP64-only kernels
        if (outs[a].fp64_from >= 0) p->inst[a].sp.mixed = 0;
      }
    }
    act.swap(next);
  }
  p->inst = save;
  if (tuning) {
    float ms = 0.f;
    if (!rc && act.empty()) {
      CK(cudaEventRecord(ev1, st));
      CK(cudaEventSynchronize(ev1));
      CK(cudaEventElapsedTime(&ms, ev0, ev1));
      p->tune_ms[p->tune_next++] = ms;
      if (p->tune_next == 3) {
        int best = 0;
        for (int c = 1; c < 3; ++c) if (p->tune_ms[c] < p->tune_ms[best]) best = c;
        p->yield_div = kTuneYield[best];
        p->tune = 2;
      }
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }
  if (!rc && !act.empty()) rc = fail(BGP_ERR_DEVICE, "solve did not finish within the relaunch limit");
  if (rc) { if (d_trace) cudaFreeAsync(d_trace, st); return rc; }
  CK(cudaMemcpyAsync(results, p->d_out, sizeof(SolveOut) * n, cudaMemcpyDeviceToHost, st));
  if (d_trace && trace)
    CK(cudaMemcpyAsync(trace, d_trace, sizeof(double) * 3 * (size_t)P.trace_cap * n, cudaMemcpyDeviceToHost, st));
  if (d_trace) CK(cudaFreeAsync(d_trace, st));
  CK(cudaStreamSynchronize(st));
  for (int i = 0; i < n; ++i)
    if (results[i].status != 0) return fail(BGP_ERR_DEVICE, "a solver team stopped on a device error");
  return BGP_OK;
}

}  // extern "C"
