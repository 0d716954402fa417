// Allocation-free Hamiltonian apply: bgp_apply_H_noalloc (include/bgp.h).
//
// Some callers cannot call cudaMalloc: a host framework that owns the whole
// device-memory budget and forbids its plugins to allocate, or a time-critical
// loop that cannot afford the device-wide synchronisation cudaMalloc implies.
// This entry point needs no plan and allocates nothing. Its only scratch (the
// partial kinetic/rotation field between the per-axis passes) and its twiddle
// table are file-scope device arrays of fixed size, which every GPU that loads
// the library holds until the process exits.
//
// Limits and behaviour:
//   - at most kNoAllocMaxPoints = 262144 grid points (2D up to 512^2, 3D up to
//     64^3); larger grids are rejected with BGP_ERR_ARG;
//   - the long-range potential is taken as given (phi, N^d real) or omitted
//     (phi = NULL); computing it would need the padded transform's scratch;
//   - every call shares both static arrays (the scratch field and the twiddle
//     table, which each call rewrites for its own N) and leaves the last call's
//     contents in them; calls that overlap on the GPU (different streams, or
//     threads without ordering) race on both and must be serialised by the
//     caller. Nothing has to start at zero: each call writes the whole scratch
//     field and the twiddles it uses before reading them.
//   - the first call on a device looks up the device addresses of the static
//     arrays (cudaGetSymbolAddress, with that device current); make that first
//     call before any stream capture on the device. The addresses are kept for
//     the lifetime of the device's primary context: after cudaDeviceReset the
//     process must not call this entry point again.
//   - errors pending from earlier, unrelated work are cleared on entry
//     (cudaGetLastError), so a launch error reported here is this call's own.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <mutex>
#include <string>

#include "../../include/bgp.h"
#include "bgp_passes.cuh"

using namespace bgp;

namespace {

constexpr int kNoAllocMaxPoints = 1 << 18;
constexpr int kNoAllocMaxLine = 512;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocMaxPoints];
static __device__ __align__(256) double2 g_noalloc_tw[kNoAllocMaxLine];

struct SymPtrs {
  int ready;
  double2* scratch;
  double2* tw;
};
SymPtrs g_sym[kMaxDevices];
std::mutex g_sym_mu;
}  // namespace

// error reporting shared with the other entry points (bgp_last_error)
int bgp_report_error(int code, const char* msg);

namespace {

int nfail(int code, const char* msg) { return bgp_report_error(code, msg); }

// Device addresses of the static arrays for the current device (looked up once).
int sym_ptrs(SymPtrs* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nfail(BGP_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return nfail(BGP_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_sym_mu);
  SymPtrs& s = g_sym[dev];
  if (!s.ready) {
    if (cudaGetSymbolAddress((void**)&s.scratch, g_noalloc_scratch) != cudaSuccess)
      return nfail(BGP_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed");
    if (cudaGetSymbolAddress((void**)&s.tw, g_noalloc_tw) != cudaSuccess)
      return nfail(BGP_ERR_CUDA, "cudaGetSymbolAddress(twiddles) failed");
    s.ready = 1;
  }
  *out = s;
  return BGP_OK;
}

// exp(-2 pi i t / N) from CUDA's sincospi
__global__ void k_noalloc_twiddles(double2* tw, int N) {
  for (int t = threadIdx.x + blockIdx.x * blockDim.x; t < N; t += blockDim.x * gridDim.x) {
    double s, c;
    sincospi(2.0 * (double)t / (double)N, &s, &c);
    tw[t] = cmk(c, -s);
  }
}

// One axis stage of H psi (the OpH pass) over every tile, one launch per stage.
template <int N>
__global__ void __launch_bounds__(kThreads) k_noalloc_hpsi(Inst I, PassArgs Q) {
  extern __shared__ double2 sm[];
  __shared__ Inst sI;
  __shared__ PassArgs sQ;
  if (threadIdx.x == 0) { sI = I; sQ = Q; }
  __syncthreads();
  OpH<N> op{sI, sQ};
  const int nt = ntiles_axis(sI);
  const bool contig = sQ.ax == sI.ndim - 1;
  for (int t = blockIdx.x; t < nt; t += gridDim.x) {
    if (contig) tile_run<N, true>(op, sm, t);
    else tile_run<N, false>(op, sm, t);
  }
}

template <int N>
int run_stages(Inst& I, PassArgs& Q, cudaStream_t st) {
  const size_t smem = tile_smem_bytes(N);
  if (cudaFuncSetAttribute(k_noalloc_hpsi<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return nfail(BGP_ERR_CUDA, "cudaFuncSetAttribute failed");
  const int nt = ntiles_axis(I);
  for (int st_ = 0; st_ < I.ndim; ++st_) {
    Q.ax = I.ndim - 1 - st_;
    Q.stage = (st_ == 0) ? 0 : (Q.ax == 0 ? 2 : 1);
    k_noalloc_hpsi<N><<<nt, kThreads, smem, st>>>(I, Q);
  }
  if (cudaGetLastError() != cudaSuccess) return nfail(BGP_ERR_CUDA, "launch failed");
  return BGP_OK;
}

}  // namespace

extern "C" {

// H psi for one instance without a plan and without any device allocation.
// psi, hpsi: device complex128 fields of N^d points (hpsi must not alias psi);
// phi: device real potential of N^d points or NULL. Enqueued on `stream`;
// returns without waiting for the result.
int bgp_apply_H_noalloc(const bgp_instance_desc* d, const void* psi, void* hpsi, const double* phi,
                        void* stream) {
  if (!d || !psi || !hpsi) return nfail(BGP_ERR_ARG, "null argument");
  if (psi == hpsi) return nfail(BGP_ERR_ARG, "hpsi must not alias psi");
  if (d->ndim != 2 && d->ndim != 3) return nfail(BGP_ERR_ARG, "ndim must be 2 or 3");
  if (!(d->L > 0)) return nfail(BGP_ERR_ARG, "L must be positive");
  const long long n = d->ndim == 2 ? (long long)d->N * d->N : (long long)d->N * d->N * d->N;
  if (d->N > kNoAllocMaxLine || n > kNoAllocMaxPoints)
    return nfail(BGP_ERR_ARG, "grid too large for bgp_apply_H_noalloc: at most 262144 points "
                              "(2D up to 512^2, 3D up to 64^3) and 512 points per axis");
  switch (d->N) {
    case 16: case 24: case 32: case 48: case 64: case 96: case 128: case 192: case 256: case 384:
    case 512: break;
    default: return nfail(BGP_ERR_UNSUPPORTED, "grid size not compiled in for bgp_apply_H_noalloc");
  }
  (void)cudaGetLastError();   // attribute only this call's launch errors to it
  SymPtrs sp;
  int rc = sym_ptrs(&sp);
  if (rc) return rc;
  Inst I;
  memset(&I, 0, sizeof(I));
  I.ndim = d->ndim; I.N = d->N; I.n = (int)n; I.kind = kNone;
  I.dx = 2.0 * d->L / d->N;
  I.dv = d->ndim == 2 ? I.dx * I.dx : I.dx * I.dx * I.dx;
  I.kfac = 1.0 / (d->N * I.dx);
  I.s = d->s; I.tc = d->trap_coeff;
  I.beta2 = d->beta2; I.beta3 = d->beta3; I.Omega = d->Omega; I.G_C = d->G_C;
  I.inv_n = 1.0 / (double)n;
  I.twN = sp.tw;
  PassArgs Q;
  memset(&Q, 0, sizeof(Q));
  Q.psi = (const double2*)psi; Q.psc = 1.0;
  Q.A = sp.scratch; Q.H = (double2*)hpsi;
  Q.phi = phi; Q.phisc = 1.0;
  cudaStream_t st = (cudaStream_t)stream;
  k_noalloc_twiddles<<<1, 256, 0, st>>>(sp.tw, d->N);
  switch (d->N) {
#define X(nn) case nn: return run_stages<nn>(I, Q, st);
    X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512)
#undef X
    default: return nfail(BGP_ERR_UNSUPPORTED, "grid size not compiled in for bgp_apply_H_noalloc");
  }
}

}  // extern "C"
