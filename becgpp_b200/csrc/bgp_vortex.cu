// Vortex count and lowest-Landau-level weight of a 2D field on the device
// (becgpp/vortex.py:10-84; a 3D state passes its z = 0 midplane as an N x N field).
//
// Vortex count (vortex.py:10-48). A vortex is a plaquette (i, j)-(i+1, j)-
// (i+1, j+1)-(i, j+1) whose wrapped phase increments sum to +-2 pi, counted when
// the plaquette lies inside the droplet: the mean of the smoothed density at its
// four corners above `thresh_frac` of the smoothed maximum and its first corner
// within R, the radius around the centre of mass that holds 99 % of the mass
// (the device centre of mass and mass-quantile radius of bgp_diag.cu). The
// reference smooths |psi|^2 with the Gaussian multiplier exp(-ell^2 k^2 / 2) of
// its periodic FFT; that multiplier is a product over the axes, so the smoothing
// is the separable periodic convolution with h = the inverse DFT of
// exp(-ell^2 k^2 / 2) along one axis (real and even, computed on the host in long
// double), done here as two direct passes. Counts are integer atomics (exact).
//
// LLL weight (vortex.py:61-84): sum over m <= mcap of |<phi_m, psi>|^2 with
// phi_m ~ r^m exp(-r^2/2) e^(i m theta) (theta negated for Omega < 0), each phi_m
// normalised on the grid. The per-point terms (log r, r^2/2, theta, psi / |psi|)
// are formed once; every m is a grid reduction of |phi_m|^2 and conj(phi_m) psi,
// in fixed-size CTA partials added in CTA order (deterministic).
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/bgp.h"

int bgp_report_error(int code, const char* msg);

namespace {

constexpr int kBlocks = 296;
constexpr int kThreads = 256;
constexpr double kPi = 3.14159265358979323846;

int vfail(int code, const std::string& msg) { return bgp_report_error(code, msg.c_str()); }
#define VCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return vfail(BGP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
// the same inside an entry point that holds scratch: free it (cleanup()) first
#define VCKF(call)                                                                    \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      cleanup();                                                                      \
      return vfail(BGP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    }                                                                                 \
  } while (0)

__device__ __forceinline__ double xcoord(int i, int N, double dx) { return (double)(i - N / 2) * dx; }

__global__ void k_abs2(const double2* __restrict__ psi, int n, double* rho) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
    const double2 p = psi[f];
    rho[f] = p.x * p.x + p.y * p.y;
  }
}

// out[i, j] = sum_b h[b] in[i, (j - b) mod N]  (axis 1), or over i (axis 0)
__global__ void k_periodic_conv(const double* __restrict__ in, const double* __restrict__ h, int N, int axis,
                                int clamp0, double* __restrict__ out) {
  const int n = N * N;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
    const int i = f / N, j = f - i * N;
    double s = 0.0;
    if (axis == 1) {
      for (int b = 0; b < N; ++b) {
        int jj = j - b;
        if (jj < 0) jj += N;
        s += __ldg(h + b) * __ldg(in + i * N + jj);
      }
    } else {
      for (int a = 0; a < N; ++a) {
        int ii = i - a;
        if (ii < 0) ii += N;
        s += __ldg(h + a) * __ldg(in + ii * N + j);
      }
    }
    out[f] = clamp0 ? fmax(s, 0.0) : s;
  }
}

__global__ void k_max_part(const double* __restrict__ v, int n, double* part) {
  __shared__ double sm[kThreads];
  double m = 0.0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) m = fmax(m, v[f]);
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

// phase difference folded into [-pi, pi): d + pi - 2 pi floor((d + pi) / 2 pi) - pi
__device__ __forceinline__ double wrap(double d) {
  const double a = d + kPi;
  return (a - 2.0 * kPi * floor(a / (2.0 * kPi))) - kPi;
}

struct PlaqArgs {
  int N;
  double dx, xc, yc, R, thr;
};

__global__ void k_plaquettes(const double2* __restrict__ psi, const double* __restrict__ smooth,
                             const double* __restrict__ smax_part, int nparts, PlaqArgs a, int* counts) {
  const int N = a.N, m = N - 1;
  double smax = 0.0;
  for (int q = 0; q < nparts; ++q) smax = fmax(smax, smax_part[q]);
  const double thr = a.thr * smax;
  int np = 0, nm = 0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m * m; f += gridDim.x * blockDim.x) {
    const int i = f / m, j = f - i * m;
    const int c0 = i * N + j, c1 = (i + 1) * N + j, c2 = (i + 1) * N + j + 1, c3 = i * N + j + 1;
    const double t0 = atan2(psi[c0].y, psi[c0].x), t1 = atan2(psi[c1].y, psi[c1].x);
    const double t2 = atan2(psi[c2].y, psi[c2].x), t3 = atan2(psi[c3].y, psi[c3].x);
    double tot = wrap(t1 - t0);
    tot = tot + wrap(t2 - t1);
    tot = tot + wrap(t3 - t2);
    tot = tot + wrap(t0 - t3);
    const double w = rint(tot / (2.0 * kPi));
    const double cell = 0.25 * (((smooth[c0] + smooth[c1]) + smooth[c2]) + smooth[c3]);
    const double dxr = __dsub_rn(xcoord(i, N, a.dx), a.xc), dyr = __dsub_rn(xcoord(j, N, a.dx), a.yc);
    const double r = sqrt(__dadd_rn(__dmul_rn(dxr, dxr), __dmul_rn(dyr, dyr)));
    if (cell > thr && r < a.R) {
      if (w >= 1.0) ++np;
      else if (w <= -1.0) ++nm;
    }
  }
  if (np) atomicAdd(counts, np);
  if (nm) atomicAdd(counts + 1, nm);
}

// ---------------------------------------------------------------- LLL weight
// per point: sums of |psi|^2 and r^2 |psi|^2 (CTA partials)
__global__ void k_lll_moments(const double2* __restrict__ psi, int N, double dx, double* part) {
  __shared__ double s0[kThreads], s1[kThreads];
  const int n = N * N;
  double a = 0.0, b = 0.0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
    const int i = f / N, j = f - i * N;
    const double x = xcoord(i, N, dx), y = xcoord(j, N, dx);
    const double2 p = psi[f];
    const double q = p.x * p.x + p.y * p.y;
    a += q;
    b += (x * x + y * y) * q;
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) { s0[threadIdx.x] += s0[threadIdx.x + o]; s1[threadIdx.x] += s1[threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = s0[0]; part[2 * blockIdx.x + 1] = s1[0]; }
}

struct LllPoint {
  double logr, hr2, theta, pr, pi;
};

__global__ void k_lll_points(const double2* __restrict__ psi, int N, double dx, double inv_norm, double sgn,
                             LllPoint* pts) {
  const int n = N * N;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
    const int i = f / N, j = f - i * N;
    const double x = xcoord(i, N, dx), y = xcoord(j, N, dx);
    const double r2 = x * x + y * y;
    LllPoint P;
    P.logr = log(fmax(sqrt(r2), 1e-300));
    P.hr2 = 0.5 * r2;
    P.theta = atan2(y, x) * sgn;
    P.pr = psi[f].x * inv_norm;
    P.pi = psi[f].y * inv_norm;
    pts[f] = P;
  }
}

// for m = 0 .. mcap: CTA partials of sum |phi_m|^2, Re and Im of sum conj(phi_m) psi
__global__ void k_lll_overlaps(const LllPoint* __restrict__ pts, int n, int mcap, double* part) {
  __shared__ double s[3][kThreads];
  const double lpi = log(kPi);
  for (int m = 0; m <= mcap; ++m) {
    const double cm = (m == 0) ? 0.0 : 0.5 * (lpi + lgamma(m + 1.0));
    double a = 0.0, b = 0.0, c = 0.0;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
      const LllPoint P = pts[f];
      const double amp = (m == 0) ? exp(-P.hr2) / sqrt(kPi) : exp(m * P.logr - P.hr2 - cm);
      double sn, cs;
      sincos(m * P.theta, &sn, &cs);
      const double br = amp * cs, bi = amp * sn;
      a += br * br + bi * bi;
      b += br * P.pr + bi * P.pi;     // Re conj(phi) psi
      c += br * P.pi - bi * P.pr;     // Im conj(phi) psi
    }
    s[0][threadIdx.x] = a;
    s[1][threadIdx.x] = b;
    s[2][threadIdx.x] = c;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o)
        for (int q = 0; q < 3; ++q) s[q][threadIdx.x] += s[q][threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0)
      for (int q = 0; q < 3; ++q) part[((size_t)m * 3 + q) * gridDim.x + blockIdx.x] = s[q][0];
    __syncthreads();
  }
}

// totals of the partials in CTA order: one thread per (m, quantity)
__global__ void k_sum_parts(const double* __restrict__ part, int rows, int cols, double* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  double s = 0.0;
  for (int q = 0; q < cols; ++q) s += part[(size_t)r * cols + q];
  out[r] = s;
}

template <class T>
int dalloc(T** p, size_t count, cudaStream_t st) {
  VCK(cudaMallocAsync((void**)p, count * sizeof(T), st));
  return BGP_OK;
}

}  // namespace

extern "C" {

int bgp_vortex_count(int N, double L, const void* psi, double Omega, double thresh_frac, int* out,
                     void* stream) {
  if (N < 2 || !(L > 0.0) || !psi || !out) return vfail(BGP_ERR_ARG, "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = N * N;
  const double dx = 2.0 * L / N;
  for (int q = 0; q < 4; ++q) out[q] = 0;
  double *rho = nullptr, *tmp = nullptr, *sm = nullptr, *h = nullptr, *part = nullptr;
  int* cnt = nullptr;
  int rc = BGP_OK;
  auto cleanup = [&]() {
    cudaFreeAsync(rho, st); cudaFreeAsync(tmp, st); cudaFreeAsync(sm, st);
    cudaFreeAsync(h, st); cudaFreeAsync(part, st); cudaFreeAsync(cnt, st);
  };
  if ((rc = dalloc(&rho, n, st)) || (rc = dalloc(&tmp, n, st)) || (rc = dalloc(&sm, n, st)) ||
      (rc = dalloc(&h, N, st)) || (rc = dalloc(&part, kBlocks, st)) || (rc = dalloc(&cnt, 2, st))) {
    cleanup();
    return rc;
  }
  k_abs2<<<kBlocks, kThreads, 0, st>>>((const double2*)psi, n, rho);
  double mass = 0.0, c[3] = {0.0, 0.0, 0.0}, R = 0.0;
  rc = bgp_density_center(2, N, L, rho, &mass, c, stream);
  if (!rc && mass > 0.0) {
    const double f99 = 0.99;
    rc = bgp_mass_quantiles(2, N, L, rho, c, &f99, 1, &R, stream);
  }
  if (rc || !(mass > 0.0) || !std::isfinite(R) || R <= 0.0) {
    cleanup();
    return rc;
  }
  // smoothing length and the periodic kernel h = IDFT of exp(-ell^2 k^2 / 2)
  const double ell = std::min(2.0 * std::sqrt(kPi / std::max(std::fabs(Omega), 1e-9)), std::max(R / 3.0, 2.0 * dx));
  std::vector<double> hh(N);
  {
    const long double two_pi = 6.283185307179586476925286766559L;
    std::vector<long double> g(N);
    for (int q = 0; q < N; ++q) {
      const int fq = (q < (N + 1) / 2) ? q : q - N;          // fftfreq order
      const long double k = two_pi * (long double)fq / ((long double)N * (long double)dx);
      g[q] = expl(-0.5L * (long double)ell * (long double)ell * k * k);
    }
    for (int b = 0; b < N; ++b) {
      long double s = 0.0L;
      for (int q = 0; q < N; ++q) s += g[q] * cosl(two_pi * (long double)(((long long)q * b) % N) / (long double)N);
      hh[b] = (double)(s / (long double)N);
    }
  }
  VCKF(cudaMemcpyAsync(h, hh.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
  k_periodic_conv<<<kBlocks, kThreads, 0, st>>>(rho, h, N, 1, 0, tmp);
  k_periodic_conv<<<kBlocks, kThreads, 0, st>>>(tmp, h, N, 0, 1, sm);
  k_max_part<<<kBlocks, kThreads, 0, st>>>(sm, n, part);
  VCKF(cudaMemsetAsync(cnt, 0, 2 * sizeof(int), st));
  PlaqArgs a{N, dx, c[0], c[1], R, thresh_frac};
  k_plaquettes<<<kBlocks, kThreads, 0, st>>>((const double2*)psi, sm, part, kBlocks, a, cnt);
  VCKF(cudaGetLastError());
  int hc[2] = {0, 0};
  VCKF(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
  VCKF(cudaStreamSynchronize(st));
  cleanup();
  out[0] = hc[0] + hc[1];
  out[1] = hc[0];
  out[2] = hc[1];
  out[3] = hc[0] - hc[1];
  return BGP_OK;
}

int bgp_lll_weight(int N, double L, const void* psi, double Omega, int Mmax, double* out, void* stream) {
  if (N < 2 || !(L > 0.0) || !psi || !out || Mmax < 0) return vfail(BGP_ERR_ARG, "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = N * N;
  const double dx = 2.0 * L / N, dv = dx * dx;
  double *part = nullptr, *tot = nullptr;
  LllPoint* pts = nullptr;
  int rc = BGP_OK;
  auto cleanup = [&]() { cudaFreeAsync(part, st); cudaFreeAsync(tot, st); cudaFreeAsync(pts, st); };
  if ((rc = dalloc(&part, 2 * (size_t)kBlocks, st))) {
    cleanup();
    return rc;
  }
  k_lll_moments<<<kBlocks, kThreads, 0, st>>>((const double2*)psi, N, dx, part);
  // the CTA partials (2 per CTA) are added in CTA order on the host
  std::vector<double> hp(2 * (size_t)kBlocks);
  VCKF(cudaMemcpyAsync(hp.data(), part, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st));
  VCKF(cudaStreamSynchronize(st));
  double s0 = 0.0, s1 = 0.0;
  for (int b = 0; b < kBlocks; ++b) { s0 += hp[2 * b]; s1 += hp[2 * b + 1]; }
  const double norm = std::sqrt(s0 * dv);
  if (!(norm > 0.0)) {
    cleanup();
    *out = 0.0;
    return BGP_OK;
  }
  const double r2mean = s1 * dv / (norm * norm);
  const int want = (int)std::ceil(r2mean + 10.0 * std::sqrt(std::max(r2mean, 1.0)) + 30.0);
  const int mcap = std::min(std::max(Mmax, want), std::max(Mmax, (int)((0.80 * L) * (0.80 * L))));
  cudaFreeAsync(part, st);
  part = nullptr;
  if ((rc = dalloc(&pts, n, st)) || (rc = dalloc(&part, 3 * (size_t)(mcap + 1) * kBlocks, st)) ||
      (rc = dalloc(&tot, 3 * (size_t)(mcap + 1), st))) {
    cleanup();
    return rc;
  }
  k_lll_points<<<kBlocks, kThreads, 0, st>>>((const double2*)psi, N, dx, 1.0 / norm, Omega >= 0.0 ? 1.0 : -1.0, pts);
  k_lll_overlaps<<<kBlocks, kThreads, 0, st>>>(pts, n, mcap, part);
  const int rows = 3 * (mcap + 1);
  k_sum_parts<<<(rows + 127) / 128, 128, 0, st>>>(part, rows, kBlocks, tot);
  VCKF(cudaGetLastError());
  std::vector<double> ht(rows);
  VCKF(cudaMemcpyAsync(ht.data(), tot, sizeof(double) * rows, cudaMemcpyDeviceToHost, st));
  VCKF(cudaStreamSynchronize(st));
  cleanup();
  double total = 0.0;
  for (int m = 0; m <= mcap; ++m) {
    const double a = ht[3 * m], re = ht[3 * m + 1], im = ht[3 * m + 2];
    if (a > 0.0) total += (re * re + im * im) * dv / a;
  }
  *out = std::min(std::max(total, 0.0), 1.0);
  return BGP_OK;
}

}  // extern "C"
