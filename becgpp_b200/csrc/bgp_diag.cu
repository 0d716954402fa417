// Density diagnostics on the device: centre of mass, mass-quantile radii and
// radial profiles of a real field on the grid (becgpp/fields.py:9-66).
//
// Mass quantile radius (becgpp/fields.py:17-30). The reference sorts every point
// by its distance r from the centre, accumulates w = max(rho, 0) dV in that order
// and returns the distance of the first point whose running mass reaches f times
// the total. Here no sort of the whole grid is needed: the distances, as IEEE
// doubles >= 0, order like their 64-bit patterns, so the wanted point is found by
// radix selection on those bits. Each level histograms 13 bits of the key (8192
// bins) of the points whose higher bits match the prefix chosen so far, weighting
// each point by its mass in 2^-58 fixed point (integer sums: exact and independent
// of the summation order); the bin where the running mass reaches the target is
// kept, until it holds at most kCandCap points, which one CTA sorts and scans.
// A point's mass moves by at most 2^-59 of the total in fixed point, so the chosen
// point can differ from the reference's only where its running mass meets the
// target within that margin. At f = 1 this reaches the last point that carries
// any mass; the reference's floating running sum stops changing earlier, once
// the mass left is below half an ulp of the total, so its f = 1 radius is set
// by its rounding (fractions below 1 do not depend on it).
//
// Radial profile (becgpp/fields.py:37-57): mean of a field over the shells
// [edges[b], edges[b+1]) (the last shell also takes everything beyond), NaN for
// empty shells. Bin sums are deterministic: a warp groups its lanes by bin and
// the group's values are added in lane order by the group's first lane, warps
// and CTAs then add up in their order.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/bgp.h"

int bgp_report_error(int code, const char* msg);

namespace {

constexpr int kDigits = 13;
constexpr int kBins = 1 << kDigits;        // histogram bins per level
constexpr int kCandCap = 8192;             // points one CTA finishes by sorting
constexpr int kRedBlocks = 296;            // CTAs of the reduction passes (fixed: deterministic sums)
constexpr int kRedThreads = 256;
constexpr double kFix = 288230376151711744.0;   // 2^58

int dfail(int code, const std::string& msg) { return bgp_report_error(code, msg.c_str()); }
#define DCK(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) return dfail(BGP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct Grid {
  int ndim, N, n;
  double dx, dv;
  double c[3];     // centre
};

__device__ __forceinline__ void coords(const Grid& g, int f, double* x) {
  const int N = g.N;
  int i, j, k = 0;
  if (g.ndim == 2) { i = f / N; j = f - i * N; }
  else { i = f / (N * N); const int r = f - i * N * N; j = r / N; k = r - j * N; }
  x[0] = (double)(i - N / 2) * g.dx;
  x[1] = (double)(j - N / 2) * g.dx;
  x[2] = (double)(k - N / 2) * g.dx;
}

// distance from the centre, summed as (x - cx)^2 + (y - cy)^2 [+ (z - cz)^2] without FMAs
__device__ __forceinline__ double radius_at(const Grid& g, int f) {
  double x[3];
  coords(g, f, x);
  double r2 = 0.0;
  for (int a = 0; a < g.ndim; ++a) {
    const double d = __dsub_rn(x[a], g.c[a]);
    r2 = __dadd_rn(r2, __dmul_rn(d, d));
  }
  return sqrt(r2);
}

__device__ __forceinline__ uint64_t rkey(double r) { return (uint64_t)__double_as_longlong(r); }

// block sum of NV doubles in a fixed tree; result in thread 0
template <int NV>
__device__ void block_sum_fixed(double (&v)[NV], double* sm) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sm[q * 32 + w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int k = 0; k < nw; ++k) s += sm[q * 32 + k];
      v[q] = s;
    }
  }
  __syncthreads();
}

// partial moments per CTA: sum rho, sum x_a rho (a < ndim), sum max(rho, 0)
__global__ void k_moments(const double* rho, Grid g, double* part) {
  __shared__ double sm[5 * 32];
  double v[5] = {0, 0, 0, 0, 0};
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n; f += gridDim.x * blockDim.x) {
    const double r = rho[f];
    double x[3];
    coords(g, f, x);
    v[0] += r;
    for (int a = 0; a < g.ndim; ++a) v[1 + a] += x[a] * r;
    v[4] += r > 0.0 ? r : 0.0;
  }
  block_sum_fixed<5>(v, sm);
  if (threadIdx.x == 0)
    for (int q = 0; q < 5; ++q) part[q * gridDim.x + blockIdx.x] = v[q];
}

// totals of the partials in CTA order: out[0..4]
__global__ void k_moments_total(const double* part, int blocks, double* out) {
  __shared__ double sm[5 * 32];
  double v[5] = {0, 0, 0, 0, 0};
  // thread t adds partials t, t + blockDim, ... in order, then the fixed tree
  for (int q = 0; q < 5; ++q)
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) v[q] += part[q * blocks + b];
  block_sum_fixed<5>(v, sm);
  if (threadIdx.x == 0) for (int q = 0; q < 5; ++q) out[q] = v[q];
}

// one selection level: histogram (mass and count) of the key digit at `dshift` over the
// points whose key >> pshift equals prefix (pshift = 64: every point)
__global__ void k_mq_hist(const double* rho, Grid g, double scale, uint64_t prefix, int pshift, int dshift,
                          int width, unsigned long long* hw, unsigned* hc) {
  extern __shared__ unsigned long long shw[];
  unsigned* shc = reinterpret_cast<unsigned*>(shw + kBins);
  for (int b = threadIdx.x; b < kBins; b += blockDim.x) { shw[b] = 0ull; shc[b] = 0u; }
  __syncthreads();
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n; f += gridDim.x * blockDim.x) {
    const uint64_t key = rkey(radius_at(g, f));
    if (pshift < 64 && (key >> pshift) != prefix) continue;
    const double r = rho[f];
    const double w = (r > 0.0 ? r : 0.0) * g.dv;
    const unsigned long long q = (unsigned long long)llrint(w * scale);
    const int d = (int)((key >> dshift) & ((1ull << width) - 1ull));
    if (q) atomicAdd(&shw[d], q);
    atomicAdd(&shc[d], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kBins; b += blockDim.x) {
    if (shw[b]) atomicAdd(&hw[b], shw[b]);
    if (shc[b]) atomicAdd(&hc[b], shc[b]);
  }
}

// State of one quantile's selection (device, one per fraction).
struct Sel {
  unsigned long long target, before, total;
  unsigned long long prefix;   // key bits chosen so far (right-aligned)
  unsigned count;              // points in the chosen bin
  int found;                   // 1: a bin was chosen
};

// ceil(f * tot) exactly (128-bit product of f's 53-bit mantissa and tot); f >= 1
// gives tot, f <= 0 gives 0.
__device__ unsigned long long frac_of_total(double f, unsigned long long tot) {
  if (!(f > 0.0)) return 0ull;
  if (f >= 1.0) return tot;
  int ex;
  const double mant = frexp(f, &ex);                              // f = mant 2^ex, ex <= 0
  const unsigned long long m = (unsigned long long)ldexp(mant, 53);   // exact 53-bit integer
  const int sh = 53 - ex;                                         // f = m 2^-sh, sh >= 53
  const unsigned long long lo = m * tot, hi = __umul64hi(m, tot);
  if (sh >= 128) return (hi | lo) ? 1ull : 0ull;
  unsigned long long q, rem;
  if (sh >= 64) {
    q = (sh == 64) ? hi : (hi >> (sh - 64));
    rem = lo | ((sh > 64) ? (hi & ((1ull << (sh - 64)) - 1ull)) : 0ull);
  } else {
    q = (hi << (64 - sh)) | (lo >> sh);
    rem = lo & ((1ull << sh) - 1ull);
  }
  return q + (rem ? 1ull : 0ull);
}

// Pick the first bin whose running mass (from `before`) reaches the target; at the
// first level the total sets the target ceil(f * total).
__global__ void k_mq_pick(const unsigned long long* hw, const unsigned* hc, Sel* s, double frac, int first_level,
                          int width) {
  __shared__ unsigned long long part[1024];
  const int t = threadIdx.x, per = kBins / blockDim.x;
  unsigned long long loc = 0;
  for (int q = 0; q < per; ++q) loc += hw[t * per + q];
  part[t] = loc;
  __syncthreads();
  if (t == 0) {
    if (first_level) {
      unsigned long long tot = 0;
      for (int k = 0; k < (int)blockDim.x; ++k) tot += part[k];
      s->total = tot;
      s->before = 0;
      s->target = frac_of_total(frac, tot);
    }
    // the chunk holding the crossing, then the bin inside it
    unsigned long long run = s->before;
    int chunk = -1;
    for (int k = 0; k < (int)blockDim.x; ++k) {
      bool any = false;
      for (int q = 0; q < per; ++q) any = any || hc[k * per + q] != 0u;
      if (any && run + part[k] >= s->target) { chunk = k; break; }
      run += part[k];
    }
    s->found = 0;
    if (chunk >= 0) {
      for (int q = 0; q < per; ++q) {
        const int b = chunk * per + q;
        if (hc[b] != 0u && run + hw[b] >= s->target) {
          s->prefix = (s->prefix << width) | (unsigned long long)b;
          s->before = run;
          s->count = hc[b];
          s->found = 1;
          break;
        }
        run += hw[b];
      }
    }
  }
}

// gather the points of the chosen bin (key >> shift == prefix)
__global__ void k_mq_collect(const double* rho, Grid g, double scale, uint64_t prefix, int shift,
                             unsigned long long* ckey, unsigned long long* cw, unsigned* ccount) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n; f += gridDim.x * blockDim.x) {
    const uint64_t key = rkey(radius_at(g, f));
    if ((key >> shift) != prefix) continue;
    const double r = rho[f];
    const double w = (r > 0.0 ? r : 0.0) * g.dv;
    const unsigned idx = atomicAdd(ccount, 1u);
    if (idx < (unsigned)kCandCap) { ckey[idx] = key; cw[idx] = (unsigned long long)llrint(w * scale); }
  }
}

// sort the candidates by key (bitonic, in shared memory), scan their masses from
// `before` and return the distance of the first that reaches the target
__global__ void k_mq_finish(const unsigned long long* ckey, const unsigned long long* cw, const unsigned* ccount,
                            const Sel* s, double* out) {
  extern __shared__ unsigned long long sk[];
  unsigned long long* sw = sk + kCandCap;
  const int n = (int)min(*ccount, (unsigned)kCandCap);
  int P = 1;
  while (P < n) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    sk[i] = i < n ? ckey[i] : ~0ull;
    sw[i] = i < n ? cw[i] : 0ull;
  }
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const unsigned long long a = sk[i], b = sk[l];
          const bool swap = up ? (a > b || (a == b && sw[i] > sw[l])) : (a < b || (a == b && sw[i] < sw[l]));
          if (swap) {
            sk[i] = b; sk[l] = a;
            const unsigned long long t = sw[i]; sw[i] = sw[l]; sw[l] = t;
          }
        }
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    unsigned long long run = s->before;
    double r = NAN;
    for (int i = 0; i < n; ++i) {
      run += sw[i];
      if (run >= s->target) { r = __longlong_as_double((long long)sk[i]); break; }
    }
    if (isnan(r) && n > 0) r = __longlong_as_double((long long)sk[n - 1]);
    *out = r;
  }
}

// largest distance over the grid (fractions above 1 clamp to the last point)
__global__ void k_max_radius(Grid g, double* part) {
  __shared__ double sm[32];
  double m = 0.0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n; f += gridDim.x * blockDim.x)
    m = fmax(m, radius_at(g, f));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) m = fmax(m, sm[k]);
    m = fmax(m, sm[0]);
    part[blockIdx.x] = m;
  }
}

// radial profile: per-CTA bin sums and counts (deterministic, see the file comment)
__global__ void k_profile(const double* fld, Grid g, const double* edges, int bins, double* psum,
                          unsigned* pcnt) {
  extern __shared__ double ssum[];     // [warps][bins] sums, then [warps][bins] counts
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  unsigned* scnt = reinterpret_cast<unsigned*>(ssum + (size_t)nw * bins);
  for (int b = threadIdx.x; b < nw * bins; b += blockDim.x) { ssum[b] = 0.0; scnt[b] = 0u; }
  __syncthreads();
  // each warp walks consecutive groups of 32 points; a CTA owns a contiguous range
  const int per_cta = (g.n + gridDim.x - 1) / gridDim.x;
  const int lo = blockIdx.x * per_cta, hi = min(g.n, lo + per_cta);
  for (int base = lo + w * 32; base < hi; base += nw * 32) {
    const int f = base + lane;
    int bin = -1;
    double v = 0.0;
    if (f < hi) {
      const double r = radius_at(g, f);
      // edges[bin] <= r < edges[bin + 1], clipped to [0, bins - 1]
      int a = 0, c = bins + 1;            // first edge index with edges[idx] > r
      while (a < c) { const int m = (a + c) >> 1; if (edges[m] <= r) a = m + 1; else c = m; }
      bin = a - 1;
      bin = bin < 0 ? 0 : (bin > bins - 1 ? bins - 1 : bin);
      v = fld[f];
    }
    const unsigned active = __ballot_sync(0xffffffffu, bin >= 0);
    const unsigned peers = __match_any_sync(0xffffffffu, bin) & active;
    const int leader = __ffs(peers) - 1;
    // the leader adds its group's values in lane order
    double s = 0.0;
    for (int l = 0; l < 32; ++l) {
      const double x = __shfl_sync(0xffffffffu, v, l);
      if ((peers >> l) & 1u) s += x;
    }
    if (bin >= 0 && lane == leader) {
      ssum[w * bins + bin] += s;
      scnt[w * bins + bin] += (unsigned)__popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  for (int b = threadIdx.x; b < bins; b += blockDim.x) {
    double s = 0.0;
    unsigned c = 0;
    for (int k = 0; k < nw; ++k) { s += ssum[k * bins + b]; c += scnt[k * bins + b]; }
    psum[(size_t)blockIdx.x * bins + b] = s;
    pcnt[(size_t)blockIdx.x * bins + b] = c;
  }
}

__global__ void k_profile_total(const double* psum, const unsigned* pcnt, int blocks, int bins, double* out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < bins; b += gridDim.x * blockDim.x) {
    double s = 0.0;
    unsigned long long c = 0;
    for (int k = 0; k < blocks; ++k) { s += psum[(size_t)k * bins + b]; c += pcnt[(size_t)k * bins + b]; }
    out[b] = c ? s / (double)c : NAN;
  }
}

// Multilinear interpolation of a complex field between two grids (the resampling
// of sweep continuations, becgpp/grid.py:140-161): each new node's coordinate is
// mapped onto the old nodes' index range (first node -> 0, last node -> N_old - 1),
// and the value is the product-weighted sum of the 2^d surrounding old nodes,
// zero for nodes outside the old grid.
__global__ void k_resample(const double2* __restrict__ src, int ndim, int No, double x0, double span,
                           double2* __restrict__ dst, int Nn, double dxn) {
  const long long nn = ndim == 2 ? (long long)Nn * Nn : (long long)Nn * Nn * Nn;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nn;
       f += (long long)gridDim.x * blockDim.x) {
    int idx[3];
    long long r = f;
    for (int a = ndim - 1; a >= 0; --a) { idx[a] = (int)(r % Nn); r /= Nn; }
    int lo[3];
    double w1[3];
    for (int a = 0; a < ndim; ++a) {
      const double c = (double)(idx[a] - Nn / 2) * dxn;
      const double u = 2.0 * (c - x0) / span - 1.0;            // [-1, 1] over the old nodes
      const double ix = ((u + 1.0) / 2.0) * (double)(No - 1);   // old index coordinate
      const double fl = floor(ix);
      lo[a] = (int)fl;
      w1[a] = ix - fl;
    }
    double2 acc = make_double2(0.0, 0.0);
    const int corners = 1 << ndim;
    for (int q = 0; q < corners; ++q) {
      double w = 1.0;
      long long off = 0;
      bool in = true;
      for (int a = 0; a < ndim; ++a) {
        const int hi = (q >> (ndim - 1 - a)) & 1;
        const int ia = lo[a] + hi;
        w *= hi ? w1[a] : (1.0 - w1[a]);
        in = in && ia >= 0 && ia < No;
        off = off * No + ia;
      }
      if (in && w != 0.0) {
        const double2 v = src[off];
        acc.x += w * v.x;
        acc.y += w * v.y;
      }
    }
    dst[f] = acc;
  }
}

// Scratch of one call, from the stream-ordered allocator.
struct Scratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  template <class T>
  int get(size_t count, T** out) {
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, count * sizeof(T) + 16, st);
    if (e != cudaSuccess) return dfail(BGP_ERR_OOM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    ptrs.push_back(p);
    *out = (T*)p;
    return BGP_OK;
  }
  ~Scratch() { for (void* p : ptrs) cudaFreeAsync(p, st); }
};

int make_grid(int ndim, int N, double L, Grid* g) {
  if (ndim != 2 && ndim != 3) return dfail(BGP_ERR_ARG, "ndim must be 2 or 3");
  if (N < 2 || !(L > 0)) return dfail(BGP_ERR_ARG, "bad grid size");
  const long long n = ndim == 2 ? (long long)N * N : (long long)N * N * N;
  if (n > (1ll << 30)) return dfail(BGP_ERR_ARG, "grid too large");
  memset(g, 0, sizeof(*g));
  g->ndim = ndim; g->N = N; g->n = (int)n;
  g->dx = 2.0 * L / N;
  g->dv = ndim == 2 ? g->dx * g->dx : g->dx * g->dx * g->dx;
  return BGP_OK;
}

// mass, centre of mass (or the given centre) and the total of max(rho, 0)
int moments(const double* rho, Grid& g, const double* center, double* mass, double* wsum, Scratch& S) {
  double* part = nullptr;
  double* tot = nullptr;
  int rc = S.get(5 * kRedBlocks, &part);
  if (rc) return rc;
  if ((rc = S.get(5, &tot))) return rc;
  k_moments<<<kRedBlocks, kRedThreads, 0, S.st>>>(rho, g, part);
  k_moments_total<<<1, kRedThreads, 0, S.st>>>(part, kRedBlocks, tot);
  DCK(cudaGetLastError());
  double h[5];
  DCK(cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, S.st));
  DCK(cudaStreamSynchronize(S.st));
  // becgpp/fields.py:11-14: mass = sum rho dV, centre = (sum x rho) dV / mass
  *mass = h[0] * g.dv;
  *wsum = h[4] * g.dv;
  for (int a = 0; a < g.ndim; ++a) {
    if (center) g.c[a] = center[a];
    else g.c[a] = (*mass <= 0.0) ? 0.0 : h[1 + a] * g.dv / *mass;
  }
  return BGP_OK;
}

}  // namespace

extern "C" {

int bgp_density_center(int ndim, int N, double L, const double* rho, double* mass_out, double* center_out,
                       void* stream) {
  if (!rho || !mass_out || !center_out) return dfail(BGP_ERR_ARG, "null pointer");
  Grid g;
  int rc = make_grid(ndim, N, L, &g);
  if (rc) return rc;
  Scratch S{(cudaStream_t)stream, {}};
  double wsum;
  if ((rc = moments(rho, g, nullptr, mass_out, &wsum, S))) return rc;
  for (int a = 0; a < ndim; ++a) center_out[a] = g.c[a];
  return BGP_OK;
}

int bgp_mass_quantiles(int ndim, int N, double L, const double* rho, const double* center,
                       const double* fractions, int nf, double* radii_out, void* stream) {
  if (!rho || !fractions || !radii_out || nf < 1) return dfail(BGP_ERR_ARG, "bad arguments");
  Grid g;
  int rc = make_grid(ndim, N, L, &g);
  if (rc) return rc;
  Scratch S{(cudaStream_t)stream, {}};
  double mass, wsum;
  if ((rc = moments(rho, g, center, &mass, &wsum, S))) return rc;
  const int blocks = 2 * kRedBlocks;
  const size_t hsmem = (size_t)kBins * (sizeof(unsigned long long) + sizeof(unsigned));
  DCK(cudaFuncSetAttribute(k_mq_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem));
  const size_t fsmem = (size_t)2 * kCandCap * sizeof(unsigned long long);
  DCK(cudaFuncSetAttribute(k_mq_finish, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsmem));
  unsigned long long *hw, *ckey, *cw;
  unsigned *hc, *ccount;
  Sel* sel;
  double *dout, *rpart;
  if ((rc = S.get(kBins, &hw)) || (rc = S.get(kBins, &hc)) || (rc = S.get(kCandCap, &ckey)) ||
      (rc = S.get(kCandCap, &cw)) || (rc = S.get(1, &ccount)) || (rc = S.get(1, &sel)) || (rc = S.get(1, &dout)) ||
      (rc = S.get(kRedBlocks, &rpart)))
    return rc;
  // fixed-point scale: the total of max(rho, 0) dV becomes about 2^58
  const double scale = wsum > 0.0 ? kFix / wsum : 0.0;
  for (int q = 0; q < nf; ++q) {
    const double frac = fractions[q];
    if (frac > 1.0 || wsum <= 0.0) {
      if (frac > 1.0) {
        // beyond the total the reference's clamp returns the last point in distance order
        k_max_radius<<<kRedBlocks, kRedThreads, 0, S.st>>>(g, rpart);
        std::vector<double> h(kRedBlocks);
        DCK(cudaMemcpyAsync(h.data(), rpart, sizeof(double) * kRedBlocks, cudaMemcpyDeviceToHost, S.st));
        DCK(cudaStreamSynchronize(S.st));
        radii_out[q] = *std::max_element(h.begin(), h.end());
      } else {
        // no mass: every running sum is 0, the first point in distance order wins, the
        // grid node nearest to the centre (nearest along each axis)
        double r2 = 0.0;
        for (int a = 0; a < g.ndim; ++a) {
          double i = floor(g.c[a] / g.dx + g.N / 2 + 0.5);
          i = std::min(std::max(i, 0.0), (double)(g.N - 1));
          const double d = (i - g.N / 2) * g.dx - g.c[a];
          r2 += d * d;
        }
        radii_out[q] = sqrt(r2);
      }
      continue;
    }
    Sel s0;
    memset(&s0, 0, sizeof(s0));
    DCK(cudaMemcpyAsync(sel, &s0, sizeof(Sel), cudaMemcpyHostToDevice, S.st));
    int shift = 64;
    bool done = false;
    for (int level = 0; level * kDigits < 64 && !done; ++level) {
      // digits of 13 bits from the top; the last one takes the 12 bits left
      const int top = 64 - kDigits * level;
      const int width = std::min(kDigits, top);
      const int dshift = top - width;
      Sel h;
      DCK(cudaMemsetAsync(hw, 0, sizeof(unsigned long long) * kBins, S.st));
      DCK(cudaMemsetAsync(hc, 0, sizeof(unsigned) * kBins, S.st));
      DCK(cudaMemcpyAsync(&h, sel, sizeof(Sel), cudaMemcpyDeviceToHost, S.st));
      DCK(cudaStreamSynchronize(S.st));
      k_mq_hist<<<blocks, kRedThreads, hsmem, S.st>>>(rho, g, scale, h.prefix, shift, dshift, width, hw, hc);
      k_mq_pick<<<1, 1024, 0, S.st>>>(hw, hc, sel, frac, level == 0, width);
      DCK(cudaGetLastError());
      DCK(cudaMemcpyAsync(&h, sel, sizeof(Sel), cudaMemcpyDeviceToHost, S.st));
      DCK(cudaStreamSynchronize(S.st));
      if (!h.found) return dfail(BGP_ERR_DEVICE, "mass quantile: no bin reached the target");
      shift = dshift;
      if (h.count <= (unsigned)kCandCap || dshift == 0) {
        DCK(cudaMemsetAsync(ccount, 0, sizeof(unsigned), S.st));
        k_mq_collect<<<blocks, kRedThreads, 0, S.st>>>(rho, g, scale, h.prefix, shift, ckey, cw, ccount);
        k_mq_finish<<<1, 1024, fsmem, S.st>>>(ckey, cw, ccount, sel, dout);
        DCK(cudaGetLastError());
        DCK(cudaMemcpyAsync(&radii_out[q], dout, sizeof(double), cudaMemcpyDeviceToHost, S.st));
        DCK(cudaStreamSynchronize(S.st));
        done = true;
      }
    }
    if (!done) return dfail(BGP_ERR_DEVICE, "mass quantile: selection did not finish");
  }
  return BGP_OK;
}

int bgp_resample(int ndim, int N_old, double L_old, const void* psi_old, int N_new, double L_new, void* psi_new,
                 void* stream) {
  if (!psi_old || !psi_new) return dfail(BGP_ERR_ARG, "null pointer");
  if (ndim != 2 && ndim != 3) return dfail(BGP_ERR_ARG, "ndim must be 2 or 3");
  if (N_old < 2 || N_new < 1 || !(L_old > 0) || !(L_new > 0)) return dfail(BGP_ERR_ARG, "bad grid");
  if (psi_old == psi_new) return dfail(BGP_ERR_ARG, "psi_new must not alias psi_old");
  const double dxo = 2.0 * L_old / N_old, dxn = 2.0 * L_new / N_new;
  const double x0 = -(double)(N_old / 2) * dxo;             // first old node, as make_grid
  const double span = (x0 + (N_old - 1) * dxo) - x0;        // last old node - first
  if (!(span > 0)) return dfail(BGP_ERR_ARG, "degenerate old grid");
  k_resample<<<592, 256, 0, (cudaStream_t)stream>>>((const double2*)psi_old, ndim, N_old, x0, span,
                                                    (double2*)psi_new, N_new, dxn);
  DCK(cudaGetLastError());
  return BGP_OK;
}

int bgp_radial_profile(int ndim, int N, double L, const double* f, const double* center, const double* edges,
                       int bins, double* prof_out, void* stream) {
  if (!f || !center || !edges || !prof_out || bins < 1) return dfail(BGP_ERR_ARG, "bad arguments");
  if (bins > 2048) return dfail(BGP_ERR_ARG, "at most 2048 bins");
  Grid g;
  int rc = make_grid(ndim, N, L, &g);
  if (rc) return rc;
  for (int a = 0; a < ndim; ++a) g.c[a] = center[a];
  Scratch S{(cudaStream_t)stream, {}};
  const int blocks = kRedBlocks, threads = 256, nw = threads / 32;
  double *dedges, *psum, *dout;
  unsigned* pcnt;
  if ((rc = S.get(bins + 1, &dedges)) || (rc = S.get((size_t)blocks * bins, &psum)) ||
      (rc = S.get((size_t)blocks * bins, &pcnt)) || (rc = S.get(bins, &dout)))
    return rc;
  DCK(cudaMemcpyAsync(dedges, edges, sizeof(double) * (bins + 1), cudaMemcpyHostToDevice, S.st));
  const size_t smem = (size_t)nw * bins * (sizeof(double) + sizeof(unsigned));
  DCK(cudaFuncSetAttribute(k_profile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_profile<<<blocks, threads, smem, S.st>>>(f, g, dedges, bins, psum, pcnt);
  k_profile_total<<<(bins + 255) / 256, 256, 0, S.st>>>(psum, pcnt, blocks, bins, dout);
  DCK(cudaGetLastError());
  DCK(cudaMemcpyAsync(prof_out, dout, sizeof(double) * bins, cudaMemcpyDeviceToHost, S.st));
  DCK(cudaStreamSynchronize(S.st));
  return BGP_OK;
}

}  // extern "C"
