// Shared device helpers: complex arithmetic, team barriers, deterministic block
// reductions and order-preserving keys for the median selection.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define BGP_HD __host__ __device__ __forceinline__
#define BGP_D __device__ __forceinline__
#else
#define BGP_HD inline
#define BGP_D inline
#endif

// Kernels with FP32 line transforms (the mixed-precision form) are compiled in
// separate translation units with BGP_MIXED=1, and every solver kernel is
// compiled once per grid dimension (BGP_NDIM = 2 or 3): the branches of the
// other dimension are then not in the code, whose size the persistent kernel's
// instruction cache feels. BGP_NDIM 0 (table builds, the allocation-free entry
// point) reads the dimension from the instance. Each build's device code lives
// in its own inline namespace so two builds of a template never share a symbol.
#ifndef BGP_MIXED
#define BGP_MIXED 0
#endif
#ifndef BGP_NDIM
#define BGP_NDIM 0
#endif
#if BGP_NDIM
#define BGP_DIM(x) BGP_NDIM
#else
#define BGP_DIM(x) ((x).ndim)
#endif
#if BGP_MIXED && BGP_NDIM == 2
#define BGP_NS_BEGIN namespace bgp { inline namespace d2_fp32 {
#elif BGP_MIXED && BGP_NDIM == 3
#define BGP_NS_BEGIN namespace bgp { inline namespace d3_fp32 {
#elif BGP_MIXED
#define BGP_NS_BEGIN namespace bgp { inline namespace with_fp32 {
#elif BGP_NDIM == 2
#define BGP_NS_BEGIN namespace bgp { inline namespace d2 {
#elif BGP_NDIM == 3
#define BGP_NS_BEGIN namespace bgp { inline namespace d3 {
#endif
#if BGP_MIXED || BGP_NDIM
#define BGP_NS_END } }
#else
#define BGP_NS_BEGIN namespace bgp {
#define BGP_NS_END }
#endif

BGP_NS_BEGIN

constexpr int kWarps = 4;                 // warps (= lines) per CTA tile
constexpr int kLines = kWarps;            // lines per tile, one warp each
constexpr int kThreads = kWarps * 32;     // threads per CTA

// Shared-memory layout of a line of L complex values: element i sits at
// swz(i) = i + i/8, one padding slot after every 8 elements. A warp's 16-byte
// accesses are served 8 lanes at a time; with the padding the radix-R stage
// outputs (stride R for the first stage) land on distinct bank groups. Lines
// are line_stride(L) apart, chosen so that the 8 lanes of a strided tile access
// (kLines lines x 8/kLines consecutive elements) also do: an odd stride for 8
// lines, a stride of 2 mod 8 for 4 lines.
BGP_HD constexpr int swz(int i) { return i + (i >> 3); }
BGP_HD constexpr int line_stride(int L) {
  return (kLines >= 8) ? ((L + L / 8 + 1) | 1) : (((L + L / 8 + 1 + 5) / 8) * 8 + 2);
}
BGP_HD constexpr size_t tile_smem_bytes(int L) { return (size_t)kLines * line_stride(L) * 16; }

// Complex arithmetic on double2 (FP64) and float2 (FP32, the transforms of the
// mixed-precision form); CT<T>::R is the real type.
template <class T> struct CT {};
template <> struct CT<double2> { using R = double; };
template <> struct CT<float2> { using R = float; };
template <class T>
BGP_HD T cmake(typename CT<T>::R x, typename CT<T>::R y) { T r; r.x = x; r.y = y; return r; }

BGP_HD double2 cmk(double x, double y) { double2 r; r.x = x; r.y = y; return r; }
template <class T> BGP_HD T cadd(T a, T b) { return cmake<T>(a.x + b.x, a.y + b.y); }
template <class T> BGP_HD T csub(T a, T b) { return cmake<T>(a.x - b.x, a.y - b.y); }
template <class T> BGP_HD T cscale(T a, typename CT<T>::R s) { return cmake<T>(a.x * s, a.y * s); }
template <class T> BGP_HD T cmul(T a, T b) {
  return cmake<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class T> BGP_HD T cconjmul(T a, T b) {  // conj(a) * b
  return cmake<T>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <class T> BGP_HD T cmul_i(T a) { return cmake<T>(-a.y, a.x); }       // i * a
template <class T> BGP_HD T cmul_mi(T a) { return cmake<T>(a.y, -a.x); }      // -i * a
BGP_HD double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
// |a|^2 of an FP32 value, formed and returned in FP64
BGP_HD double cabs2(float2 a) { return (double)a.x * (double)a.x + (double)a.y * (double)a.y; }

// conversions between the storage type (double2) and a transform type
template <class T> BGP_HD T to_c(double2 a);
template <> BGP_HD double2 to_c<double2>(double2 a) { return a; }
template <> BGP_HD float2 to_c<float2>(double2 a) { return cmake<float2>((float)a.x, (float)a.y); }
BGP_HD double2 to_d(double2 a) { return a; }
BGP_HD double2 to_d(float2 a) { return cmk((double)a.x, (double)a.y); }

// Order-preserving map from double to uint64: unsigned comparison of the keys
// equals numeric comparison of the values (NaN excluded). Key 0 is never the
// image of a non-NaN double and marks "not in the sample".
BGP_HD uint64_t dkey(double v) {
#if defined(__CUDA_ARCH__)
  uint64_t b = (uint64_t)__double_as_longlong(v);
#else
  uint64_t b; memcpy(&b, &v, 8);
#endif
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
BGP_HD double dkey_inv(uint64_t k) {
  uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)b);
#else
  double v; memcpy(&v, &b, 8); return v;
#endif
}

#if defined(__CUDACC__)

// Cache-global loads/stores: fields written by one CTA are read by another CTA
// of the same persistent launch after a team barrier, so they bypass L1. The
// stores are volatile asm without a "memory" clobber: unlike __stcg they do not
// make the compiler reload every value from memory after each store (which
// reloads the operands kept in shared memory and serialises the loads of a
// tile behind its stores). Ordering against other threads comes from the
// barriers (__syncthreads, the team barrier's release/acquire), which are
// compiler barriers; volatile asm keeps the program order among these loads
// and stores.
BGP_D double2 ld2(const double2* p) { return __ldcg(p); }
BGP_D double ld1(const double* p) { return __ldcg(p); }
BGP_D void st2(double2* p, double2 v) {
  asm volatile("st.global.cg.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y));
}
BGP_D void st1(double* p, double v) { asm volatile("st.global.cg.f64 [%0], %1;" ::"l"(p), "d"(v)); }

BGP_D uint64_t gtimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Error codes written to the device status word.
enum DevErr : int { kDevOk = 0, kDevBarrierTimeout = 1, kDevBadSize = 2, kDevNonFinite = 3 };

// A team is a set of co-resident CTAs working on one instance. Its barrier is a
// monotonically increasing 64-bit counter; each arrival adds one, and a CTA waits
// until the counter reaches the next multiple of the team size. Every wait is
// bounded: after `limit_ns` (or as soon as any CTA has raised the abort flag)
// the CTA records the failure and returns false, so a fault can never hang the GPU.
struct Team {
  int rank;                          // CTA rank within the team
  int size;                          // CTAs in the team
  unsigned long long* bar;           // team barrier counter (null when size == 1)
  int* abort_flag;                   // grid-wide abort word
};

BGP_D void compiler_fence() { asm volatile("" ::: "memory"); }

BGP_D bool team_sync(const Team& t, uint64_t limit_ns = 4000000000ull) {
  // The global stores and loads of the passes are volatile asm without a
  // "memory" clobber; these fences keep the compiler from moving them across
  // the barrier (a store sunk below it would be released too late, a load
  // hoisted above it would read another CTA's data before it is written).
  compiler_fence();
  __syncthreads();
  compiler_fence();
  if (t.size == 1) return true;
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    // arrive with release semantics (covers the CTA's writes ordered by the
    // __syncthreads above), wait with acquire loads
    unsigned long long old;
    asm volatile("atom.add.release.gpu.u64 %0, [%1], %2;" : "=l"(old) : "l"(t.bar), "l"(1ull) : "memory");
    t.abort_flag[4 + blockIdx.x] = (int)(old + 1ull);   // this CTA's last arrival (diagnostics)
    unsigned long long target = (old / (unsigned long long)t.size + 1ull) * (unsigned long long)t.size;
    int ok = 1;
    uint64_t t0 = gtimer_ns();
    unsigned spins = 0;
    while (true) {
      unsigned long long cur;
      asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(cur) : "l"(t.bar) : "memory");
      if (cur >= target) break;
      // the abort word and the clock every 64 polls: a load after the acquire
      // load waits for it, so checking both on every poll doubles its latency
      if ((++spins & 63u) != 0) continue;
      if (*((volatile int*)t.abort_flag) != 0) { ok = 0; break; }
      if (gtimer_ns() - t0 > limit_ns) {
        // the first CTA to give up records where: its block, the barrier count it
        // waited for and the count it saw (abort_flag[1..3])
        if (atomicCAS(t.abort_flag, 0, (int)kDevBarrierTimeout) == 0) {
          t.abort_flag[1] = (int)blockIdx.x;
          t.abort_flag[2] = (int)target;
          t.abort_flag[3] = (int)cur;
        }
        ok = 0;
        break;
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  compiler_fence();
  return s_ok != 0;
}

// Deterministic CTA-wide sum of the first NV of the doubles v[]: butterfly
// shuffles within each warp, then the warp totals added in warp order. Result
// valid in all threads.
template <int NV, int CAP>
BGP_D void block_sum(double (&v)[CAP], double* smem /* >= NV * kWarps */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double x = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    v[i] = x;
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) smem[i * kWarps + w] = v[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kWarps; ++k) s += smem[i * kWarps + k];
    v[i] = s;
  }
  __syncthreads();
}

// Warp reduce-scatter of 16 doubles: each of the five butterfly steps halves
// the values a lane carries (16 shuffles in all instead of 80). Afterwards v[0]
// of lane l holds the warp sum of slot rs16_slot(l); lanes l and l^1 agree. The
// summation tree is fixed, so the result is deterministic.
BGP_D int rs16_slot(int lane) {
  return ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
}
BGP_D void warp_rs16(double (&v)[16], int lane) {
#pragma unroll
  for (int h = 8; h >= 1; h >>= 1) {
    const bool hi = (lane & (2 * h)) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const double send = hi ? v[i] : v[i + h];
      const double keep = hi ? v[i + h] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 2 * h);
    }
  }
  v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
}

BGP_D void block_max(double& v, double* smem) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) smem[w] = v;
  __syncthreads();
  double m = smem[0];
#pragma unroll
  for (int k = 1; k < kWarps; ++k) m = fmax(m, smem[k]);
  v = m;
  __syncthreads();
}

#endif  // __CUDACC__

BGP_NS_END  // namespace bgp
