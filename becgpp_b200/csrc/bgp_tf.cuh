// Thomas-Fermi reference density on the device (becgpp/thomasfermi.py:33-120).
//
// The density n solves  mu = V_eff + b2 n + b3 n^2 + phi[n]  with  sum n dV = 1,
// V_eff = V - Omega^2 (x^2 + y^2) / 2 and phi the long-range potential of n
// (zero for the local references). One launch of k_tf_iter is one step of the
// reference's relaxed fixed point:
//   base  = V_eff + phi                      (phi = -G_C dV (K * n), from the plan)
//   mu    : sum_i rho(mu, base_i) dV = 1, by the reference's bracket expansion and
//           90 bisection halvings, each a full-grid sum
//   n_new = rho(mu, base) / (sum rho dV)
//   dn    = sum |n_new - n| dV,  n <- (1 - relax) n + relax n_new,  n <- n / (sum n dV)
// with rho(mu, b) the upper non-negative root of b3 rho^2 + b2 rho = mu - b.
// The local references (no long-range term) use the same launch once, in mode 0:
// n = n_new, no relaxation.
//
// Work decomposition: all CTAs of the launch form one team (cooperative launch,
// bounded team barrier); every full-grid sum is a deterministic grid reduction
// (thread partials in a fixed grid-stride order, warp butterflies, warp totals
// in order, CTA partials added in CTA order after the barrier), so every CTA
// holds the same totals and takes the same bisection decisions without a
// broadcast. The arithmetic of V_eff and rho uses round-to-nearest intrinsics
// (no contraction into FMAs), the operation order of the reference's tensor
// expressions.
#pragma once
#include "bgp_common.cuh"

BGP_NS_BEGIN

struct TfArgs {
  int ndim, N, n, mode;          // mode 0: local (one mu solve), 1: one fixed-point step
  double dx, dv, tc, s, Omega, b2, b3, gc, relax;
  const double* conv;            // dV (K * n) of the current n (mode 1), else null
  double* nf;                    // density: current n in, new n out
  double* part;                  // 2 x 4 x gridDim.x partial sums
  unsigned long long* bar;       // team barrier counter
  int* abort_flag;               // status word (4 + gridDim.x ints)
  double* state;                 // out: [0] mu, [1] dn, [2] status, [3] converged
};

enum TfStatus : int { kTfOk = 0, kTfNoBracket = 1, kTfEmpty = 2, kTfBarrier = 3 };

// V_eff at flat index f (becgpp/thomasfermi.py:21-30 with becgpp/grid.py:86-91).
BGP_D double tf_veff(const TfArgs& A, int f) {
  const int N = A.N;
  int i, j, k = 0;
  if (A.ndim == 2) { i = f / N; j = f - i * N; }
  else { i = f / (N * N); const int r = f - i * N * N; j = r / N; k = r - j * N; }
  const double x = (double)(i - N / 2) * A.dx, y = (double)(j - N / 2) * A.dx;
  const double rp2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
  double r2 = rp2;
  if (A.ndim == 3) { const double z = (double)(k - N / 2) * A.dx; r2 = __dadd_rn(r2, __dmul_rn(z, z)); }
  double V = 0.0;
  if (A.s > 0.0) V = (A.s == 2.0) ? __dmul_rn(A.tc, r2) : __dmul_rn(A.tc, pow(r2, 0.5 * A.s));
  const double c = (0.5 * A.Omega) * A.Omega;
  return __dsub_rn(V, __dmul_rn(c, rp2));
}

// Upper physical root rho >= 0 of b3 rho^2 + b2 rho = mu - b, zero where there is
// no real root (becgpp/thomasfermi.py:33-45).
BGP_D double tf_rho(double mu, double b, double b2, double b3) {
  const double rhs = __dsub_rn(mu, b);
  if (b3 > 1e-30) {
    const double disc = __dadd_rn(__dmul_rn(b2, b2), __dmul_rn(4.0 * b3, rhs));
    if (!(disc > 0.0)) return 0.0;
    const double root = __ddiv_rn(__dadd_rn(-b2, sqrt(disc)), 2.0 * b3);
    return root > 0.0 ? root : 0.0;
  }
  if (fabs(b2) > 1e-30) {
    const double q = __ddiv_rn(rhs, b2);
    return q > 0.0 ? q : 0.0;
  }
  return 0.0;
}

#if defined(__CUDACC__)

// Deterministic grid-wide reduction of NV values per thread (op: 0 sum, 1 min,
// 2 max), identical totals in every CTA. sm: NV * kWarps + NV doubles. The
// partials of the two alternating slots sit 4 values apart whatever NV is, so a
// reduction never writes where the previous one (other slot) is still being read.
template <int NV>
BGP_D bool grid_reduce(double (&v)[NV], const int (&op)[NV], double* part, int& slot, const Team& T,
                       double* sm) {
  static_assert(NV <= 4, "at most 4 values per reduction");
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, G = gridDim.x;
  auto comb = [](int o, double a, double b) { return o == 0 ? a + b : (o == 1 ? fmin(a, b) : fmax(a, b)); };
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = comb(op[q], x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) sm[q * kWarps + w] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int q = threadIdx.x;
    double x = sm[q * kWarps];
    for (int k = 1; k < kWarps; ++k) x = comb(op[q], x, sm[q * kWarps + k]);
    st1(part + ((size_t)slot * 4 + q) * G + blockIdx.x, x);
  }
  if (!team_sync(T)) return false;
  // warp q adds the G partials of value q: lane l takes CTAs l, l+32, ... in order,
  // then the 32 lane totals meet in a fixed butterfly
  if (w < NV) {
    const int q = w;
    const double* p = part + ((size_t)slot * 4 + q) * G;
    double x = (op[q] == 0) ? 0.0 : ld1(p);
    for (int b = lane; b < G; b += 32) x = comb(op[q], x, ld1(p + b));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = comb(op[q], x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) sm[NV * kWarps + q] = x;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = sm[NV * kWarps + q];
  __syncthreads();
  slot ^= 1;
  return true;
}

// One Thomas-Fermi step (see the file comment). Launched cooperatively with every
// CTA resident; kThreads threads per CTA.
__global__ void __launch_bounds__(kThreads) k_tf_iter(TfArgs A) {
  static_assert(kWarps >= 4, "grid_reduce needs a warp per reduced value");
  __shared__ double sm[4 * kWarps + 4];
  Team T{(int)blockIdx.x, (int)gridDim.x, A.bar, A.abort_flag};
  int slot = 0;
  const int n = A.n;
  const int first = blockIdx.x * kThreads + threadIdx.x, stride = gridDim.x * kThreads;
  const double gc = A.gc;
  auto base = [&](int f) {
    const double v = tf_veff(A, f);
    return A.conv ? __dadd_rn(v, __dmul_rn(-gc, ld1(A.conv + f))) : v;
  };
  auto fail = [&](int code) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { A.state[2] = (double)code; A.state[3] = 0.0; }
  };
  // bracket of mu: [min base, max base + |b2| + |b3| + 1] (becgpp/thomasfermi.py:99-100)
  double lo, hi;
  {
    double v[2] = {INFINITY, -INFINITY};
    const int op[2] = {1, 2};
    for (int f = first; f < n; f += stride) { const double b = base(f); v[0] = fmin(v[0], b); v[1] = fmax(v[1], b); }
    if (!grid_reduce<2>(v, op, A.part, slot, T, sm)) { fail(kTfBarrier); return; }
    lo = v[0];
    hi = v[1] + fabs(A.b2) + fabs(A.b3) + 1.0;
  }
  auto mass = [&](double mu, double& out) {
    double v[1] = {0.0};
    const int op[1] = {0};
    for (int f = first; f < n; f += stride) v[0] += tf_rho(mu, base(f), A.b2, A.b3);
    if (!grid_reduce<1>(v, op, A.part, slot, T, sm)) return false;
    out = v[0] * A.dv;
    return true;
  };
  // expand the upper end until it holds unit mass (becgpp/thomasfermi.py:51-55)
  for (int guard = 0;; ++guard) {
    double m;
    if (!mass(hi, m)) { fail(kTfBarrier); return; }
    if (m >= 1.0) break;
    if (guard >= 200) { fail(kTfNoBracket); return; }
    hi = lo + 2.0 * (hi - lo) + 1e-9;
  }
  for (int step = 0; step < 90; ++step) {     // becgpp/thomasfermi.py:56-61
    const double mid = 0.5 * (lo + hi);
    double m;
    if (!mass(mid, m)) { fail(kTfBarrier); return; }
    if (m < 1.0) lo = mid; else hi = mid;
  }
  const double mu = 0.5 * (lo + hi);
  double ssum;
  if (!mass(mu, ssum)) { fail(kTfBarrier); return; }
  if (!(ssum > 0.0)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) A.state[0] = mu;
    fail(kTfEmpty);
    return;
  }
  double dn = 0.0;
  if (A.mode == 0) {
    // local reference: n = rho(mu) / (sum rho dV)
    for (int f = first; f < n; f += stride) st1(A.nf + f, __ddiv_rn(tf_rho(mu, base(f), A.b2, A.b3), ssum));
  } else {
    // relaxed update and its renormalisation (becgpp/thomasfermi.py:103-110)
    double v[2] = {0.0, 0.0};
    const int op[2] = {0, 0};
    const double a = 1.0 - A.relax, r = A.relax;
    for (int f = first; f < n; f += stride) {
      const double nn = __ddiv_rn(tf_rho(mu, base(f), A.b2, A.b3), ssum);
      const double old = ld1(A.nf + f);
      v[0] += fabs(__dsub_rn(nn, old));
      const double upd = __dadd_rn(__dmul_rn(a, old), __dmul_rn(r, nn));
      st1(A.nf + f, upd);
      v[1] += upd;
    }
    if (!grid_reduce<2>(v, op, A.part, slot, T, sm)) { fail(kTfBarrier); return; }
    dn = v[0] * A.dv;
    const double norm = v[1] * A.dv;
    for (int f = first; f < n; f += stride) st1(A.nf + f, __ddiv_rn(ld1(A.nf + f), norm));
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.state[0] = mu;
    A.state[1] = dn;
    A.state[2] = (double)kTfOk;
    A.state[3] = (A.mode == 0 || dn < 1e-9) ? 1.0 : 0.0;
  }
}

// Initial density of the fixed point, exp(-r^2 / (2 sigma^2)) with sigma = 0.15 L,
// normalised to unit mass (becgpp/thomasfermi.py:89-91). Cooperative launch.
__global__ void __launch_bounds__(kThreads) k_tf_seed(TfArgs A, double two_s2) {
  __shared__ double sm[4 * kWarps + 4];
  Team T{(int)blockIdx.x, (int)gridDim.x, A.bar, A.abort_flag};
  int slot = 0;
  const int n = A.n, N = A.N;
  const int first = blockIdx.x * kThreads + threadIdx.x, stride = gridDim.x * kThreads;
  double v[1] = {0.0};
  const int op[1] = {0};
  for (int f = first; f < n; f += stride) {
    int i, j, k = 0;
    if (A.ndim == 2) { i = f / N; j = f - i * N; }
    else { i = f / (N * N); const int r = f - i * N * N; j = r / N; k = r - j * N; }
    const double x = (double)(i - N / 2) * A.dx, y = (double)(j - N / 2) * A.dx;
    double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
    if (A.ndim == 3) { const double z = (double)(k - N / 2) * A.dx; r2 = __dadd_rn(r2, __dmul_rn(z, z)); }
    const double e = exp(__ddiv_rn(-r2, two_s2));
    st1(A.nf + f, e);
    v[0] += e;
  }
  if (!grid_reduce<1>(v, op, A.part, slot, T, sm)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) A.state[2] = (double)kTfBarrier;
    return;
  }
  const double norm = v[0] * A.dv;
  for (int f = first; f < n; f += stride) st1(A.nf + f, __ddiv_rn(ld1(A.nf + f), norm));
}

#endif  // __CUDACC__

BGP_NS_END  // namespace bgp
