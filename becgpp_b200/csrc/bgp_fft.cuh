// Line FFTs for lengths N = 2^a 3^b 5^c, one warp per line, in shared memory.
//
// Stockham autosort, decimation in time. A stage of radix R after sub-transforms
// of length P (the product of the radices already applied) maps butterfly
// b in [0, N/R):
//     k = b mod P,  inputs  x_q = in[b + q N/R],          q = 0..R-1
//     x_q *= w^(q k N/(P R))            (w = exp(-+2 pi i / N), table entry)
//     y   = DFT_R(x)
//     out[(b - k) R + k + q P] = y_q
// and leaves the transform in natural order after the last stage, with no bit
// reversal. The warp version runs each stage in place: every lane first loads
// all inputs of its butterflies into registers, the warp synchronises, then the
// outputs are written. The index arithmetic and butterflies are shared with a
// host emulation (bgp_fft_host_line) used by the CPU tests.
#pragma once
#include "bgp_common.cuh"

BGP_NS_BEGIN

struct RPlan {
  int n;
  int r[16];
};

// Radix schedule: at each stage the largest radix in {8, 5, 4, 3, 2} that divides
// what is left and keeps the stage's butterfly count N/R a multiple of the warp
// width (so no lane idles); if none does, the largest radix that divides.
BGP_HD constexpr RPlan make_rplan(int N) {
  RPlan p{};
  int m = N;
  const int cand[5] = {8, 5, 4, 3, 2};
  while (m > 1 && p.n < 16) {
    int pick = 0;
    for (int q = 0; q < 5 && !pick; ++q)
      if (m % cand[q] == 0 && (N / cand[q]) % 32 == 0) pick = cand[q];
    for (int q = 0; q < 5 && !pick; ++q)
      if (m % cand[q] == 0) pick = cand[q];
    if (!pick) { p.n = -1; return p; }
    p.r[p.n++] = pick;
    m /= pick;
  }
  return p;
}

BGP_HD constexpr bool fft_size_ok(int N) { return N >= 2 && make_rplan(N).n > 0; }

// cos/sin of 2 pi / 3, 2 pi / 5, 4 pi / 5 and sqrt(1/2) (closed forms:
// (sqrt5 - 1)/4, -(sqrt5 + 1)/4, sqrt(10 + 2 sqrt5)/4, sqrt(10 - 2 sqrt5)/4).
constexpr double kS3 = 0.86602540378443864676;
constexpr double kC51 = 0.30901699437494742410;
constexpr double kC52 = -0.80901699437494742410;
constexpr double kS51 = 0.95105651629515357212;
constexpr double kS52 = 0.58778525229247312917;
constexpr double kR2 = 0.70710678118654752440;

// multiply by -i (forward) or +i (inverse)
template <bool INV, class T>
BGP_HD T rot90(T a) { return INV ? cmul_i(a) : cmul_mi(a); }

template <int R, bool INV, class T>
BGP_HD void dft_small(T* v) {
  using Rt = typename CT<T>::R;
  if constexpr (R == 2) {
    T a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 3) {
    T t = cadd(v[1], v[2]);
    T m = csub(v[0], cscale(t, (Rt)0.5));
    T d = rot90<INV>(cscale(csub(v[1], v[2]), (Rt)kS3));
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, d);
    v[2] = csub(m, d);
  } else if constexpr (R == 4) {
    T a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    T b0 = cadd(v[1], v[3]), b1 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1);
    v[3] = csub(a1, b1);
  } else if constexpr (R == 5) {
    T a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
    T b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
    T m1 = cadd(v[0], cadd(cscale(a1, (Rt)kC51), cscale(a2, (Rt)kC52)));
    T m2 = cadd(v[0], cadd(cscale(a1, (Rt)kC52), cscale(a2, (Rt)kC51)));
    T d1 = rot90<INV>(cadd(cscale(b1, (Rt)kS51), cscale(b2, (Rt)kS52)));
    T d2 = rot90<INV>(csub(cscale(b1, (Rt)kS52), cscale(b2, (Rt)kS51)));
    v[0] = cadd(v[0], cadd(a1, a2));
    v[1] = cadd(m1, d1);
    v[4] = csub(m1, d1);
    v[2] = cadd(m2, d2);
    v[3] = csub(m2, d2);
  } else if constexpr (R == 8) {
    // radix 8 = radix 2 over two radix-4 halves (even / odd inputs)
    T e[4] = {v[0], v[2], v[4], v[6]};
    T o[4] = {v[1], v[3], v[5], v[7]};
    dft_small<4, INV>(e);
    dft_small<4, INV>(o);
    // twiddles exp(-+ 2 pi i m / 8), m = 1,2,3
    T o1 = cscale(cadd(o[1], rot90<INV>(o[1])), (Rt)kR2);   // (1 -+ i)/sqrt2
    T o2 = rot90<INV>(o[2]);
    T o3 = cscale(csub(rot90<INV>(o[3]), o[3]), (Rt)kR2);   // (-1 -+ i)/sqrt2
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
}

// Twiddle, butterfly and output position of butterfly b (shared host/device).
template <int N, int R, int P, bool INV, class T>
BGP_HD int butterfly_at(T* v, const T* tw, int b) {
  const int k = b % P;
  if constexpr (P > 1) {
    constexpr int step = N / (P * R);
#pragma unroll
    for (int q = 1; q < R; ++q) {
      T w = tw[q * k * step];
      if (INV) w.y = -w.y;
      v[q] = cmul(v[q], w);
    }
  }
  dft_small<R, INV>(v);
  return (b - k) * R + k;
}

// Host emulation of one full line transform (out-of-place per stage).
template <int N, int S, int P, bool INV>
inline void host_stages(double2* a, double2* b, const double2* tw) {
  constexpr RPlan pl = make_rplan(N);
  if constexpr (S < pl.n) {
    constexpr int R = pl.r[S];
    constexpr int B = N / R;
    for (int bi = 0; bi < B; ++bi) {
      double2 v[R];
      for (int q = 0; q < R; ++q) v[q] = a[bi + q * B];
      int j = butterfly_at<N, R, P, INV>(v, tw, bi);
      for (int q = 0; q < R; ++q) b[j + q * P] = v[q];
    }
    for (int i = 0; i < N; ++i) a[i] = b[i];
    host_stages<N, S + 1, P * R, INV>(a, b, tw);
  }
}

#if defined(__CUDACC__)

template <int N, int S, int P, bool INV, class T>
BGP_D void warp_stages(T* buf, const T* __restrict__ tw, int lane) {
  constexpr RPlan pl = make_rplan(N);
  if constexpr (S < pl.n) {
    constexpr int R = pl.r[S];
    constexpr int B = N / R;
    constexpr int U = (B + 31) / 32;
    T v[U][R];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int b = lane + 32 * u;
      if (B % 32 == 0 || b < B) {
#pragma unroll
        for (int q = 0; q < R; ++q) v[u][q] = buf[swz(b + q * B)];
      }
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int b = lane + 32 * u;
      if (B % 32 == 0 || b < B) {
        const int j = butterfly_at<N, R, P, INV>(v[u], tw, b);
#pragma unroll
        for (int q = 0; q < R; ++q) buf[swz(j + q * P)] = v[u][q];
      }
    }
    __syncwarp();
    warp_stages<N, S + 1, P * R, INV>(buf, tw, lane);
  }
}

// Unnormalised transform of the N-point line in shared memory `buf` (element i
// at buf[swz(i)]) by one warp, in the arithmetic of T (double2 or float2):
// forward X_k = sum x_n exp(-2 pi i n k / N); inverse with +i (no 1/N).
template <int N, bool INV, class T>
BGP_D void warp_fft(T* buf, const T* __restrict__ tw, int lane) {
  static_assert(fft_size_ok(N), "FFT length must be 2^a 3^b 5^c");
  warp_stages<N, 0, 1, INV>(buf, tw, lane);
}

#endif  // __CUDACC__

BGP_NS_END  // namespace bgp
