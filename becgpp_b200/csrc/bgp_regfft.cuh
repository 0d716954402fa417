// Register-resident line transform of a warp (N = 32 R), in complex128 or
// complex64 arithmetic: the stream passes' transform and the persistent solver's
// line transform of the sizes N = 32 R.
#pragma once
#include "bgp_device.cuh"

BGP_NS_BEGIN

// For N = 32 R a warp holds its line in registers: lane l, slot q holds
// x[l + 32 q]. With n = l + 32 q and k = k1 + R k2,
//   X[k1 + R k2] = sum_l w32^(l k2) [ wN^(l k1) sum_q x[l + 32 q] wR^(q k1) ],
// so the forward transform is an R-point DFT in each lane's registers, a twiddle
// by wN^(l k1), and for every slot k1 a 32-point DFT across the lanes, done as a
// decimation-in-frequency butterfly network over lane pairs (shuffles). It leaves
// lane l, slot k1 holding X[k1 + R rev5(l)] (rev5: the 5-bit reversal). The
// inverse runs the network backwards (each stage undone, up to a factor 2),
// the conjugate twiddles and inverse R-point DFTs, and returns N x (the input)
// to natural order: an unnormalised inverse, as warp_fft's. A multiplier that
// depends on k is applied in between at k = k1 + R rev5(l). Nothing of the line
// transform touches shared memory.
BGP_HD constexpr int rev5(int l) {
  return ((l & 1) << 4) | ((l & 2) << 2) | (l & 4) | ((l & 8) >> 2) | ((l & 16) >> 4);
}

#if defined(__CUDACC__)

// In-register DFT of R values v[0..R-1] (natural order in and out). wR^m is
// tw[m * (N / R)] of the line's twiddle table.
template <int R, bool INV, int N, class T>
BGP_D void dft_reg(T (&v)[R], const T* __restrict__ tw) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2 || R == 3 || R == 4 || R == 5 || R == 8) {
    dft_small<R, INV>(v);
  } else {
    // R = A * B, A the first factor; n = B n1 + n2, k = k1 + A k2:
    // X[k1 + A k2] = sum_n2 wB^(n2 k2) wR^(n2 k1) sum_n1 x[B n1 + n2] wA^(n1 k1)
    constexpr int A = (R % 4 == 0) ? 4 : ((R % 3 == 0) ? 3 : 2);
    constexpr int B = R / A;
    T t[B][A];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      T a[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) a[n1] = v[B * n1 + n2];
      dft_small<A, INV>(a);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        T w = __ldg(tw + ((n2 * k1) % R) * (N / R));
        if (INV) w.y = -w.y;
        t[n2][k1] = (n2 * k1 == 0) ? a[k1] : cmul(a[k1], w);
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      T b[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) b[n2] = t[n2][k1];
      dft_reg<B, INV, N, T>(b, tw);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = b[k2];
    }
  }
}

// Forward: natural slots in, spectrum X[k1 + R rev5(lane)] in slot k1 out.
template <int N, class T>
BGP_D void reg_fft_fwd(T (&v)[N / 32], const T* __restrict__ tw, int lane) {
  constexpr int R = N / 32;
  dft_reg<R, false, N, T>(v, tw);
#pragma unroll
  for (int k1 = 1; k1 < R; ++k1) v[k1] = cmul(v[k1], __ldg(tw + (lane * k1) % N));
  // DIF across lanes: pairs (l, l ^ m), m = 16 .. 1; the upper lane of a pair
  // takes (a - b) w32^(j 16 / m), j = l mod m; the lower takes a + b
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) {
    const bool up = (lane & m) != 0;
    const T w = __ldg(tw + ((lane & (m - 1)) * (16 / m)) * (N / 32));
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      T o;
      o.x = __shfl_xor_sync(0xffffffffu, v[k1].x, m);
      o.y = __shfl_xor_sync(0xffffffffu, v[k1].y, m);
      v[k1] = up ? cmul(csub(o, v[k1]), w) : cadd(v[k1], o);
    }
  }
}

// Inverse of reg_fft_fwd times N: spectrum in the forward's order in, natural out.
template <int N, class T>
BGP_D void reg_fft_inv(T (&v)[N / 32], const T* __restrict__ tw, int lane) {
  constexpr int R = N / 32;
  // undo each DIF stage: from (u, v') = (a + b, (a - b) w): a = u + v' conj(w),
  // b = u - v' conj(w) (each times 2)
#pragma unroll
  for (int m = 1; m <= 16; m <<= 1) {
    const bool up = (lane & m) != 0;
    T w = __ldg(tw + ((lane & (m - 1)) * (16 / m)) * (N / 32));
    w.y = -w.y;
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      T o;
      o.x = __shfl_xor_sync(0xffffffffu, v[k1].x, m);
      o.y = __shfl_xor_sync(0xffffffffu, v[k1].y, m);
      v[k1] = up ? csub(o, cmul(v[k1], w)) : cadd(v[k1], cmul(o, w));
    }
  }
#pragma unroll
  for (int k1 = 1; k1 < R; ++k1) {
    T w = __ldg(tw + (lane * k1) % N);
    w.y = -w.y;
    v[k1] = cmul(v[k1], w);
  }
  dft_reg<R, true, N, T>(v, tw);
}


// A line in shared memory (element i at swz(i), natural order) transformed in
// registers: mode 0 forward; 1 inverse; 2 forward, v <- mult(k, v), inverse.
// The forward-only result is stored in natural order too; `spec(k, v)` sees
// every spectral value after a forward transform (for sums over the spectrum).
template <int L, class T, class F, class S>
BGP_D void reg_line(T* b, const T* __restrict__ tw, int lane, int mode, F mult, S spec, bool store = true) {
  constexpr int R = L / 32;
  const int kb = R * rev5(lane);
  T v[R];
  if (mode == 1) {
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) v[k1] = b[swz(k1 + kb)];
  } else {
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = b[swz(lane + 32 * q)];
  }
  __syncwarp();
  if (mode != 1) {
    reg_fft_fwd<L, T>(v, tw, lane);
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) spec(k1 + kb, v[k1]);
  }
  if (mode == 2) {
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) v[k1] = mult(k1 + kb, v[k1]);
  }
  if (mode != 0) reg_fft_inv<L, T>(v, tw, lane);
  if (!store) return;
  if (mode == 0) {
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) b[swz(k1 + kb)] = v[k1];
  } else {
#pragma unroll
    for (int q = 0; q < R; ++q) b[swz(lane + 32 * q)] = v[q];
  }
  __syncwarp();
}

#endif  // __CUDACC__

BGP_NS_END
