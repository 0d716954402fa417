// Stream passes: the Hamiltonian apply and the zero-padded convolution as plain
// (non-persistent) launches, one launch per axis pass over every tile of every
// instance of a batch, for the standalone and batched H psi entry points.
//
// Unlike the solver's persistent team kernel, a stream pass needs no team
// barrier: the launch boundary orders the passes, so all SMs work on one pass at
// a time and nothing waits on the host. Each pass is templated on
//   L   the line length,
//   LN  the lines per tile (one warp per line; a CTA is LN warps). On a strided
//       axis a tile groups LN neighbours along the contiguous axis, so each of its
//       rows is LN x 16 contiguous bytes (LN = 8: one 128-byte line),
//   V   the radix order of the line FFT (0: largest radix first, 1: reversed,
//       2: radix 4 first),
// and the host's autotuner times the compiled (LN, V) candidates of a plan's grid
// size on its own data and keeps the fastest.
//
// H psi of an instance (operators.py:36-45 of the reference) is a sum of
// per-axis terms: along a y-line the multiplier (k_y^2/2 - Omega x k_y), along an
// x-line (k_x^2/2 + Omega y k_x), along z k_z^2/2, each applied by a forward and
// an inverse line FFT. The passes accumulate them in a scratch field A; the last
// pass adds (V + b2 rho + b3 rho^2 + phi) psi, writes H psi and each CTA's part
// of Re<psi, H psi>.
#pragma once
#include "bgp_device.cuh"
#include "bgp_regfft.cuh"

BGP_NS_BEGIN

// ---------------------------------------------------------------- radix orders
template <int V>
BGP_HD constexpr RPlan make_rplan_v(int N) {
  if constexpr (V == 0) {
    return make_rplan(N);
  } else if constexpr (V == 1) {
    RPlan p = make_rplan(N);
    for (int a = 0, b = p.n - 1; a < b; ++a, --b) { const int t = p.r[a]; p.r[a] = p.r[b]; p.r[b] = t; }
    return p;
  } else {
    RPlan p{};
    int m = N;
    const int cand[5] = {4, 8, 5, 3, 2};
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
}

// Host emulation of a line transform in radix order V (CPU tests of the orders).
template <int N, int V, int S, int P, bool INV>
inline void host_stages_v(double2* a, double2* b, const double2* tw) {
  constexpr RPlan pl = make_rplan_v<V>(N);
  if constexpr (S < pl.n) {
    constexpr int R = pl.r[S];
    constexpr int B = N / R;
    for (int bi = 0; bi < B; ++bi) {
      double2 v[R];
      for (int q = 0; q < R; ++q) v[q] = a[bi + q * B];
      const int j = butterfly_at<N, R, P, INV>(v, tw, bi);
      for (int q = 0; q < R; ++q) b[j + q * P] = v[q];
    }
    for (int i = 0; i < N; ++i) a[i] = b[i];
    host_stages_v<N, V, S + 1, P * R, INV>(a, b, tw);
  }
}

#if defined(__CUDACC__)

template <int N, int V, int S, int P, bool INV>
BGP_D void warp_stages_v(double2* buf, const double2* __restrict__ tw, int lane) {
  constexpr RPlan pl = make_rplan_v<V>(N);
  if constexpr (S < pl.n) {
    constexpr int R = pl.r[S];
    constexpr int B = N / R;
    constexpr int U = (B + 31) / 32;
    double2 v[U][R];
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
    warp_stages_v<N, V, S + 1, P * R, INV>(buf, tw, lane);
  }
}

template <int N, bool INV, int V>
BGP_D void warp_fft_v(double2* buf, const double2* __restrict__ tw, int lane) {
  static_assert(make_rplan_v<V>(N).n > 0, "FFT length must be 2^a 3^b 5^c");
  warp_stages_v<N, V, 0, 1, INV>(buf, tw, lane);
}

#endif  // __CUDACC__

// ------------------------------------------------ register-resident line FFT
// -------------------------------------------------------------- tile geometry
// Shared-memory line pitch for LN lines of length L: element i of a line at
// swz(i); the pitch keeps the LN-lane row accesses of a strided tile on distinct
// banks (odd pitch for LN >= 8, 2 mod 8 for LN = 4).
BGP_HD constexpr int s_pitch(int L, int LN) {
  return (LN >= 8) ? ((L + L / 8 + 1) | 1) : (((L + L / 8 + 1 + 5) / 8) * 8 + 2);
}
BGP_HD constexpr size_t s_smem(int L, int LN) { return (size_t)LN * s_pitch(L, LN) * 16; }
// Convolution passes: the line buffers, then the tile's slab of the kernel
// quadrant, (M/2 + 1) values per line (doubles; the pitch is odd, so that the
// lanes of a line read distinct banks).
BGP_HD constexpr int s_kpitch(int M) { return (M / 2 + 1) | 1; }
BGP_HD constexpr size_t s_conv_smem(int M, int LN) {
  return s_smem(M, LN) + (((size_t)LN * s_kpitch(M) * 8 + 15) / 16) * 16;
}

// One instance of a stream batch (device copy).
struct SInst {
  int ndim, N, n, M, Mh, i0;
  double dx, kfac, s, tc, beta2, beta3, Omega, dv;
  const double2* psi;     // input state
  double2* A;             // per-axis accumulator (scratch, n)
  double2* H;             // output H psi
  const double* phi;      // long-range potential (n) or null
  double* part;           // per-tile partial sums of Re<psi, H psi> (last pass)
  // zero-padded convolution (phi from |psi|^2): scratch and kernel quadrant
  double2* cb1;           // 2D: N x Mh; 3D: N x N x Mh
  double2* cb2;           // 3D: N x M x Mh
  const double* Kq;       // real even quadrant of the kernel transform, (Mh)^d
  double* phi_out;        // computed potential (n)
  double conv_scale;      // -G_C dV / M^d
  const double2* twN;
  const double2* twM;
};

// A launch of one pass over up to kStreamBatch instances of one size, passed by
// value (kernel parameter space), so nothing is staged in device memory per call.
constexpr int kStreamBatch = 64;
struct SLaunch {
  SInst insts[kStreamBatch];
  int ninst;
  int tiles;              // tiles of one instance in this pass
};

// lines of the last (contiguous) axis of an instance
BGP_HD int ndim_lines(const SInst& I) { return I.ndim == 2 ? I.N : I.N * I.N; }

// flat index of element r of line c of tile t along axis ax (N-lines)
template <int LN>
BGP_D int s_elem(int ndim, int N, int ax, int t, int r, int c, int& i, int& j, int& k) {
  if (ndim == 2) {
    k = 0;
    if (ax == 1) { i = t * LN + c; j = r; } else { j = t * LN + c; i = r; }
    return i * N + j;
  }
  const int tpl = N / LN;
  if (ax == 2) { const int line = t * LN + c; i = line / N; j = line - i * N; k = r; }
  else if (ax == 1) { i = t / tpl; k = (t - i * tpl) * LN + c; j = r; }
  else { j = t / tpl; k = (t - j * tpl) * LN + c; i = r; }
  return (i * N + j) * N + k;
}

#if defined(__CUDACC__)

template <int L, int LN, bool CONTIG>
BGP_D void s_map(int e, int& r, int& c) {
  if (CONTIG) { c = e / L; r = e - c * L; } else { r = e / LN; c = e - r * LN; }
}

// --------------------------------------------------------------- H psi pass
// stage 0: A = T(psi) on the first (contiguous) axis; 1: A += T(psi) (3D middle);
// 2: H = A + T(psi) + (V + b2 rho + b3 rho^2 + phi) psi and the CTA's part of
// Re<psi, H> (axis 0). T = inverse FFT o multiplier o forward FFT along the axis.
// Transform of one warp's line b (shared memory, natural order) by radix order
// V (0-2: Stockham stages in shared memory, 3: the register-resident transform).
// mode 0: forward only; 1: inverse only; 2: forward, v <- mult(k, v), inverse.
// The result is left in b in natural order.
template <int L, int V, class F>
BGP_D void line_xform(double2* b, const double2* __restrict__ tw, int lane, int mode, F mult) {
  if constexpr (V == 3) {
    constexpr int R = L / 32;
    const int kb = R * rev5(lane);
    double2 v[R];
    if (mode == 1) {
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) v[k1] = b[swz(k1 + kb)];
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) v[q] = b[swz(lane + 32 * q)];
    }
    __syncwarp();
    if (mode != 1) reg_fft_fwd<L>(v, tw, lane);
    if (mode == 2) {
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) v[k1] = mult(k1 + kb, v[k1]);
    }
    if (mode != 0) reg_fft_inv<L>(v, tw, lane);
    if (mode == 0) {
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) b[swz(k1 + kb)] = v[k1];
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) b[swz(lane + 32 * q)] = v[q];
    }
    __syncwarp();
  } else {
    if (mode != 1) warp_fft_v<L, false, V>(b, tw, lane);
    if (mode == 2) {
      constexpr int PL = (L + 31) / 32;
#pragma unroll
      for (int q = 0; q < PL; ++q) {
        const int r = lane + 32 * q;
        if (L % 32 == 0 || r < L) b[swz(r)] = mult(r, b[swz(r)]);
      }
      __syncwarp();
    }
    if (mode != 0) warp_fft_v<L, true, V>(b, tw, lane);
  }
}

// Occupancy floor of the stream passes: 16 warps per SM (at most 128 registers).
template <int LN>
constexpr int s_min_blocks() { return (LN >= 16) ? 1 : 16 / LN; }

// V: 0-3 the line transform (see line_xform) at 16 warps per SM; 4-7 the same
// transform (V - 4) with the register budget halved for 32 warps per SM.
template <int N, int LN, int V>
__global__ void __launch_bounds__(LN * 32, (V >= 4 ? 2 : 1) * s_min_blocks<LN>()) k_stream_h(SLaunch SL, int ax,
                                                                                            int stage) {
  constexpr int VT = V & 3;   // the line transform
  extern __shared__ double2 sm[];
  constexpr int NT = LN * 32, TOT = LN * N, PER = (TOT + NT - 1) / NT, LS = s_pitch(N, LN);
  constexpr int CH = PER < 4 ? PER : 4;    // elements per thread in flight on the way out
  const int inst = blockIdx.x / SL.tiles, t = blockIdx.x - inst * SL.tiles;
  const SInst& I = SL.insts[inst];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int ndim = I.ndim;
  const bool contig = (ax == ndim - 1);
  const double2* __restrict__ psi = I.psi;
  auto where = [&](int e, int& r, int& c) {
    if (contig) s_map<N, LN, true>(e, r, c); else s_map<N, LN, false>(e, r, c);
  };
  if constexpr (VT == 3) {
    if (contig && stage == 0) {
      // contiguous lines straight from and to global memory: warp w owns line
      // t LN + w, lane l slot q element l + 32 q (coalesced in every q)
      constexpr int R = N / 32;
      const int line = t * LN + w;
      const size_t base = (size_t)line * N;
      double2 v[R];
#pragma unroll
      for (int q = 0; q < R; ++q) v[q] = __ldg(psi + base + lane + 32 * q);
      reg_fft_fwd<N>(v, I.twN, lane);
      // 2D y-line: wx = -Omega x(i), i = line; 3D z-line: no rotation term
      const double wx = (ndim == 2) ? -I.Omega * ((double)(line - N / 2) * I.dx) : 0.0;
      const double inv = 1.0 / (double)N, kf = I.kfac;
      const int kb = R * rev5(lane);
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) {
        const int kk_i = k1 + kb;
        const int mm = (kk_i < (N + 1) / 2) ? kk_i : kk_i - N;
        const double kk = kTwoPi * ((double)mm * kf);
        v[k1] = cscale(v[k1], (0.5 * kk * kk + wx * kk) * inv);
      }
      reg_fft_inv<N>(v, I.twN, lane);
#pragma unroll
      for (int q = 0; q < R; ++q) I.A[base + lane + 32 * q] = v[q];
      return;
    }
  }
  // load the tile: every load of the thread first, then into shared memory
  {
    double2 va[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * NT;
      if (TOT % NT == 0 || e < TOT) {
        int r, c, i, j, k;
        where(e, r, c);
        va[q] = __ldg(psi + s_elem<LN>(ndim, N, ax, t, r, c, i, j, k));
      }
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * NT;
      if (TOT % NT == 0 || e < TOT) {
        int r, c;
        where(e, r, c);
        sm[c * LS + swz(r)] = va[q];
      }
    }
  }
  __syncthreads();
  {
    double2* b = sm + w * LS;
    int i, j, k;
    s_elem<LN>(ndim, N, ax, t, 0, w, i, j, k);
    const double dx = I.dx, Om = I.Omega;
    const double wx = (ax == 1) ? -Om * ((double)(i - N / 2) * dx)
                                : ((ax == 0) ? Om * ((double)(j - N / 2) * dx) : 0.0);
    const double inv = 1.0 / (double)N, kf = I.kfac;
    line_xform<N, VT>(b, I.twN, lane, 2, [&](int r, double2 x) {
      const int mm = (r < (N + 1) / 2) ? r : r - N;
      const double kk = kTwoPi * ((double)mm * kf);
      return cscale(x, (0.5 * kk * kk + wx * kk) * inv);
    });
  }
  __syncthreads();
  double acc = 0.0;
#pragma unroll 1
  for (int q0 = 0; q0 < PER; q0 += CH) {
    // issue the chunk's loads (A, and psi and phi on the last axis), then use them
    double2 pa[CH], pv[CH];
    double pp[CH];
    int f[CH];
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      const int e = tid + (q0 + u) * NT;
      f[u] = -1;
      if (q0 + u < PER && (TOT % NT == 0 || e < TOT)) {
        int r, c, i, j, k;
        where(e, r, c);
        f[u] = s_elem<LN>(ndim, N, ax, t, r, c, i, j, k);
        if (stage > 0) pa[u] = I.A[f[u]];
        if (stage == 2) {
          pv[u] = __ldg(psi + f[u]);
          pp[u] = I.phi ? __ldg(I.phi + f[u]) : 0.0;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < CH; ++u) {
      if (f[u] < 0) continue;
      const int e = tid + (q0 + u) * NT;
      int r, c, i, j, k;
      where(e, r, c);
      const double2 v = sm[c * LS + swz(r)];
      if (stage == 0) { I.A[f[u]] = v; continue; }
      const double2 a2 = cadd(pa[u], v);
      if (stage == 1) { I.A[f[u]] = a2; continue; }
      s_elem<LN>(ndim, N, ax, t, r, c, i, j, k);
      const double2 p = pv[u];
      const double rho = cabs2(p);
      // trap tc r^s from the indices (becgpp/grid.py:90-91)
      const double x = (double)(i - N / 2) * I.dx, y = (double)(j - N / 2) * I.dx;
      double r2 = x * x + y * y;
      if (ndim == 3) { const double z = (double)(k - N / 2) * I.dx; r2 = r2 + z * z; }
      const double Vt = (I.s <= 0.0) ? 0.0 : ((I.s == 2.0) ? I.tc * r2 : I.tc * pow(r2, 0.5 * I.s));
      const double pot = Vt + I.beta2 * rho + I.beta3 * rho * rho + pp[u];
      const double2 h = cadd(a2, cscale(p, pot));
      I.H[f[u]] = h;
      acc += p.x * h.x + p.y * h.y;
    }
  }
  if (stage == 2 && I.part) {
    __shared__ double red[LN];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[w] = acc;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < LN; ++q) s += red[q];
      I.part[t] = s;
    }
  }
}

// ------------------------------------------------- zero-padded convolution
// The padded density of an instance lives in the M^d box with the N^d grid at
// offset i0 = (M - N)/2; only M/2+1 spectral columns of the last axis are kept
// (the input is real), only the N^d central outputs are written, and K^ is read
// from its real even quadrant Kq.
//   step a  (2D/3D): lines of the last axis, padded: FFT, keep kj <= M/2 -> cb1
//   step b  (2D): columns kj along i: FFT, times K^, inverse FFT, central i -> cb1
//   3D: step b fwd (j-lines) cb1 -> cb2, step c (i-lines: FFT, K^, IFFT) in cb2,
//       step b inv (j-lines) cb2 -> cb1 (central j)
//   last   : lines of the last axis: Hermitian rebuild, inverse FFT, central part:
//            phi = conv_scale * Re
// op: 0 step a, 1 2D step b, 2 3D step b fwd, 3 3D step c, 4 3D step b inv, 5 last.
template <int M, int LN, int V>
__global__ void __launch_bounds__(LN * 32, s_min_blocks<LN>()) k_stream_conv(SLaunch SL, int op) {
  extern __shared__ double2 sm[];
  constexpr int NT = LN * 32, TOT = LN * M, PER = (TOT + NT - 1) / NT, LS = s_pitch(M, LN);
  const int inst = blockIdx.x / SL.tiles, t = blockIdx.x - inst * SL.tiles;
  const SInst& I = SL.insts[inst];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int N = I.N, Mh = I.Mh, i0 = I.i0;
  const bool contig = (op == 0 || op == 5);
  const int tpl = (Mh + LN - 1) / LN;
  // decode (a, b) of the tile's line c for the strided ops
  auto line_ab = [&](int c, int& a, int& b2) {
    if (op == 1) { a = t * LN + c; b2 = 0; }                  // 2D column kj
    else { a = t / tpl; b2 = (t - a * tpl) * LN + c; }       // 3D: (i or jj, kk)
  };
  // kernel multiply (ops 1, 3): K^ is real and even, so line c needs the
  // M/2 + 1 values K^[a, ...] of its quadrant; the LN lines of a tile are
  // consecutive in the quadrant's contiguous index, so the slab is read as runs
  // of LN doubles, issued with the tile's own loads
  constexpr int KH = M / 2 + 1, KP = s_kpitch(M), KTOT = KH * LN, KPER = (KTOT + NT - 1) / NT;
  double* ks = reinterpret_cast<double*>(sm + LN * LS);
  const bool kmul = (op == 1 || op == 3);
  const size_t mh = (size_t)Mh;
  double kv[KPER];
  if (kmul) {
    int a1 = 0, a2 = 0;
    line_ab(0, a1, a2);
    const int bj = (a1 <= M / 2) ? a1 : M - a1;
#pragma unroll
    for (int q = 0; q < KPER; ++q) {
      const int e = tid + q * NT;
      kv[q] = 0.0;
      if (KTOT % NT == 0 || e < KTOT) {
        const int a = e / LN, c = e - a * LN;
        // op 1: column kj = a1 + c of row a; op 3: (a, bj, kk = a2 + c)
        const int col = (op == 1 ? a1 : a2) + c;
        if (col < Mh) kv[q] = __ldg(I.Kq + ((op == 1) ? (size_t)a * mh : ((size_t)a * mh + bj) * mh) + col);
      }
    }
  }
  double2 va[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = tid + q * NT;
    va[q] = cmk(0.0, 0.0);
    if (!(TOT % NT == 0 || e < TOT)) continue;
    int r, c;
    if (contig) s_map<M, LN, true>(e, r, c); else s_map<M, LN, false>(e, r, c);
    if (op == 0) {
      const int line = t * LN + c, j = r - i0;
      if (j >= 0 && j < N && line < (ndim_lines(I))) {
        const double2 p = __ldg(I.psi + (size_t)line * N + j);
        va[q] = cmk(cabs2(p), 0.0);
      }
    } else if (op == 5) {
      const int line = t * LN + c;
      if (line < ndim_lines(I)) {
        const double2* row = I.cb1 + (size_t)line * Mh;
        if (r < Mh) va[q] = row[r];
        else { const double2 v = row[M - r]; va[q] = cmk(v.x, -v.y); }
      }
    } else if (op == 1) {
      int kj, u;
      line_ab(c, kj, u);
      const int i = r - i0;
      if (kj < Mh && i >= 0 && i < N) va[q] = I.cb1[(size_t)i * Mh + kj];
    } else if (op == 2) {
      int i, kk;
      line_ab(c, i, kk);
      const int j = r - i0;
      if (kk < Mh && j >= 0 && j < N) va[q] = I.cb1[((size_t)i * N + j) * Mh + kk];
    } else if (op == 3) {
      int jj, kk;
      line_ab(c, jj, kk);
      const int i = r - i0;
      if (kk < Mh && i >= 0 && i < N) va[q] = I.cb2[((size_t)i * M + jj) * Mh + kk];
    } else {  // op 4
      int i, kk;
      line_ab(c, i, kk);
      if (kk < Mh) va[q] = I.cb2[((size_t)i * M + r) * Mh + kk];
    }
  }
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = tid + q * NT;
    if (TOT % NT == 0 || e < TOT) {
      int r, c;
      if (contig) s_map<M, LN, true>(e, r, c); else s_map<M, LN, false>(e, r, c);
      sm[c * LS + swz(r)] = va[q];
    }
  }
  if (kmul) {
#pragma unroll
    for (int q = 0; q < KPER; ++q) {
      const int e = tid + q * NT;
      if (KTOT % NT == 0 || e < KTOT) {
        const int a = e / LN, c = e - a * LN;
        ks[c * KP + a] = kv[q];
      }
    }
  }
  __syncthreads();
  {
    double2* b = sm + w * LS;
    const double2* tw = I.twM;
    const int mode = (op == 5 || op == 4) ? 1 : ((op == 0 || op == 2) ? 0 : 2);
    int a1 = 0, a2 = 0;
    if (mode == 2) line_ab(w, a1, a2);
    const bool valid = (op == 1) ? (a1 < Mh) : (a2 < Mh);
    const double* kl = ks + w * KP;
    line_xform<M, V>(b, tw, lane, mode, [&](int r, double2 x) {
      if (!valid) return x;
      return cscale(x, kl[(r <= M / 2) ? r : M - r]);
    });
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = tid + q * NT;
    if (!(TOT % NT == 0 || e < TOT)) continue;
    int r, c;
    if (contig) s_map<M, LN, true>(e, r, c); else s_map<M, LN, false>(e, r, c);
    const double2 v = sm[c * LS + swz(r)];
    if (op == 0) {
      const int line = t * LN + c;
      if (r < Mh && line < ndim_lines(I)) I.cb1[(size_t)line * Mh + r] = v;
    } else if (op == 5) {
      const int line = t * LN + c, j = r - i0;
      if (j >= 0 && j < N && line < ndim_lines(I)) I.phi_out[(size_t)line * N + j] = I.conv_scale * v.x;
    } else if (op == 1) {
      int kj, u;
      line_ab(c, kj, u);
      const int i = r - i0;
      if (kj < Mh && i >= 0 && i < N) I.cb1[(size_t)i * Mh + kj] = v;
    } else if (op == 2) {
      int i, kk;
      line_ab(c, i, kk);
      if (kk < Mh) I.cb2[((size_t)i * M + r) * Mh + kk] = v;
    } else if (op == 3) {
      int jj, kk;
      line_ab(c, jj, kk);
      const int i = r - i0;
      if (kk < Mh && i >= 0 && i < N) I.cb2[((size_t)i * M + jj) * Mh + kk] = v;
    } else {  // op 4
      int i, kk;
      line_ab(c, i, kk);
      const int j = r - i0;
      if (kk < Mh && j >= 0 && j < N) I.cb1[((size_t)i * N + j) * Mh + kk] = v;
    }
  }
}

#endif  // __CUDACC__

BGP_NS_END  // namespace bgp
