// Tiled line passes. Each operator supplies load(tile, r, c) -> value placed in
// shared memory, line(buf, lane, tile, warp) run by one warp on one line, and
// (optionally) store(tile, r, c, value). Operands come from the shared PassArgs
// block; reductions go to the operator's Acc.
#pragma once
#include "bgp_device.cuh"

namespace bgp {

// Reduction-record slots of the energy sums (trial / energy passes)
enum : int { S_N0 = 0, S_V = 1, S_2 = 2, S_3 = 3, S_KX = 4, S_KY = 5, S_KZ = 6, S_LY = 7, S_LX = 8,
             S_G = 9, S_R2 = 10, S_PERP = 11, S_Z2 = 12 };

// One tile: every thread first issues all of its global loads (independent, so
// they are in flight together), then fills shared memory; each warp transforms
// its line; the stores are issued the same way.
template <int L, bool CONTIG, class Op>
BGP_D void tile_run(Op& op, double2* sm, int t) {
  constexpr int TOT = 8 * L;
  constexpr int PER = (TOT + kThreads - 1) / kThreads;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  double2 v[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * kThreads;
    if (TOT % kThreads == 0 || e < TOT) {
      int r, c;
      if (CONTIG) map_contig<L>(e, r, c); else map_strided<L>(e, r, c);
      v[u] = op.load(t, r, c);
    }
  }
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * kThreads;
    if (TOT % kThreads == 0 || e < TOT) {
      int r, c;
      if (CONTIG) map_contig<L>(e, r, c); else map_strided<L>(e, r, c);
      sm[c * (L + kPad) + r] = v[u];
    }
  }
  __syncthreads();
  op.line(sm + w * (L + kPad), lane, t, w);
  __syncthreads();
  if (Op::kStore) {
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = tid + u * kThreads;
      if (TOT % kThreads == 0 || e < TOT) {
        int r, c;
        if (CONTIG) map_contig<L>(e, r, c); else map_strided<L>(e, r, c);
        v[u] = sm[c * (L + kPad) + r];
      }
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = tid + u * kThreads;
      if (TOT % kThreads == 0 || e < TOT) {
        int r, c;
        if (CONTIG) map_contig<L>(e, r, c); else map_strided<L>(e, r, c);
        op.store(t, r, c, v[u]);
      }
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------ H psi passes
// stage 0: A = IFFT(m FFT psi) along the first (contiguous) axis
// stage 1: A += ...   (3D middle axis)
// stage 2: H = A + IFFT(m FFT psi) + (V + b2 rho + b3 rho^2 + phi) psi  (axis 0)
// with m = (k^2/2 - Omega X k) on y, (k^2/2 + Omega Y k) on x, k^2/2 on z: the
// kinetic term and -Omega L_z are separable into 1D spectral multipliers.
template <int N>
struct OpH {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D double2 load(int t, int r, int c) {
    int i, j, k;
    return psi_at(Q, nline_elem(I, Q.ax, t, r, c, i, j, k));
  }
  BGP_D void line(double2* b, int lane, int t, int w) {
    warp_fft<N, false>(b, I.twN, lane);
    int i, j, k;
    const int ax = Q.ax;
    nline_elem(I, ax, t, 0, w, i, j, k);
    const double wx = (ax == 1) ? -I.Omega * xcoord(I, i) : ((ax == 0) ? I.Omega * xcoord(I, j) : 0.0);
    const double inv = 1.0 / (double)N;
#pragma unroll 4
    for (int r = lane; r < N; r += 32) {
      const double kk = kof(I, r);
      const double m = 0.5 * kk * kk + wx * kk;
      b[r] = cscale(b[r], m * inv);
    }
    __syncwarp();
    warp_fft<N, true>(b, I.twN, lane);
  }
  BGP_D void store(int t, int r, int c, double2 v) {
    int i, j, k;
    const int f = nline_elem(I, Q.ax, t, r, c, i, j, k);
    if (Q.stage == 0) { st2(Q.A + f, v); return; }
    if (Q.stage == 1) { st2(Q.A + f, cadd(ld2(Q.A + f), v)); return; }
    const double2 p = psi_at(Q, f);
    const double rho = cabs2(p);
    double pot = potential(I, i, j, k) + I.beta2 * rho + I.beta3 * rho * rho;
    if (Q.phi) pot += Q.phisc * ld1(Q.phi + f);
    const double2 h = cadd(cadd(ld2(Q.A + f), v), cscale(p, pot));
    st2(Q.H + f, h);
    acc.s[0] += p.x * h.x + p.y * h.y;
    acc.mx = fmax(acc.mx, rho);
  }
};

// ------------------------------------------------------------- energy sums pass
// Along axis ax: the spectral sums  sum k^2 |w^|^2  and the L_z weights
// (X sum k_y |w^|^2 on y lines, Y sum k_x |w^|^2 on x lines; Parseval along one
// axis). On the first axis the state w = psi - t dirc (or the input state) is
// formed, optionally stored, and the local sums of |w|^2 are taken.
template <int N>
struct OpT {
  static constexpr bool kStore = false;
  const Inst& I;
  const PassArgs& Q;
  int ax;
  Acc acc;
  BGP_D double2 load(int tt, int r, int c) {
    int i, j, k;
    const int f = nline_elem(I, ax, tt, r, c, i, j, k);
    if (ax != I.ndim - 1) return ld2(Q.src + f);
    double2 w;
    if (Q.init) {
      w = ld2(Q.cin + f);
    } else {
      double2 d;
      if (Q.write_dirc) { d = dirc_at(Q, f); st2(Q.DIRC + f, d); }
      else d = ld2(Q.DIRC + f);
      w = csub(psi_at(Q, f), cscale(d, Q.t));
    }
    if (Q.write_w) st2(Q.W + f, w);
    const double q = cabs2(w);
    const double x = xcoord(I, i), y = xcoord(I, j);
    acc.s[S_N0] += q;
    acc.s[S_V] += potential(I, i, j, k) * q;
    acc.s[S_2] += q * q;
    acc.s[S_3] += q * q * q;
    const double rp = x * x + y * y;
    double r2 = rp;
    if (I.ndim == 3) {
      const double z = xcoord(I, k);
      r2 = r2 + z * z;
      acc.s[S_PERP] += rp * q;
      acc.s[S_Z2] += z * z * q;
    }
    acc.s[S_R2] += r2 * q;
    acc.mx = fmax(acc.mx, q);
    return w;
  }
  BGP_D void line(double2* b, int lane, int tt, int w) {
    warp_fft<N, false>(b, I.twN, lane);
    int i, j, k;
    nline_elem(I, ax, tt, 0, w, i, j, k);
    double sk = 0.0, sl = 0.0;
    for (int r = lane; r < N; r += 32) {
      const double kk = kof(I, r);
      const double a2 = cabs2(b[r]);
      sk += kk * kk * a2;
      sl += kk * a2;
    }
    if (ax == 0) { acc.s[S_KX] += sk; acc.s[S_LX] += xcoord(I, j) * sl; }
    else if (ax == 1) { acc.s[S_KY] += sk; acc.s[S_LY] += xcoord(I, i) * sl; }
    else acc.s[S_KZ] += sk;
  }
  BGP_D void store(int, int, int, double2) {}
};

// ---------------------------------------------------- gradient + first FFT pass
// g = H - mu psi (or the given gradient); stores g, sums |g|^2, writes the median
// keys of  V + 2 b2 rho + 3 b3 rho^2 (+ phi)  over rho > thr, and transforms g
// along the contiguous axis into A.
template <int N>
struct OpG {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D double2 load(int t, int r, int c) {
    int i, j, k;
    const int f = nline_elem(I, I.ndim - 1, t, r, c, i, j, k);
    const double2 p = psi_at(Q, f);
    double2 g;
    if (Q.gin) g = ld2(Q.gin + f);
    else g = csub(ld2(Q.H + f), cscale(p, Q.mu));
    if (Q.Gout) st2(Q.Gout + f, g);
    acc.s[0] += cabs2(g);
    if (Q.keys_on) {
      const double rho = cabs2(p);
      unsigned long long key = 0ull;
      if (rho > Q.thr) {
        double loc = potential(I, i, j, k) + 2.0 * I.beta2 * rho + 3.0 * I.beta3 * (rho * rho);
        if (Q.phi) loc = loc + Q.phisc * ld1(Q.phi + f);
        key = dkey(loc);
        atomicAdd(&Q.shist[key >> 56], 1u);
        if (Q.win_on) {
          if (key < Q.win_lo) {
            acc.s[1] += 1.0;
          } else if (key <= Q.win_hi) {
            const unsigned idx = atomicAdd(&I.hist[8 * 256 + 1], 1u);
            if (idx < (unsigned)kSelCap) I.wcand[idx] = key;
          }
        }
      }
      I.keys[f] = key;
    }
    return g;
  }
  BGP_D void line(double2* b, int lane, int, int) { warp_fft<N, false>(b, I.twN, lane); }
  BGP_D void store(int t, int r, int c, double2 v) {
    int i, j, k;
    st2(Q.A + nline_elem(I, I.ndim - 1, t, r, c, i, j, k), v);
  }
};

// ------------------------------------------------------ preconditioner passes
// mode 0: forward FFT; 1: forward, divide by (K2/2 + sigma), inverse;
// 2: inverse; 3: inverse, scale 1/n, store z and sum conj(psi) z.
template <int N>
struct OpP {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D double2 load(int t, int r, int c) {
    int i, j, k;
    return ld2(Q.A + nline_elem(I, Q.ax, t, r, c, i, j, k));
  }
  BGP_D void line(double2* b, int lane, int t, int w) {
    const int mode = Q.mode;
    if (mode <= 1) warp_fft<N, false>(b, I.twN, lane);
    if (mode == 1) {
      int i, j, k;
      nline_elem(I, Q.ax, t, 0, w, i, j, k);
      const double ky = kof(I, j);
      const double kz = (I.ndim == 3) ? kof(I, k) : 0.0;
      const double sigma = Q.sigma;
      for (int r = lane; r < N; r += 32) {
        const double kx = kof(I, r);
        double K2 = kx * kx + ky * ky;
        if (I.ndim == 3) K2 = K2 + kz * kz;
        const double den = 0.5 * K2 + sigma;
        b[r] = cmk(b[r].x / den, b[r].y / den);
      }
      __syncwarp();
    }
    if (mode >= 1) warp_fft<N, true>(b, I.twN, lane);
  }
  BGP_D void store(int t, int r, int c, double2 v) {
    int i, j, k;
    const int f = nline_elem(I, Q.ax, t, r, c, i, j, k);
    if (Q.mode < 3) { st2(Q.A + f, v); return; }
    const double2 z = cscale(v, I.inv_n);
    st2(Q.Z + f, z);
    const double2 pz = cconjmul(psi_at(Q, f), z);
    acc.s[0] += pz.x;
    acc.s[1] += pz.y;
  }
};

// -------------------------------------------------- zero-padded convolution
// 2D, step a: rows i of the padded density, FFT along j, keep kj <= M/2.
// 3D, step a: lines (i,j), FFT along k, keep kk <= M/2 (same code: line = t*8+c).
template <int M>
struct OpCa {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  BGP_D double2 load(int t, int r, int c) {
    const int line = t * 8 + c, j = r - I.i0;
    if (j < 0 || j >= I.N) return cmk(0.0, 0.0);
    return cmk(rho_at(Q, Q.rmode, line * I.N + j), 0.0);
  }
  BGP_D void line(double2* b, int lane, int, int) { warp_fft<M, false>(b, I.twM, lane); }
  BGP_D void store(int t, int r, int c, double2 v) {
    if (r < I.Mh) st2(I.cb1 + (size_t)(t * 8 + c) * I.Mh + r, v);
  }
};

// 2D, step b: columns kj, FFT along i (padded), multiply by the kernel, inverse.
template <int M>
struct OpC2b {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  BGP_D double2 load(int t, int r, int c) {
    const int kj = t * 8 + c, i = r - I.i0;
    if (kj >= I.Mh || i < 0 || i >= I.N) return cmk(0.0, 0.0);
    return ld2(I.cb1 + (size_t)i * I.Mh + kj);
  }
  BGP_D void line(double2* b, int lane, int t, int w) {
    warp_fft<M, false>(b, I.twM, lane);
    const int kj = t * 8 + w;
    if (kj < I.Mh) {
      const double* Kq = Q.Kq;
      for (int r = lane; r < M; r += 32) {
        const int a = (r <= M / 2) ? r : M - r;
        b[r] = cscale(b[r], __ldg(Kq + (size_t)a * I.Mh + kj));
      }
    }
    __syncwarp();
    warp_fft<M, true>(b, I.twM, lane);
  }
  BGP_D void store(int t, int r, int c, double2 v) {
    const int kj = t * 8 + c, i = r - I.i0;
    if (kj < I.Mh && i >= 0 && i < I.N) st2(I.cb1 + (size_t)i * I.Mh + kj, v);
  }
};

// Last step (2D rows / 3D k-lines): rebuild the Hermitian row spectrum, inverse
// FFT, keep the central N points: out = cscale * Re, and sum out * rho.
template <int M>
struct OpCinv {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D double2 load(int t, int r, int c) {
    const double2* row = I.cb1 + (size_t)(t * 8 + c) * I.Mh;
    if (r < I.Mh) return ld2(row + r);
    const double2 v = ld2(row + (M - r));
    return cmk(v.x, -v.y);
  }
  BGP_D void line(double2* b, int lane, int, int) { warp_fft<M, true>(b, I.twM, lane); }
  BGP_D void store(int t, int r, int c, double2 v) {
    const int j = r - I.i0;
    if (j < 0 || j >= I.N) return;
    const int f = (t * 8 + c) * I.N + j;
    const double val = Q.cscale * v.x;
    st1(Q.cout + f, val);
    if (Q.sum_on) acc.s[S_G] += val * rho_at(Q, Q.smode, f);
  }
};

// 3D step b (forward) / d (inverse): lines (i, kk) along j.
//   forward: cb1[i][j][kk] (j padded) -> FFT -> cb2[i][jj][kk]
//   inverse: cb2[i][jj][kk] -> IFFT -> central j -> cb1[i][j][kk]
template <int M>
struct OpC3b {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  BGP_D void decode(int t, int c, int& i, int& kk) const {
    const int tpl = (I.Mh + 7) >> 3;
    i = t / tpl;
    kk = (t - i * tpl) * 8 + c;
  }
  BGP_D double2 load(int t, int r, int c) {
    int i, kk;
    decode(t, c, i, kk);
    if (kk >= I.Mh) return cmk(0.0, 0.0);
    if (Q.inverse) return ld2(I.cb2 + ((size_t)i * M + r) * I.Mh + kk);
    const int j = r - I.i0;
    if (j < 0 || j >= I.N) return cmk(0.0, 0.0);
    return ld2(I.cb1 + ((size_t)i * I.N + j) * I.Mh + kk);
  }
  BGP_D void line(double2* b, int lane, int, int) {
    if (Q.inverse) warp_fft<M, true>(b, I.twM, lane);
    else warp_fft<M, false>(b, I.twM, lane);
  }
  BGP_D void store(int t, int r, int c, double2 v) {
    int i, kk;
    decode(t, c, i, kk);
    if (kk >= I.Mh) return;
    if (!Q.inverse) { st2(I.cb2 + ((size_t)i * M + r) * I.Mh + kk, v); return; }
    const int j = r - I.i0;
    if (j >= 0 && j < I.N) st2(I.cb1 + ((size_t)i * I.N + j) * I.Mh + kk, v);
  }
};

// 3D step c: lines (jj, kk) along i: FFT (padded), kernel multiply, IFFT.
template <int M>
struct OpC3c {
  static constexpr bool kStore = true;
  const Inst& I;
  const PassArgs& Q;
  BGP_D void decode(int t, int c, int& jj, int& kk) const {
    const int tpl = (I.Mh + 7) >> 3;
    jj = t / tpl;
    kk = (t - jj * tpl) * 8 + c;
  }
  BGP_D double2 load(int t, int r, int c) {
    int jj, kk;
    decode(t, c, jj, kk);
    const int i = r - I.i0;
    if (kk >= I.Mh || i < 0 || i >= I.N) return cmk(0.0, 0.0);
    return ld2(I.cb2 + ((size_t)i * M + jj) * I.Mh + kk);
  }
  BGP_D void line(double2* b, int lane, int t, int w) {
    warp_fft<M, false>(b, I.twM, lane);
    int jj, kk;
    decode(t, w, jj, kk);
    if (kk < I.Mh) {
      const int bj = (jj <= M / 2) ? jj : M - jj;
      const double* Kq = Q.Kq;
      for (int r = lane; r < M; r += 32) {
        const int a = (r <= M / 2) ? r : M - r;
        b[r] = cscale(b[r], __ldg(Kq + ((size_t)a * I.Mh + bj) * I.Mh + kk));
      }
    }
    __syncwarp();
    warp_fft<M, true>(b, I.twM, lane);
  }
  BGP_D void store(int t, int r, int c, double2 v) {
    int jj, kk;
    decode(t, c, jj, kk);
    const int i = r - I.i0;
    if (kk < I.Mh && i >= 0 && i < I.N) st2(I.cb2 + ((size_t)i * M + jj) * I.Mh + kk, v);
  }
};

}  // namespace bgp
