// Tiled line passes. A pass runs over tiles of kLines lines of one axis; each
// operator supplies
//   Pre    fetch(tile, r, c)              the loads element (r, c) needs on the way in
//   double2 enter(P, tile, r, c)          the value placed in shared memory (may store)
//   void   line(buf, lane, tile, warp)    one warp's work on one line
//   Pre    fetch_out(tile, r, c)          the loads the way out needs
//   void   leave(P, tile, r, c, value)    the way out (stores, sums)
// and the pass issues all loads of a batch before any of its stores, so loads
// never wait behind stores. Operands come from the shared PassArgs block;
// reductions go to the operator's Acc.
#pragma once
#include "bgp_device.cuh"

BGP_NS_BEGIN

// Reduction-record slots of the energy sums (trial / energy passes)
enum : int { S_N0 = 0, S_V = 1, S_2 = 2, S_3 = 3, S_KX = 4, S_KY = 5, S_KZ = 6, S_LY = 7, S_LX = 8,
             S_G = 9, S_R2 = 10, S_PERP = 11, S_Z2 = 12 };

// Members of an operator without loads on the way out; `chunk` = elements per
// fetch batch and thread.
#define BGP_NO_OUT(chunk)                                 \
  static constexpr int kChunk = (chunk);                  \
  static constexpr int kChunkOut = 64;                    \
  BGP_D Pre fetch_out(int, int, int) { return Pre{}; }

template <int L, bool CONTIG>
BGP_D void tile_map(int e, int& r, int& c) {
  if (CONTIG) map_contig<L>(e, r, c); else map_strided<L>(e, r, c);
}

// One tile of kLines lines. Loads are issued in batches of Op::kChunk elements per thread (all
// loads of a batch in flight together), then the batch is entered into shared
// memory; each warp transforms its line; the way out fetches every operand of
// the thread's elements, then stores.
template <int L, bool CONTIG, class T, class Op>
BGP_D void tile_run_t(Op& op, double2* smd, int t) {
  constexpr int TOT = kLines * L;
  constexpr int PER = (TOT + kThreads - 1) / kThreads;
  constexpr int LS = line_stride(L);
  constexpr int CH = (Op::kChunk < PER) ? Op::kChunk : PER;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  T* sm = reinterpret_cast<T*>(smd);
#pragma unroll
  for (int u0 = 0; u0 < PER; u0 += CH) {
    Pre pre[CH];
#pragma unroll
    for (int q = 0; q < CH; ++q) {
      const int e = tid + (u0 + q) * kThreads;
      if (u0 + q < PER && (TOT % kThreads == 0 || e < TOT)) {
        int r, c;
        tile_map<L, CONTIG>(e, r, c);
        pre[q] = op.fetch(t, r, c);
      }
    }
#pragma unroll
    for (int q = 0; q < CH; ++q) {
      const int e = tid + (u0 + q) * kThreads;
      if (u0 + q < PER && (TOT % kThreads == 0 || e < TOT)) {
        int r, c;
        tile_map<L, CONTIG>(e, r, c);
        sm[c * LS + swz(r)] = to_c<T>(op.enter(pre[q], t, r, c));
      }
    }
  }
  __syncthreads();
  op.line(sm + w * LS, lane, t, w);
  __syncthreads();
  if (Op::kStore) {
    constexpr int CO = (Op::kChunkOut < PER) ? Op::kChunkOut : PER;
#pragma unroll
    for (int u0 = 0; u0 < PER; u0 += CO) {
      Pre pre[CO];
      double2 v[CO];
#pragma unroll
      for (int q = 0; q < CO; ++q) {
        const int e = tid + (u0 + q) * kThreads;
        if (u0 + q < PER && (TOT % kThreads == 0 || e < TOT)) {
          int r, c;
          tile_map<L, CONTIG>(e, r, c);
          pre[q] = op.fetch_out(t, r, c);
          v[q] = to_d(sm[c * LS + swz(r)]);
        }
      }
#pragma unroll
      for (int q = 0; q < CO; ++q) {
        const int e = tid + (u0 + q) * kThreads;
        if (u0 + q < PER && (TOT % kThreads == 0 || e < TOT)) {
          int r, c;
          tile_map<L, CONTIG>(e, r, c);
          op.leave(pre[q], t, r, c, v[q]);
        }
      }
    }
  }
  __syncthreads();
}

// A tile in the operator's FP64 arithmetic, or with FP32 transforms when
// `fp32` is set, the operator supports them (Op::kMixed) and this is a
// mixed-precision build (BGP_MIXED).
template <int L, bool CONTIG, class Op>
BGP_D void tile_run(Op& op, double2* sm, int t, int fp32 = 0) {
  if constexpr (Op::kMixed && BGP_MIXED) {
    if (fp32) { tile_run_t<L, CONTIG, float2>(op, sm, t); return; }
  }
  tile_run_t<L, CONTIG, double2>(op, sm, t);
}

// Multiply line element r (r = lane, lane + 32, ...) by the real kernel value
// Kq[idx(r)]: every lane loads all of its kernel values first.
template <int M, class F>
BGP_D void line_times_kernel(double2* b, int lane, const double* Kq, F idx) {
  constexpr int PL = (M + 31) / 32;
  double kv[PL];
#pragma unroll
  for (int q = 0; q < PL; ++q) {
    const int r = lane + 32 * q;
    kv[q] = (M % 32 == 0 || r < M) ? __ldg(Kq + idx(r)) : 0.0;
  }
#pragma unroll
  for (int q = 0; q < PL; ++q) {
    const int r = lane + 32 * q;
    if (M % 32 == 0 || r < M) b[swz(r)] = cscale(b[swz(r)], kv[q]);
  }
}

// ------------------------------------------------------------------ H psi passes
// stage 0: A = IFFT(m FFT psi) along the first (contiguous) axis
// stage 1: A += ...   (3D middle axis)
// stage 2: H = A + IFFT(m FFT psi) + (V + b2 rho + b3 rho^2 + phi) psi  (axis 0)
// with m = (k^2/2 - Omega X k) on y, (k^2/2 + Omega Y k) on x, k^2/2 on z: the
// kinetic term and -Omega L_z are separable into 1D spectral multipliers.
// Every operator copies the scalars and pointers it uses into registers when it
// is constructed (after the phase's operands are published).
template <int N>
#define OPH_ARGS \
  [[maybe_unused]] const GeoT<N> g = geo_t<N>(I); \
  [[maybe_unused]] const double2* tw = I.twN; \
  [[maybe_unused]] const double2* psi = Q.psi; \
  [[maybe_unused]] double2* A = Q.A; \
  [[maybe_unused]] double2* H = Q.H; \
  [[maybe_unused]] const double* phi = Q.phi; \
  [[maybe_unused]] const double psc = Q.psc, phisc = Q.phisc; \
  [[maybe_unused]] const int ax = Q.ax, stage = Q.stage, sp = Q.fp32;
struct OpH {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = true;
  static constexpr int kChunk = 64;
  static constexpr int kChunkOut = 4;    // A, psi and phi per element on the way out
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D Pre fetch(int t, int r, int c) {
    OPH_ARGS
    int i, j, k;
    Pre P;
    P.a = cscale(ldp(psi, nline_elem(g, ax, t, r, c, i, j, k), sp), psc);
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int, int) { return P.a; }
  template <class T>
  BGP_D void line(T* b, int lane, int t, int w) {
    OPH_ARGS
    using Rt = typename CT<T>::R;
    const T* twt = twN_of<T>(I);
    warp_fft<N, false>(b, twt, lane);
    int i, j, k;
    nline_elem(g, ax, t, 0, w, i, j, k);
    const double wx = (ax == 1) ? -g.Omega * xcoord(g, i) : ((ax == 0) ? g.Omega * xcoord(g, j) : 0.0);
    const double inv = 1.0 / (double)N;
    constexpr int PL = (N + 31) / 32;
#pragma unroll 4
    for (int q = 0; q < PL; ++q) {
      const int r = lane + 32 * q;
      if (N % 32 == 0 || r < N) {
        const double kk = kof(g, r);
        const double m = 0.5 * kk * kk + wx * kk;
        b[swz(r)] = cscale(b[swz(r)], (Rt)(m * inv));
      }
    }
    __syncwarp();
    warp_fft<N, true>(b, twt, lane);
  }
  BGP_D Pre fetch_out(int t, int r, int c) {
    OPH_ARGS
    Pre P{};
    if (stage == 0) return P;
    int i, j, k;
    const int f = nline_elem(g, ax, t, r, c, i, j, k);
    P.b = ldp(A, f, sp);
    if (stage == 2) {
      P.a = cscale(ldp(psi, f, sp), psc);
      P.r = phi ? phisc * ld1(phi + f) : 0.0;
    }
    return P;
  }
  BGP_D void leave(const Pre& P, int t, int r, int c, double2 v) {
    OPH_ARGS
    int i, j, k;
    const int f = nline_elem(g, ax, t, r, c, i, j, k);
    if (stage == 0) { stp(A, f, v, sp); return; }
    if (stage == 1) { stp(A, f, cadd(P.b, v), sp); return; }
    const double2 p = P.a;
    const double rho = cabs2(p);
    const double pot = potential(g, i, j, k) + g.beta2 * rho + g.beta3 * rho * rho + P.r;
    const double2 h = cadd(cadd(P.b, v), cscale(p, pot));
    stp(H, f, h, sp);
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
#define OPT_ARGS \
  [[maybe_unused]] const GeoT<N> g = geo_t<N>(I); \
  [[maybe_unused]] const double2* tw = I.twN; \
  [[maybe_unused]] const DirArgs D = dir_args(Q); \
  [[maybe_unused]] const double2* src = Q.src; \
  [[maybe_unused]] const double2* cin = Q.cin; \
  [[maybe_unused]] double2* W = Q.W; \
  [[maybe_unused]] double2* DIRC = Q.DIRC; \
  [[maybe_unused]] const int init = Q.init, write_dirc = Q.write_dirc, write_w = Q.write_w, sp = Q.fp32;
struct OpT {
  static constexpr bool kStore = false;
  static constexpr bool kMixed = true;
  BGP_NO_OUT(4)                          // three complex operands per element
  const Inst& I;
  const PassArgs& Q;
  int ax;
  Acc acc;
  BGP_D Pre fetch(int tt, int r, int c) {
    OPT_ARGS
    int i, j, k;
    const int f = nline_elem(g, ax, tt, r, c, i, j, k);
    Pre P;
    // src: the stored trial state (pool; the caller's state when sp == 0 in mode 2)
    if (ax != BGP_DIM(g) - 1) { P.a = ldp(src, f, sp); return P; }
    if (init) { P.a = ld2(cin + f); return P; }      // the caller's state: complex128
    if (write_dirc) { dirc_fetch(D, f, P); return P; }
    P.a = cscale(ldp(D.psi, f, sp), D.psc);
    P.b = ldp(DIRC, f, sp);
    return P;
  }
  BGP_D double2 enter(const Pre& P, int tt, int r, int c) {
    OPT_ARGS
    if (ax != BGP_DIM(g) - 1) return P.a;
    int i, j, k;
    const int f = nline_elem(g, ax, tt, r, c, i, j, k);
    double2 w;
    if (init) {
      w = rnd_sp(P.a, sp);
    } else {
      double2 d;
      if (write_dirc) { d = rnd_sp(dirc_of(D, P), sp); stp(DIRC, f, d, sp); }
      else d = P.b;
      w = rnd_sp(csub(P.a, cscale(d, D.t)), sp);
    }
    if (write_w) stp(W, f, w, sp);
    const double q = cabs2(w);
    const double x = xcoord(g, i), y = xcoord(g, j);
    acc.s[S_N0] += q;
    acc.s[S_V] += potential(g, i, j, k) * q;
    acc.s[S_2] += q * q;
    acc.s[S_3] += q * q * q;
    const double rp = x * x + y * y;
    double r2 = rp;
    if (BGP_DIM(g) == 3) {
      const double z = xcoord(g, k);
      r2 = r2 + z * z;
      acc.s[S_PERP] += rp * q;
      acc.s[S_Z2] += z * z * q;
    }
    acc.s[S_R2] += r2 * q;
    acc.mx = fmax(acc.mx, q);
    return w;
  }
  template <class T>
  BGP_D void line(T* b, int lane, int tt, int w) {
    OPT_ARGS
    warp_fft<N, false>(b, twN_of<T>(I), lane);
    int i, j, k;
    nline_elem(g, ax, tt, 0, w, i, j, k);
    double sk = 0.0, sl = 0.0;
    constexpr int PL = (N + 31) / 32;
#pragma unroll
    for (int q = 0; q < PL; ++q) {
      const int r = lane + 32 * q;
      if (N % 32 == 0 || r < N) {
        const double kk = kof(g, r);
        const double a2 = cabs2(b[swz(r)]);
        sk += kk * kk * a2;
        sl += kk * a2;
      }
    }
    if (ax == 0) { acc.s[S_KX] += sk; acc.s[S_LX] += xcoord(g, j) * sl; }
    else if (ax == 1) { acc.s[S_KY] += sk; acc.s[S_LY] += xcoord(g, i) * sl; }
    else acc.s[S_KZ] += sk;
  }
  BGP_D void leave(const Pre&, int, int, int, double2) {}
};

// ---------------------------------------------------- gradient + first FFT pass
// g = H - mu psi (or the given gradient); stores g, sums |g|^2, writes the median
// keys of  V + 2 b2 rho + 3 b3 rho^2 (+ phi)  over rho > thr, and transforms g
// along the contiguous axis into A.
template <int N>
#define OPG_ARGS \
  [[maybe_unused]] const GeoT<N> g = geo_t<N>(I); \
  [[maybe_unused]] const double2* tw = I.twN; \
  [[maybe_unused]] const double2* psi = Q.psi; \
  [[maybe_unused]] const double2* gin = Q.gin; \
  [[maybe_unused]] const double2* Hin = Q.H; \
  [[maybe_unused]] double2* Gout = Q.Gout; \
  [[maybe_unused]] double2* A = Q.A; \
  [[maybe_unused]] const double* phi = Q.phi; \
  [[maybe_unused]] unsigned* shist = Q.shist; \
  [[maybe_unused]] unsigned long long* keys = I.keys; \
  [[maybe_unused]] unsigned* wcount = I.hist + 8 * 256 + 1; \
  [[maybe_unused]] unsigned long long* wcand = I.wcand; \
  [[maybe_unused]] const double psc = Q.psc, mu = Q.mu, thr = Q.thr, phisc = Q.phisc; \
  [[maybe_unused]] const unsigned long long win_lo = Q.win_lo, win_hi = Q.win_hi; \
  [[maybe_unused]] const int keys_on = Q.keys_on, win_on = Q.win_on, sp = Q.fp32;
struct OpG {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = true;
  BGP_NO_OUT(4)
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D int elem(int t, int r, int c, int& i, int& j, int& k) const {
    OPG_ARGS
    return nline_elem(g, BGP_DIM(g) - 1, t, r, c, i, j, k);
  }
  BGP_D Pre fetch(int t, int r, int c) {
    OPG_ARGS
    int i, j, k;
    const int f = elem(t, r, c, i, j, k);
    Pre P;
    P.a = cscale(ldp(psi, f, sp), psc);
    P.b = gin ? ld2(gin + f) : ldp(Hin, f, sp);      // a given gradient is the caller's
    P.r = (keys_on && phi) ? ld1(phi + f) : 0.0;
    return P;
  }
  BGP_D double2 enter(const Pre& P, int t, int r, int c) {
    OPG_ARGS
    int i, j, k;
    const int f = elem(t, r, c, i, j, k);
    const double2 p = P.a;
    const double2 gr = gin ? P.b : csub(P.b, cscale(p, mu));
    if (Gout) stp(Gout, f, gr, sp);
    acc.s[0] += cabs2(gr);
    if (keys_on) {
      const double rho = cabs2(p);
      unsigned long long key = 0ull;
      if (rho > thr) {
        double loc = potential(g, i, j, k) + 2.0 * g.beta2 * rho + 3.0 * g.beta3 * (rho * rho);
        if (phi) loc = loc + phisc * P.r;
        key = dkey(loc);
        acc.s[3] += 1.0;
        atomicAdd(&shist[key >> 56], 1u);
        if (win_on) {
          if (key < win_lo) {
            acc.s[1] += 1.0;
          } else if (key <= win_hi) {
            acc.s[4] += 1.0;
            const unsigned idx = atomicAdd(wcount, 1u);
            if (idx < (unsigned)kSelCap) wcand[idx] = key;
          }
        }
      }
      keys[f] = key;
    }
    return gr;
  }
  template <class T>
  BGP_D void line(T* b, int lane, int, int) { warp_fft<N, false>(b, twN_of<T>(I), lane); }
  BGP_D void leave(const Pre&, int t, int r, int c, double2 v) {
    OPG_ARGS
    int i, j, k;
    stp(A, elem(t, r, c, i, j, k), v, sp);
  }
};

// ------------------------------------------------------ preconditioner passes
// mode 0: forward FFT; 1: forward, divide by (K2/2 + sigma), inverse;
// 2: inverse; 3: inverse, scale 1/n, store z and sum conj(psi) z.
template <int N>
#define OPP_ARGS \
  [[maybe_unused]] const GeoT<N> g = geo_t<N>(I); \
  [[maybe_unused]] const double2* tw = I.twN; \
  [[maybe_unused]] const double2* psi = Q.psi; \
  [[maybe_unused]] double2* A = Q.A; \
  [[maybe_unused]] double2* Z = Q.Z; \
  [[maybe_unused]] const double psc = Q.psc, sigma = Q.sigma, inv_n = I.inv_n; \
  [[maybe_unused]] const int ax = Q.ax, mode = Q.mode, sp = Q.fp32;
struct OpP {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = true;
  static constexpr int kChunk = 64;
  static constexpr int kChunkOut = 8;
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D Pre fetch(int t, int r, int c) {
    OPP_ARGS
    int i, j, k;
    Pre P;
    P.a = ldp(A, nline_elem(g, ax, t, r, c, i, j, k), sp);
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int, int) { return P.a; }
  template <class T>
  BGP_D void line(T* b, int lane, int t, int w) {
    OPP_ARGS
    using Rt = typename CT<T>::R;
    const T* twt = twN_of<T>(I);
    if (mode <= 1) warp_fft<N, false>(b, twt, lane);
    if (mode == 1) {
      int i, j, k;
      nline_elem(g, ax, t, 0, w, i, j, k);
      const double ky = kof(g, j);
      const double kz = (BGP_DIM(g) == 3) ? kof(g, k) : 0.0;
      constexpr int PL = (N + 31) / 32;
#pragma unroll
      for (int q = 0; q < PL; ++q) {
        const int r = lane + 32 * q;
        if (N % 32 == 0 || r < N) {
          const double kx = kof(g, r);
          double K2 = kx * kx + ky * ky;
          if (BGP_DIM(g) == 3) K2 = K2 + kz * kz;
          const double rden = 1.0 / (0.5 * K2 + sigma);
          b[swz(r)] = cscale(b[swz(r)], (Rt)rden);
        }
      }
      __syncwarp();
    }
    if (mode >= 1) warp_fft<N, true>(b, twt, lane);
  }
  BGP_D Pre fetch_out(int t, int r, int c) {
    OPP_ARGS
    Pre P{};
    if (mode == 3) {
      int i, j, k;
      P.a = cscale(ldp(psi, nline_elem(g, ax, t, r, c, i, j, k), sp), psc);
    }
    return P;
  }
  BGP_D void leave(const Pre& P, int t, int r, int c, double2 v) {
    OPP_ARGS
    int i, j, k;
    const int f = nline_elem(g, ax, t, r, c, i, j, k);
    if (mode < 3) { stp(A, f, v, sp); return; }
    const double2 z = cscale(v, inv_n);
    stp(Z, f, z, sp);
    const double2 pz = cconjmul(P.a, z);
    acc.s[0] += pz.x;
    acc.s[1] += pz.y;
  }
};

// -------------------------------------------------- zero-padded convolution
// Convolution scalars of an instance, copied into registers.
struct ConvGeo {
  int N, Mh, i0;
  double2* cb1;
  double2* cb2;
  const double2* twM;
};
BGP_D ConvGeo conv_geo(const Inst& I) { return ConvGeo{I.N, I.Mh, I.i0, I.cb1, I.cb2, I.twM}; }

// 2D, step a: rows i of the padded density, FFT along j, keep kj <= M/2.
// 3D, step a: lines (i,j), FFT along k, keep kk <= M/2 (same code: line = t*kLines+c).
template <int M>
#define OPCA_ARGS \
  [[maybe_unused]] const ConvGeo cg = conv_geo(I); \
  [[maybe_unused]] const RhoArgs R = rho_args(Q, Q.rmode);
struct OpCa {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = false;
  BGP_NO_OUT(4)
  const Inst& I;
  const PassArgs& Q;
  BGP_D Pre fetch(int t, int r, int c) {
    OPCA_ARGS
    Pre P;
    const int line = t * kLines + c, j = r - cg.i0;
    if (j >= 0 && j < cg.N) rho_fetch(R, line * cg.N + j, P);
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int r, int) {
    OPCA_ARGS
    const int j = r - cg.i0;
    if (j < 0 || j >= cg.N) return czero();
    return cmk(rho_of(R, P), 0.0);
  }
  BGP_D void line(double2* b, int lane, int, int) { warp_fft<M, false>(b, I.twM, lane); }
  BGP_D void leave(const Pre&, int t, int r, int c, double2 v) {
    OPCA_ARGS
    if (r < cg.Mh) st2(cg.cb1 + (size_t)(t * kLines + c) * cg.Mh + r, v);
  }
};

// 2D, step b: columns kj, FFT along i (padded), multiply by the kernel, inverse.
template <int M>
#define OPC2B_ARGS \
  [[maybe_unused]] const ConvGeo cg = conv_geo(I); \
  [[maybe_unused]] const double* Kq = Q.Kq;
struct OpC2b {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = false;
  BGP_NO_OUT(64)
  const Inst& I;
  const PassArgs& Q;
  BGP_D Pre fetch(int t, int r, int c) {
    OPC2B_ARGS
    Pre P;
    P.a = czero();
    const int kj = t * kLines + c, i = r - cg.i0;
    if (kj < cg.Mh && i >= 0 && i < cg.N) P.a = ld2(cg.cb1 + (size_t)i * cg.Mh + kj);
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int, int) { return P.a; }
  BGP_D void line(double2* b, int lane, int t, int w) {
    OPC2B_ARGS
    warp_fft<M, false>(b, cg.twM, lane);
    const int kj = t * kLines + w;
    if (kj < cg.Mh) {
      const size_t mh = (size_t)cg.Mh;
      line_times_kernel<M>(b, lane, Kq, [&](int r) {
        const int a = (r <= M / 2) ? r : M - r;
        return (size_t)a * mh + kj;
      });
    }
    __syncwarp();
    warp_fft<M, true>(b, cg.twM, lane);
  }
  BGP_D void leave(const Pre&, int t, int r, int c, double2 v) {
    OPC2B_ARGS
    const int kj = t * kLines + c, i = r - cg.i0;
    if (kj < cg.Mh && i >= 0 && i < cg.N) st2(cg.cb1 + (size_t)i * cg.Mh + kj, v);
  }
};

// Last step (2D rows / 3D k-lines): rebuild the Hermitian row spectrum, inverse
// FFT, keep the central N points: out = cscale * Re, and sum out * rho.
template <int M>
#define OPCINV_ARGS \
  [[maybe_unused]] const ConvGeo cg = conv_geo(I); \
  [[maybe_unused]] const RhoArgs R = rho_args(Q, Q.smode); \
  [[maybe_unused]] double* cout = Q.cout; \
  [[maybe_unused]] const double cscale_ = Q.cscale; \
  [[maybe_unused]] const int sum_on = Q.sum_on;
struct OpCinv {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = false;
  static constexpr int kChunk = 8;
  static constexpr int kChunkOut = 4;
  const Inst& I;
  const PassArgs& Q;
  Acc acc;
  BGP_D Pre fetch(int t, int r, int c) {
    OPCINV_ARGS
    const double2* row = cg.cb1 + (size_t)(t * kLines + c) * cg.Mh;
    Pre P;
    if (r < cg.Mh) {
      P.a = ld2(row + r);
    } else {
      const double2 v = ld2(row + (M - r));
      P.a = cmk(v.x, -v.y);
    }
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int, int) { return P.a; }
  BGP_D void line(double2* b, int lane, int, int) { warp_fft<M, true>(b, I.twM, lane); }
  BGP_D Pre fetch_out(int t, int r, int c) {
    OPCINV_ARGS
    Pre P{};
    const int j = r - cg.i0;
    if (sum_on && j >= 0 && j < cg.N) rho_fetch(R, (t * kLines + c) * cg.N + j, P);
    return P;
  }
  BGP_D void leave(const Pre& P, int t, int r, int c, double2 v) {
    OPCINV_ARGS
    const int j = r - cg.i0;
    if (j < 0 || j >= cg.N) return;
    const int f = (t * kLines + c) * cg.N + j;
    const double val = cscale_ * v.x;
    st1(cout + f, val);
    if (!sum_on) return;
    if (R.mode == 8) {
      // pair sums of the potential just formed with the density parts a, b, c,
      // and of the current potential with a
      double a, b, cc;
      rho_parts(R, P, a, b, cc);
      acc.s[0] += val * a;
      acc.s[1] += val * b;
      acc.s[2] += val * cc;
      acc.s[3] += P.r * a;
      return;
    }
    acc.s[S_G] += val * rho_of(R, P);
  }
};

// 3D step b (forward) / d (inverse): lines (i, kk) along j.
//   forward: cb1[i][j][kk] (j padded) -> FFT -> cb2[i][jj][kk]
//   inverse: cb2[i][jj][kk] -> IFFT -> central j -> cb1[i][j][kk]
template <int M>
#define OPC3B_ARGS \
  [[maybe_unused]] const ConvGeo cg = conv_geo(I); \
  [[maybe_unused]] const int inverse = Q.inverse;
struct OpC3b {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = false;
  BGP_NO_OUT(64)
  const Inst& I;
  const PassArgs& Q;
  BGP_D void decode(int t, int c, int& i, int& kk) const {
    OPC3B_ARGS
    const int tpl = (cg.Mh + kLines - 1) / kLines;
    i = t / tpl;
    kk = (t - i * tpl) * kLines + c;
  }
  BGP_D Pre fetch(int t, int r, int c) {
    OPC3B_ARGS
    int i, kk;
    decode(t, c, i, kk);
    Pre P;
    P.a = czero();
    if (kk >= cg.Mh) return P;
    if (inverse) { P.a = ld2(cg.cb2 + ((size_t)i * M + r) * cg.Mh + kk); return P; }
    const int j = r - cg.i0;
    if (j >= 0 && j < cg.N) P.a = ld2(cg.cb1 + ((size_t)i * cg.N + j) * cg.Mh + kk);
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int, int) { return P.a; }
  BGP_D void line(double2* b, int lane, int, int) {
    OPC3B_ARGS
    if (inverse) warp_fft<M, true>(b, cg.twM, lane);
    else warp_fft<M, false>(b, cg.twM, lane);
  }
  BGP_D void leave(const Pre&, int t, int r, int c, double2 v) {
    OPC3B_ARGS
    int i, kk;
    decode(t, c, i, kk);
    if (kk >= cg.Mh) return;
    if (!inverse) { st2(cg.cb2 + ((size_t)i * M + r) * cg.Mh + kk, v); return; }
    const int j = r - cg.i0;
    if (j >= 0 && j < cg.N) st2(cg.cb1 + ((size_t)i * cg.N + j) * cg.Mh + kk, v);
  }
};

// 3D step c: lines (jj, kk) along i: FFT (padded), kernel multiply, IFFT.
template <int M>
#define OPC3C_ARGS \
  [[maybe_unused]] const ConvGeo cg = conv_geo(I); \
  [[maybe_unused]] const double* Kq = Q.Kq;
struct OpC3c {
  static constexpr bool kStore = true;
  static constexpr bool kMixed = false;
  BGP_NO_OUT(64)
  const Inst& I;
  const PassArgs& Q;
  BGP_D void decode(int t, int c, int& jj, int& kk) const {
    OPC3C_ARGS
    const int tpl = (cg.Mh + kLines - 1) / kLines;
    jj = t / tpl;
    kk = (t - jj * tpl) * kLines + c;
  }
  BGP_D Pre fetch(int t, int r, int c) {
    OPC3C_ARGS
    int jj, kk;
    decode(t, c, jj, kk);
    Pre P;
    P.a = czero();
    const int i = r - cg.i0;
    if (kk < cg.Mh && i >= 0 && i < cg.N) P.a = ld2(cg.cb2 + ((size_t)i * M + jj) * cg.Mh + kk);
    return P;
  }
  BGP_D double2 enter(const Pre& P, int, int, int) { return P.a; }
  BGP_D void line(double2* b, int lane, int t, int w) {
    OPC3C_ARGS
    warp_fft<M, false>(b, cg.twM, lane);
    int jj, kk;
    decode(t, w, jj, kk);
    if (kk < cg.Mh) {
      const int bj = (jj <= M / 2) ? jj : M - jj;
      const size_t mh = (size_t)cg.Mh;
      line_times_kernel<M>(b, lane, Kq, [&](int r) {
        const int a = (r <= M / 2) ? r : M - r;
        return ((size_t)a * mh + bj) * mh + kk;
      });
    }
    __syncwarp();
    warp_fft<M, true>(b, cg.twM, lane);
  }
  BGP_D void leave(const Pre&, int t, int r, int c, double2 v) {
    OPC3C_ARGS
    int jj, kk;
    decode(t, c, jj, kk);
    const int i = r - cg.i0;
    if (kk < cg.Mh && i >= 0 && i < cg.N) st2(cg.cb2 + ((size_t)i * M + jj) * cg.Mh + kk, v);
  }
};

BGP_NS_END  // namespace bgp
