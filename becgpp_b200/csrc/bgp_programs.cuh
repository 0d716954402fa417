// Team programs: the device-resident PCG solver and the single-shot operators.
//
// Solver (one team per instance, all state on the device). Follows the
// Riemannian PCG of becgpp/solvers.py:48-235:
//   preconditioner   sigma = max(lower median of V + 2 b2 rho + 3 b3 rho^2 (+phi)
//                    over rho > 0.05 max rho, shift_min); z = P_T[(k^2/2+sigma)^-1 g]
//   beta             pr_precond <z, g-g_prev>/<z_prev, g_prev> | pr | none,
//                    restart every cg_restart iterations
//   direction        P_T(z + beta dir), falling back to z, then P_T(g) when not descent
//   step             alpha <- alpha/2 + clamp(<s,s>/<s,y>)/2, clamped
//   Armijo           psi_t = (psi - t dir)/||.||, E_t <= E - c1 t <g,dir>, halving
//   stops            residual < res_tol, windowed energy plateau, stalled line search
// The normalised trial state is kept lazily as (w, c = 1/||w||); energies of the
// normalised state follow from the sums of w scaled by powers of c.
#pragma once
#include "bgp_passes.cuh"

BGP_NS_BEGIN

struct Ctl {
  int f[F_NLOG];
  double sc[F_NLOG];
  int phi_cur;
  double phisc;
  int it, n_iter, n_fail, stop, converged, it_ref, ntrials, ntrace, z_proj, need_pz, accepted, naccept;
  int ok, done;
  double E, E_ref, alpha, trial, gd, beta, sigma, mu, resid_abs, resid_rel, best_resid, maxrho;
  double cz, cd, cg;
  double2 cpsi;
  int use_psi;
  double Et, ct;
  double tsum[kNRec];
  unsigned long long sel_r, sel_prefix, sel_key;
  int sel_level, sel_done, sel_bin;
  unsigned sel_cnt, sel_total;
  double med_prev, med_eps, below, wcnt;   // median window of the gradient pass: keys
                                           // under it and in it
  double nkeys;                      // keys written by the last gradient pass
  int med_valid, win_used, fast_hits, slow_runs;
  int yield, it_next;                 // segmented solve
  int fp32, cg_reset, fp64_from, do_switch;  // mixed form: FP32 on; restart CG; hand-over
  // line search of 3D instances with a kernel: pair sums G_xy = sum Phi_x y of the
  // trial density's parts a = |psi|^2, b = Re(conj(psi) dirc), c = |dirc|^2
  // (aa, ab, ac, bb, bc, cc)
  double qG[6];
};

struct Ctx {
  const Inst& I;
  Team T;
  double2* sm;
  double* sred;
  double* tot;
  PassArgs& Q;
  int slot;
  unsigned long long t_last;   // phase profiler: end of the previous phase (thread 0)
};

// Phase profiler (compiled in with -DBGP_PROF only): per phase kind, thread 0
// of team rank 0 accumulates {count, work, commit, barrier wait, gather} in ns
// into I.prof[5 * kind]; kind = the number of reduced slots, 16 = plain barrier.
#if defined(BGP_PROF)
#define BGP_PROF_T(v) const uint64_t v = gtimer_ns();
#define BGP_PROF_REC(C, kind, t0, t1, t2)                                               \
  if ((C).I.prof && (C).T.rank == 0 && threadIdx.x == 0) {                              \
    const uint64_t t3_ = gtimer_ns();                                                   \
    unsigned long long* p_ = (C).I.prof + 5 * (kind);                                   \
    p_[0] += 1; p_[1] += (t0) - (C).t_last; p_[2] += (t1) - (t0); p_[3] += (t2) - (t1); \
    p_[4] += t3_ - (t2);                                                                \
    (C).t_last = t3_;                                                                   \
  }
// time spent inside the tile loops (kind 18: count, ns)
#define BGP_PROF_ADD(C, kind, dt)                                                       \
  if ((C).I.prof && (C).T.rank == 0 && threadIdx.x == 0) {                              \
    unsigned long long* p_ = (C).I.prof + 5 * (kind);                                   \
    p_[0] += 1; p_[1] += (dt);                                                          \
  }
#else
#define BGP_PROF_T(v)
#define BGP_PROF_REC(C, kind, t0, t1, t2)
#define BGP_PROF_ADD(C, kind, dt)
#endif

// phase boundary with a reduction of the first NV slots (and the max slot)
template <int NV>
__device__ __noinline__ bool phase_end(Ctx& C, Acc a) {
  BGP_PROF_T(t0)
  acc_commit<NV>(C.I, C.T, a, C.slot, C.sred);
  BGP_PROF_T(t1)
  const bool ok = team_sync(C.T);
  BGP_PROF_T(t2)
  if (ok) acc_gather<NV>(C.I, C.slot, C.tot);
  BGP_PROF_REC(C, NV, t0, t1, t2)
  C.slot ^= 1;
  return ok;
}
// slots used by each kind of phase
constexpr int kRedH = 1, kRedG = 5, kRedZ = 2, kRedT = 13, kRedD = 15;

// phase boundary without a reduction record: only the team barrier
static __device__ __noinline__ bool phase_sync(Ctx& C) {
  BGP_PROF_T(t0)
  const bool ok = team_sync(C.T);
  BGP_PROF_T(t2)
  BGP_PROF_REC(C, 16, t0, t0, t2)
  return ok;
}

BGP_D bool phase_end0(Ctx& C) { return phase_sync(C); }

template <int L1, bool C1, class Op1>
BGP_D void run_one(Ctx& C, Op1& a, int n1) {
  BGP_PROF_T(ta)
  const int fp32 = C.Q.fp32;
  for (int u = C.T.rank; u < n1; u += C.T.size) tile_run<L1, C1>(a, C.sm, u, fp32);
  BGP_PROF_T(tb)
  BGP_PROF_ADD(C, 18, tb - ta)
}

template <int L1, bool C1, class Op1, int L2, bool C2, class Op2>
BGP_D void run_two(Ctx& C, Op1& a, int n1, Op2& b, int n2) {
  BGP_PROF_T(ta)
  const int fp32 = C.Q.fp32;
  for (int u = C.T.rank; u < n1 + n2; u += C.T.size) {
    if (u < n1) tile_run<L1, C1>(a, C.sm, u, fp32);
    else tile_run<L2, C2>(b, C.sm, u - n1, fp32);
  }
  BGP_PROF_T(tb)
  BGP_PROF_ADD(C, 18, tb - ta)
}

BGP_D double2* pool_buf(const Inst& I, int b) { return I.pool + (size_t)b * I.n; }
BGP_D double* phi_buf(const Inst& I, int b) { return I.phi2 + (size_t)b * I.n; }

// first free pool buffer (not referenced by any logical field)
BGP_D int pool_alloc(const Ctl& S) {
  unsigned used = 0u;
#pragma unroll
  for (int q = 0; q < F_NLOG; ++q) {
    const int b = S.f[q];
    if (b >= 0) used |= 1u << b;
  }
  const unsigned avail = ~used & ((1u << kNB) - 1u);
  return avail ? __ffs(avail) - 1 : -1;
}

// ---------------------------------------------------------------- energy assembly
// comp: E, Ekin, Etrap, Econtact, Ethree, Erot, Egrav, Lz from the sums of w and
// c2 = c^2 (the normalised state is c w).
BGP_HD void energy_assemble(const Inst& I, const double* s, double c2, double* comp) {
  const double dv = I.dv, inv = 1.0 / (double)I.N;
  const double c4 = c2 * c2;
  const double Ekin = 0.5 * (s[S_KX] + s[S_KY] + s[S_KZ]) * inv * dv * c2;
  const double Etrap = s[S_V] * dv * c2;
  const double Econ = 0.5 * I.beta2 * s[S_2] * dv * c4;
  const double Ethr = (I.beta3 / 3.0) * s[S_3] * dv * (c4 * c2);
  const double Lz = (s[S_LY] - s[S_LX]) * inv * dv * c2;
  const double Erot = -I.Omega * Lz;
  const double Egr = (I.kind != kNone) ? 0.5 * s[S_G] * dv * c4 : 0.0;
  comp[0] = Ekin + Etrap + Econ + Ethr + Erot + Egr;
  comp[1] = Ekin; comp[2] = Etrap; comp[3] = Econ; comp[4] = Ethr; comp[5] = Erot;
  comp[6] = Egr; comp[7] = Lz;
}

BGP_D void tsum_add(Ctl& S, const double* tot) {
  if (threadIdx.x == 0) {
    for (int q = 0; q < kNSum; ++q) S.tsum[q] += tot[q];
    S.tsum[kNSum] = fmax(S.tsum[kNSum], tot[kNSum]);
  }
  __syncthreads();
}

// --------------------------------------------------------------- energy phases
// mode: 0 trial (w = psi - t dirc; Q.psi, Q.t and the direction terms set by the
//         caller), 1 initial state (w = Q.cin, copied to Q.W),
//       2 API energy (w = Q.cin, nothing written).
// Sums of w over every axis and, with a kernel, the convolution of |w|^2 (to
// phi_out, unscaled by c) with its sum  sum phi_w |w|^2. Totals in S.tsum.
template <int N, int M>
__device__ __noinline__ bool energy_phases(Ctx& C, Ctl& S, int mode, int write_dirc, double2* W, double2* DIRC,
                         double* phi_out, bool conv = true) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  if (threadIdx.x == 0) {
    for (int q = 0; q < kNRec; ++q) S.tsum[q] = 0.0;
    Q.W = W; Q.DIRC = DIRC;
    Q.src = (mode == 2) ? Q.cin : W;
    Q.init = (mode != 0); Q.write_w = (mode != 2); Q.write_dirc = write_dirc;
    Q.rmode = (mode == 0) ? (write_dirc ? 1 : 5) : 3;
    Q.smode = (mode == 2) ? 3 : 4;
    Q.Kq = I.Kq; Q.cscale = I.conv_scale; Q.cout = phi_out; Q.sum_on = 1;
  }
  __syncthreads();
  const bool kern = conv && (I.kind != kNone) && M > 0;
  const int nt = ntiles_axis(I);
  const int last = BGP_DIM(I) - 1;
  {
    OpT<N> tf{I, Q, last};
    bool did = false;
    if constexpr (M > 0) {
      if (kern) {
        did = true;
        OpCa<M> cv{I, Q};
        run_two<N, true, OpT<N>, M, true, OpCa<M>>(C, tf, nt, cv, nt);
      }
    }
    if (!did) run_one<N, true>(C, tf, nt);
    if (!phase_end<kRedT>(C, tf.acc)) return false;
    tsum_add(S, C.tot);
  }
  const int tpl = (I.Mh + kLines - 1) / kLines;
  for (int ax = last - 1; ax >= 0; --ax) {
    if (threadIdx.x == 0) Q.inverse = 0;
    __syncthreads();
    OpT<N> to{I, Q, ax};
    bool did = false;
    if constexpr (M > 0) {
      if (kern) {
        did = true;
        if (BGP_DIM(I) == 2) {
          OpC2b<M> cv{I, Q};
          run_two<N, false, OpT<N>, M, false, OpC2b<M>>(C, to, nt, cv, tpl);
        } else if (ax == 1) {
          OpC3b<M> cv{I, Q};
          run_two<N, false, OpT<N>, M, false, OpC3b<M>>(C, to, nt, cv, I.N * tpl);
        } else {
          OpC3c<M> cv{I, Q};
          run_two<N, false, OpT<N>, M, false, OpC3c<M>>(C, to, nt, cv, M * tpl);
        }
      }
    }
    if (!did) run_one<N, false>(C, to, nt);
    if (!phase_end<kRedT>(C, to.acc)) return false;
    tsum_add(S, C.tot);
  }
  if constexpr (M > 0) {
    if (kern) {
      if (BGP_DIM(I) == 3) {
        if (threadIdx.x == 0) Q.inverse = 1;
        __syncthreads();
        OpC3b<M> cv{I, Q};
        run_one<M, false>(C, cv, I.N * tpl);
        if (!phase_end0(C)) return false;
      }
      OpCinv<M> ci{I, Q};
      run_one<M, true>(C, ci, nt);
      if (!phase_end<kRedT>(C, ci.acc)) return false;
      tsum_add(S, C.tot);
    }
  }
  return true;
}

// Convolution only: Q.cout = Q.cscale * (Q.Kq * rho), rho from Q.rmode; with
// sum_on the last phase also sums out * rho (density from Q.smode) into tot[S_G].
template <int N, int M>
__device__ __noinline__ bool conv_phases(Ctx& C, int sum_on = 0) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  if constexpr (M > 0) {
    const int nt = ntiles_axis(I);
    const int tpl = (I.Mh + kLines - 1) / kLines;
    if (threadIdx.x == 0) { Q.sum_on = sum_on; Q.inverse = 0; }
    __syncthreads();
    { OpCa<M> s1{I, Q}; run_one<M, true>(C, s1, nt); }
    if (!phase_end0(C)) return false;
    if (BGP_DIM(I) == 2) {
      OpC2b<M> s2{I, Q};
      run_one<M, false>(C, s2, tpl);
      if (!phase_end0(C)) return false;
    } else {
      { OpC3b<M> s2{I, Q}; run_one<M, false>(C, s2, I.N * tpl); }
      if (!phase_end0(C)) return false;
      { OpC3c<M> s3{I, Q}; run_one<M, false>(C, s3, M * tpl); }
      if (!phase_end0(C)) return false;
      if (threadIdx.x == 0) Q.inverse = 1;
      __syncthreads();
      { OpC3b<M> s4{I, Q}; run_one<M, false>(C, s4, I.N * tpl); }
      if (!phase_end0(C)) return false;
    }
    OpCinv<M> ci{I, Q};
    run_one<M, true>(C, ci, nt);
    if (!phase_end<kRedT>(C, ci.acc)) return false;
  }
  return true;
}

// H psi phases (Q.psi/psc, Q.A, Q.H, Q.phi/phisc set by the caller): writes H,
// leaves mu-sum in tot[0] and max rho in tot[max]. The first phase also clears
// the median histograms (rank 0).
template <int N>
__device__ __noinline__ bool hpsi_phases(Ctx& C) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  const int nt = ntiles_axis(I);
  for (int st = 0; st < BGP_DIM(I); ++st) {
    const int ax = BGP_DIM(I) - 1 - st;
    if (threadIdx.x == 0) { Q.ax = ax; Q.stage = (st == 0) ? 0 : (ax == 0 ? 2 : 1); }
    if (st == 0 && C.T.rank == 0) {
      for (int q = threadIdx.x; q < 8 * 256 + 2; q += kThreads) I.hist[q] = 0u;
    }
    __syncthreads();
    OpH<N> op{I, Q};
    if (ax == BGP_DIM(I) - 1) run_one<N, true>(C, op, nt);
    else run_one<N, false>(C, op, nt);
    if (ax != 0) { if (!phase_sync(C)) return false; }
    else if (!phase_end<kRedH>(C, op.acc)) return false;
  }
  return true;
}

// Gradient pass (Q.psi, Q.H or Q.gin, Q.mu, Q.Gout, Q.A, Q.phi, Q.thr, Q.keys_on
// set by the caller); the level-0 median histogram is merged into I.hist.
template <int N>
__device__ __noinline__ bool grad_phase(Ctx& C, double vote) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  unsigned* shist = reinterpret_cast<unsigned*>(C.sred + (kNSum + 1) * kWarps);
  for (int q = threadIdx.x; q < 256; q += kThreads) shist[q] = 0u;
  if (threadIdx.x == 0) Q.shist = shist;
  __syncthreads();
  OpG<N> g{I, Q};
  run_one<N, true>(C, g, ntiles_axis(I));
  if (C.T.rank == 0 && threadIdx.x == 0) g.acc.s[2] += vote;
  if (Q.keys_on)
    for (int q = threadIdx.x; q < 256; q += kThreads) if (shist[q]) atomicAdd(&I.hist[q], shist[q]);
  return phase_end<kRedG>(C, g.acc);
}

// --------------------------------------------------------------------- median
// Lower median (rank (m-1)/2) of the keys written by OpG, by radix selection on
// bytes from the top; the level-0 histogram is already filled. When the bucket
// holding the rank has at most kSelCap keys they are gathered and ranked in
// shared memory. Returns the selected value, or `floor` if no key was written.
BGP_D void hist_scan(const unsigned* h, Ctl& S) {
  // warp 0: find the bin containing rank S.sel_r
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    unsigned c[8];
    unsigned long long tot = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) { c[q] = __ldcg(h + lane * 8 + q); tot += c[q]; }
    unsigned long long inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    const unsigned long long excl = inc - tot;
    const unsigned long long all = __shfl_sync(0xffffffffu, inc, 31);
    if (lane == 0) S.sel_total = (unsigned)all;
    const unsigned long long r = S.sel_r;
    if (r >= excl && r < inc) {
      unsigned long long run = excl;
      int found = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        if (!found && r < run + c[q]) {
          S.sel_bin = lane * 8 + q;
          S.sel_cnt = c[q];
          S.sel_r = r - run;
          found = 1;
        }
        run += c[q];
      }
    }
  }
  __syncthreads();
}

// r-th smallest of cnt (<= kSelCap) keys, ranked in shared memory by counting
BGP_D unsigned long long rank_select(Ctx& C, Ctl& S, const unsigned long long* src, int cnt,
                                     unsigned long long r) {
  unsigned long long* sk = reinterpret_cast<unsigned long long*>(C.sm);
  for (int q = threadIdx.x; q < cnt; q += kThreads) sk[q] = __ldcg(src + q);
  __syncthreads();
  // T consecutive threads per key (4 or 2 when the keys are few), each counting
  // over every T-th key; their counts meet by shuffles
  const int T = (cnt * 4 <= kThreads) ? 4 : ((cnt * 2 <= kThreads) ? 2 : 1);
  for (int base = 0; base < cnt * T; base += kThreads) {
    const int idx = base + threadIdx.x, q = idx / T, part = idx % T;
    unsigned long long x = 0, lt = 0, le = 0;
    if (q < cnt) {
      x = sk[q];
      for (int p = part; p < cnt; p += T) { lt += (sk[p] < x); le += (sk[p] <= x); }
    }
    for (int o = 1; o < T; o <<= 1) {
      lt += __shfl_xor_sync(0xffffffffu, lt, o);
      le += __shfl_xor_sync(0xffffffffu, le, o);
    }
    if (q < cnt && part == 0 && lt <= r && r < le) S.sel_key = x;
  }
  __syncthreads();
  const unsigned long long key = S.sel_key;
  __syncthreads();
  return key;
}

// S.below and S.wcnt (keys under and in the window, from the gradient pass) must
// be set by the caller when S.win_used. Returns the lower median, or `floor` with no keys.
static __device__ __noinline__ bool median_select(Ctx& C, Ctl& S, double floor_v, double& out);

// Median selection, timed as its own kind (17) by the phase profiler.
static __device__ __noinline__ bool median_phases(Ctx& C, Ctl& S, double floor_v, double& out) {
  const bool ok = median_select(C, S, floor_v, out);
  BGP_PROF_T(t0)
  BGP_PROF_REC(C, 17, t0, t0, t0)
  return ok;
}

static __device__ __noinline__ bool median_select(Ctx& C, Ctl& S, double floor_v, double& out) {
  const Inst& I = C.I;
  __shared__ unsigned sh[256];
  if (threadIdx.x == 0) { S.sel_r = ~0ull; }
  __syncthreads();
  // the number of keys is the gradient pass's count (S.nkeys)
  const unsigned m = (unsigned)S.nkeys;
  if (m == 0) { out = floor_v; return true; }
  if (threadIdx.x == 0) { S.sel_r = (unsigned long long)((m - 1u) / 2u); S.sel_prefix = 0ull; }
  __syncthreads();
  // window path: the rank lies among the gathered keys around the last median
  if (S.win_used) {
    const unsigned wc = (unsigned)S.wcnt;   // the gradient pass's count of window keys
    const unsigned long long r = S.sel_r, below = (unsigned long long)S.below;
    if (wc <= (unsigned)kSelCap && r >= below && r < below + wc) {
      out = dkey_inv(rank_select(C, S, I.wcand, (int)wc, r - below));
      if (threadIdx.x == 0) {
        S.fast_hits++;
        // keep the window near kWinTarget keys: the ranking costs O(keys) a thread
        if (wc > (unsigned)kWinTarget) S.med_eps = fmax(S.med_eps * 0.7, 1e-12);
      }
      __syncthreads();
      return true;
    }
    if (threadIdx.x == 0) {
      // widen the window when the median moved out of it, narrow it when it overflowed
      S.med_eps = (wc > (unsigned)kSelCap) ? fmax(S.med_eps * 0.25, 1e-9) : fmin(S.med_eps * 4.0, 0.25);
    }
  }
  if (threadIdx.x == 0) S.slow_runs++;
  __syncthreads();
  const long long n = I.n;
  const long long lo = n * C.T.rank / C.T.size, hi = n * (C.T.rank + 1) / C.T.size;
  for (int level = 0; level < 8; ++level) {
    hist_scan(I.hist + level * 256, S);
    const int shift = 56 - 8 * level;
    if (threadIdx.x == 0) S.sel_prefix |= ((unsigned long long)S.sel_bin) << shift;
    __syncthreads();
    const unsigned long long prefix = S.sel_prefix;
    if (level == 7) { out = dkey_inv(prefix); break; }
    if (S.sel_cnt <= (unsigned)kSelCap) {
      // gather the bucket, rank it in shared memory
      for (long long f = lo + threadIdx.x; f < hi; f += kThreads) {
        const unsigned long long key = __ldcg(I.keys + f);
        if (key != 0ull && (key >> shift) == (prefix >> shift)) {
          const unsigned idx = atomicAdd(&I.hist[8 * 256], 1u);
          if (idx < (unsigned)kSelCap) I.cand[idx] = key;
        }
      }
      if (!team_sync(C.T)) return false;
      out = dkey_inv(rank_select(C, S, I.cand, (int)S.sel_cnt, S.sel_r));
      break;
    }
    // next byte histogram over the keys of this bucket
    for (int q = threadIdx.x; q < 256; q += kThreads) sh[q] = 0u;
    __syncthreads();
    const int nshift = shift - 8;
    for (long long f = lo + threadIdx.x; f < hi; f += kThreads) {
      const unsigned long long key = __ldcg(I.keys + f);
      if (key != 0ull && (key >> shift) == (prefix >> shift))
        atomicAdd(&sh[(key >> nshift) & 255ull], 1u);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 256; q += kThreads)
      if (sh[q]) atomicAdd(&I.hist[(level + 1) * 256 + q], sh[q]);
    if (!team_sync(C.T)) return false;
  }
  return true;
}

// preconditioner transforms after OpG (Q.A holds g transformed along the last
// axis); Q.sigma, Q.Z, Q.psi set by the caller. Leaves sum conj(psi) z_raw in tot[0,1].
template <int N>
__device__ __noinline__ bool precond_phases(Ctx& C) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  const int nt = ntiles_axis(I);
  const int seq2[1][2] = {{0, 1}};
  const int seq3[3][2] = {{1, 0}, {0, 1}, {1, 2}};
  const int nsteps = (BGP_DIM(I) == 2) ? 1 : 3;
  for (int s = 0; s < nsteps; ++s) {
    if (threadIdx.x == 0) {
      Q.ax = (BGP_DIM(I) == 2) ? seq2[0][0] : seq3[s][0];
      Q.mode = (BGP_DIM(I) == 2) ? seq2[0][1] : seq3[s][1];
    }
    __syncthreads();
    OpP<N> op{I, Q};
    run_one<N, false>(C, op, nt);
    if (!phase_sync(C)) return false;
  }
  if (threadIdx.x == 0) { Q.ax = BGP_DIM(I) - 1; Q.mode = 3; }
  __syncthreads();
  OpP<N> pz{I, Q};
  run_one<N, true>(C, pz, nt);
  return phase_end<kRedZ>(C, pz.acc);
}

// residual of the current state: H psi, mu, then g = H - mu psi with |g|^2 and
// the median keys. Uses S.f[F_PSI], S.phi_cur; allocates F_H and F_G.
template <int N, int M>
__device__ __noinline__ bool residual_phases(Ctx& C, Ctl& S) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  const bool kern = (I.kind != kNone) && (M > 0);
  if (threadIdx.x == 0) {
    S.f[F_H] = pool_alloc(S);
    S.ok = S.f[F_H] >= 0;
    if (!S.ok) S.f[F_H] = 0;
    Q.psi = pool_buf(I, S.f[F_PSI]); Q.psc = S.sc[F_PSI];
    Q.A = pool_buf(I, S.f[F_A]); Q.H = pool_buf(I, S.f[F_H]);
    Q.phi = kern ? phi_buf(I, S.phi_cur) : nullptr; Q.phisc = S.phisc;
  }
  __syncthreads();
  if (!S.ok) return false;
  if (!hpsi_phases<N>(C)) return false;
  if (threadIdx.x == 0) {
    S.mu = C.tot[0] * I.dv; S.maxrho = C.tot[kNSum];
    S.f[F_G] = pool_alloc(S);
    S.ok = S.f[F_G] >= 0;
    if (!S.ok) S.f[F_G] = 0;
    Q.mu = S.mu; Q.gin = nullptr; Q.Gout = pool_buf(I, S.f[F_G]);
    Q.thr = 0.05 * S.maxrho; Q.keys_on = 1;
    S.win_used = S.med_valid;
    Q.win_on = S.med_valid;
    if (S.med_valid) {
      const double w = fabs(S.med_prev) * S.med_eps + 1e-300;
      Q.win_lo = dkey(S.med_prev - w);
      Q.win_hi = dkey(S.med_prev + w);
    }
  }
  __syncthreads();
  if (!S.ok) return false;
  // yield vote: rank 0 reads how many instances of this launch have finished;
  // the reduction makes the decision the same in every CTA of the team
  double vote = 0.0;
  if (C.T.rank == 0 && threadIdx.x == 0 && I.finished)
    vote = (*((volatile int*)I.finished) >= I.yield_at) ? 1.0 : 0.0;
  if (!grad_phase<N>(C, vote)) return false;
  if (threadIdx.x == 0) {
    S.yield = C.tot[2] > 0.5;
    S.below = C.tot[1];
    S.nkeys = C.tot[3];
    S.wcnt = C.tot[4];
    S.f[F_H] = -1;
    S.resid_abs = sqrt(C.tot[0] * I.dv);
    S.resid_rel = S.resid_abs / fmax(1.0, fabs(S.mu));
  }
  __syncthreads();
  return true;
}

// Mixed form: consecutive failed line searches in FP32 after which the FP64
// iterations take over.
constexpr int kMixedFailSwitch = 3;

// Mixed form: hand over from FP32 to FP64 transforms. The energy, potential,
// residual and median keys of the current state are evaluated again in FP64,
// the CG recurrence restarts (beta = 0, no Barzilai-Borwein update) and the
// energy window and the lowest-residual iterate start afresh.
template <int N, int M>
__device__ __noinline__ bool switch_to_fp64(Ctx& C, Ctl& S, int it) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  // every thread has read the control state that led here (S.fp32 among it)
  // before thread 0 changes it
  __syncthreads();
  // the FP32 phase stored the pool fields as complex64: widen the state into a
  // free pool field (complex128), unscaled; the fields of the earlier iterates are
  // not read again (the recurrence restarts from the new gradient and z)
  if (threadIdx.x == 0) {
    S.f[F_G] = -1; S.f[F_Z] = -1; S.f[F_W] = -1; S.f[F_DIRC] = -1;
    S.f[F_PSIP] = -1; S.f[F_GP] = -1; S.f[F_ZP] = -1; S.f[F_DIR] = -1; S.f[F_BEST] = -1;
    S.f[F_H] = pool_alloc(S);
    S.ok = S.f[F_H] >= 0;
  }
  __syncthreads();
  if (!S.ok) return false;
  {
    const double2* src = pool_buf(I, S.f[F_PSI]);
    double2* dst = pool_buf(I, S.f[F_H]);
    for (int f = C.T.rank * kThreads + threadIdx.x; f < I.n; f += C.T.size * kThreads)
      st2(dst + f, ldp(src, f, 1));
  }
  if (!phase_end0(C)) return false;
  if (threadIdx.x == 0) {
    S.f[F_PSI] = S.f[F_H]; S.f[F_H] = -1;
    S.f[F_PSIP] = S.f[F_PSI]; S.sc[F_PSIP] = S.sc[F_PSI];
    S.fp32 = 0; Q.fp32 = 0; S.fp64_from = it;
    Q.cin = pool_buf(I, S.f[F_PSI]);
  }
  __syncthreads();
  if (!energy_phases<N, M>(C, S, 2, 0, nullptr, nullptr, phi_buf(I, S.phi_cur))) return false;
  if (threadIdx.x == 0) {
    // the complex64 state's norm differs from 1 by its rounding: normalize it again
    const double c = 1.0 / sqrt(S.tsum[S_N0] * I.dv);
    S.sc[F_PSI] = c; S.sc[F_PSIP] = c;
    double comp[8];
    energy_assemble(I, S.tsum, c * c, comp);
    S.E = comp[0];
    S.phisc = c * c;
  }
  __syncthreads();
  if (!residual_phases<N, M>(C, S)) return false;
  if (threadIdx.x == 0) {
    S.f[F_GP] = S.f[F_G];
    S.need_pz = 1; S.cg_reset = 1; S.n_fail = 0;
    S.best_resid = S.resid_rel; S.f[F_BEST] = S.f[F_PSI]; S.sc[F_BEST] = S.sc[F_PSI];
    S.E_ref = S.E; S.it_ref = it;
  }
  __syncthreads();
  return true;
}

// ------------------------------------------------------------------ the solver
template <int N, int M>
BGP_D void prog_solve(Ctx& C, Ctl& S) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  const SolverParams& P = I.sp;
  const int tid = threadIdx.x;
  const double dv = I.dv;
  const bool kern = (I.kind != kNone) && (M > 0);
  const bool poly = kern && BGP_DIM(I) == 3;   // the line search's quartic (above)
  int it0 = 0;
  if (I.resume) {
    // continue a yielded solve: restore the control state saved by the last launch
    if (tid == 0) { S = *reinterpret_cast<const Ctl*>(I.save); Q.fp32 = S.fp32; }
    __syncthreads();
    it0 = S.it_next;
    goto iterate;
  }
  if (tid == 0) {
    for (int q = 0; q < F_NLOG; ++q) { S.f[q] = -1; S.sc[q] = 1.0; }
    S.f[F_A] = 0;
    S.f[F_W] = 1;
    S.phi_cur = 0; S.phisc = 1.0;
    S.it = 0; S.n_iter = 0; S.n_fail = 0; S.stop = kStopMaxit; S.converged = 0; S.it_ref = 0;
    S.ntrials = 0; S.ntrace = 0; S.z_proj = 0; S.need_pz = 1; S.accepted = 0; S.ok = 1; S.naccept = 0;
    S.med_valid = 0; S.med_eps = 1e-3; S.win_used = 0; S.fast_hits = 0; S.slow_runs = 0; S.med_prev = 0.0;
    S.alpha = P.alpha0; S.sigma = P.shift_min; S.beta = 0.0; S.done = 0;
    S.fp32 = BGP_MIXED ? P.mixed : 0; S.cg_reset = 0; S.fp64_from = S.fp32 ? -1 : 0;
    Q.cin = I.in_psi; Q.fp32 = S.fp32;
  }
  __syncthreads();
  // ---- initial state: psi = psi0 / ||psi0||, its energy and potential
  if (!energy_phases<N, M>(C, S, 1, 0, pool_buf(I, 1), nullptr, phi_buf(I, 1))) goto fail;
  if (tid == 0) {
    const double c = 1.0 / sqrt(S.tsum[S_N0] * dv);
    double comp[8];
    energy_assemble(I, S.tsum, c * c, comp);
    S.E = comp[0];
    S.f[F_PSI] = S.f[F_W]; S.sc[F_PSI] = c; S.f[F_W] = -1;
    S.phi_cur = 1; S.phisc = c * c;
    S.f[F_PSIP] = S.f[F_PSI]; S.sc[F_PSIP] = c;
  }
  __syncthreads();
  if (!residual_phases<N, M>(C, S)) goto fail;
  if (tid == 0) {
    S.f[F_GP] = S.f[F_G];
    S.f[F_BEST] = S.f[F_PSI]; S.sc[F_BEST] = S.sc[F_PSI];
    S.best_resid = S.resid_rel;
    S.E_ref = S.E; S.it_ref = 0;
    if (P.record_trace && S.ntrace < P.trace_cap) {
      I.trace[0] = 0.0; I.trace[1] = S.E; I.trace[2] = NAN; S.ntrace = 1;
    }
  }
  __syncthreads();
  // ---- iterations
iterate:
  for (int it = it0; it < P.maxit; ++it) {
    if (tid == 0) { S.it = it; S.n_iter = it + 1; }
    __syncthreads();
    if (S.need_pz) {
      double sig;
      if (!median_phases(C, S, P.shift_min, sig)) goto fail;
      if (tid == 0) {
        if (S.nkeys > 0.5) { S.med_prev = sig; S.med_valid = 1; }
        S.sigma = fmax(sig, P.shift_min);
        S.f[F_Z] = pool_alloc(S);
        S.ok = S.f[F_Z] >= 0;
        if (!S.ok) S.f[F_Z] = 0;
        Q.sigma = S.sigma; Q.Z = pool_buf(I, S.f[F_Z]); Q.A = pool_buf(I, S.f[F_A]);
        Q.psi = pool_buf(I, S.f[F_PSI]); Q.psc = S.sc[F_PSI];
      }
      __syncthreads();
      if (!S.ok) goto fail;
      if (!precond_phases<N>(C)) goto fail;
      if (tid == 0) {
        S.cpsi = cmk(C.tot[0] * dv, C.tot[1] * dv);   // <psi, z_raw> dV
        S.z_proj = 0;
        // first iteration, and the first after the hand-over to FP64 (whose earlier
        // z and direction are FP32 fields): start the recurrence from z
        if (it == 0 || S.cg_reset) { S.f[F_ZP] = S.f[F_Z]; S.f[F_DIR] = S.f[F_Z]; }
      }
      __syncthreads();
    }
    // ---- direction reductions (elementwise)
    {
      Acc a; a.zero();
      const double2* ps = pool_buf(I, S.f[F_PSI]);
      const double psc = S.sc[F_PSI];
      const double2* pp = pool_buf(I, S.f[F_PSIP]);
      const double ppc = S.sc[F_PSIP];
      double2* Z = pool_buf(I, S.f[F_Z]);
      const double2* G = pool_buf(I, S.f[F_G]);
      const double2* GP = pool_buf(I, S.f[F_GP]);
      const double2* ZP = pool_buf(I, S.f[F_ZP]);
      const double2* D = pool_buf(I, S.f[F_DIR]);
      const bool zp_alias = S.f[F_ZP] == S.f[F_Z], d_alias = S.f[F_DIR] == S.f[F_Z];
      const bool proj = !S.z_proj;
      const double2 aproj = S.cpsi;
      const int n = I.n;
      const int sp = S.fp32;     // pool fields in FP32 while the mixed form runs in FP32
      for (int f = C.T.rank * kThreads + tid; f < n; f += C.T.size * kThreads) {
        const double2 p = cscale(ldp(ps, f, sp), psc);
        double2 z = ldp(Z, f, sp);
        if (proj) { z = csub(z, cmul(aproj, p)); stp(Z, f, z, sp); }
        const double2 g = ldp(G, f, sp), gp = ldp(GP, f, sp);
        const double2 zp = zp_alias ? z : ldp(ZP, f, sp);
        const double2 d = d_alias ? z : ldp(D, f, sp);
        const double2 q = cscale(ldp(pp, f, sp), ppc);
        const double2 y = csub(g, gp), s = csub(p, q);
        a.s[0] += z.x * y.x + z.y * y.y;
        a.s[1] += zp.x * gp.x + zp.y * gp.y;
        a.s[2] += g.x * y.x + g.y * y.y;
        a.s[3] += cabs2(gp);
        const double2 pz = cconjmul(p, z), pd = cconjmul(p, d), gpsi = cconjmul(g, p);
        a.s[4] += pz.x; a.s[5] += pz.y;
        a.s[6] += pd.x; a.s[7] += pd.y;
        a.s[8] += g.x * z.x + g.y * z.y;
        a.s[9] += g.x * d.x + g.y * d.y;
        a.s[10] += gpsi.x; a.s[11] += gpsi.y;
        a.s[12] += s.x * y.x + s.y * y.y;
        a.s[13] += cabs2(s);
        a.s[14] += cabs2(g);
      }
      if (!phase_end<kRedD>(C, a)) goto fail;
      if (tid == 0) {
        S.z_proj = 1;
        const double* r = C.tot;
        double beta = 0.0;
        if (!(it == 0 || S.cg_reset || P.cg_beta == 2 || (P.restart > 0 && it % P.restart == 0))) {
          if (P.cg_beta == 0) {
            const double den = fmax(r[1] * dv, 1e-300);
            beta = fmax(0.0, (r[0] * dv) / den);
          } else {
            const double den = fmax(r[3] * dv, 1e-300);
            beta = fmax(0.0, (r[2] * dv) / den);
          }
          if (!isfinite(beta)) beta = 0.0;
        }
        S.beta = beta;
        // dirc = z + beta dir - b psi,  b = <psi, z + beta dir> dV
        const double2 b = cmk((r[4] + beta * r[6]) * dv, (r[5] + beta * r[7]) * dv);
        const double2 gpsi = cmk(r[10], r[11]);
        S.cz = 1.0; S.cd = beta; S.cg = 0.0;
        S.cpsi = cmk(-b.x, -b.y); S.use_psi = 1;
        double gd = (r[8] + beta * r[9] - (b.x * gpsi.x - b.y * gpsi.y)) * dv;
        if (gd <= 0.0) {
          S.cd = 0.0; S.use_psi = 0; S.cpsi = cmk(0.0, 0.0);
          gd = r[8] * dv;
        }
        if (gd <= 0.0) {
          // P_T(g) = g - psi <psi, g> dV,  <psi, g> = conj(sum conj(g) psi)
          const double2 pg = cmk(gpsi.x * dv, -gpsi.y * dv);
          S.cz = 0.0; S.cd = 0.0; S.cg = 1.0; S.use_psi = 1; S.cpsi = cmk(-pg.x, -pg.y);
          gd = (r[14] - (pg.x * gpsi.x - pg.y * gpsi.y)) * dv;
        }
        S.gd = gd;
        if (it > 0 && !S.cg_reset) {
          const double sy = r[12] * dv;
          if (sy > 1e-30 && isfinite(sy)) {
            double bb = (r[13] * dv) / sy;
            if (isfinite(bb)) {
              bb = fmin(fmax(bb, P.bb_min), P.bb_max);
              S.alpha = (1.0 - P.bb_mix) * S.alpha + P.bb_mix * bb;
            }
          }
        }
        S.alpha = fmin(fmax(S.alpha, P.alpha_min), P.alpha_max);
        S.cg_reset = 0;
        S.trial = S.alpha;
        S.accepted = 0;
        S.f[F_DIRC] = pool_alloc(S);
        S.f[F_W] = pool_alloc(S);
        S.ok = (S.f[F_DIRC] >= 0 && S.f[F_W] >= 0 && S.f[F_DIRC] != S.f[F_W]);
        // operands of the trial passes
        Q.psi = pool_buf(I, S.f[F_PSI]); Q.psc = S.sc[F_PSI];
        Q.dz = pool_buf(I, S.f[F_Z]); Q.dd = pool_buf(I, S.f[F_DIR]); Q.dg = pool_buf(I, S.f[F_G]);
        Q.cz = S.cz; Q.cd = S.cd; Q.cg = S.cg; Q.cpsi = S.cpsi; Q.use_psi = S.use_psi;
      }
      __syncthreads();
      if (!S.ok) goto fail;
    }
    // ---- 3D with a long-range kernel (the reference's trials: becgpp/solvers.py:165-174,
    // each a full energy with its own convolution): the trial density |psi - t dirc|^2 is
    // a - 2 t b + t^2 c and the potential is linear in it, so the long-range sum
    // sum Phi[|w|^2] |w|^2 of every trial is a quartic in t whose coefficients are
    // the pair sums of Phi_a (the current potential), Phi_b and Phi_c (two
    // convolutions here) with a, b, c; no trial needs a convolution of its own
    if (poly) {
      if (tid == 0) {
        Q.rmode = 6; Q.smode = 8; Q.Kq = I.Kq; Q.cscale = I.conv_scale; Q.cout = phi_buf(I, 2);
        Q.phia = phi_buf(I, S.phi_cur); Q.phisc = S.phisc;
      }
      __syncthreads();
      if (!conv_phases<N, M>(C, 1)) goto fail;
      if (tid == 0) {
        S.qG[1] = C.tot[0]; S.qG[3] = C.tot[1]; S.qG[4] = C.tot[2]; S.qG[0] = C.tot[3];
        Q.rmode = 7; Q.cout = phi_buf(I, 3); Q.phia = nullptr;
      }
      __syncthreads();
      if (!conv_phases<N, M>(C, 1)) goto fail;
      if (tid == 0) { S.qG[2] = C.tot[0]; S.qG[5] = C.tot[2]; }
      __syncthreads();
    }
    // ---- Armijo line search
    {
      const int phit = 1 - S.phi_cur;
      for (int ls = 0; ls < P.ls_max; ++ls) {
        const double t = S.trial;
        if (tid == 0) Q.t = t;
        __syncthreads();
        if (!energy_phases<N, M>(C, S, 0, ls == 0, pool_buf(I, S.f[F_W]), pool_buf(I, S.f[F_DIRC]),
                                 phi_buf(I, phit), !poly)) goto fail;
        if (tid == 0) {
          S.ntrials++;
          if (poly) {
            const double* G = S.qG;
            S.tsum[S_G] = (((G[5] * t - 4.0 * G[4]) * t + (2.0 * G[2] + 4.0 * G[3])) * t - 4.0 * G[1]) * t + G[0];
          }
          const double c = 1.0 / sqrt(S.tsum[S_N0] * dv);
          double comp[8];
          energy_assemble(I, S.tsum, c * c, comp);
          S.Et = comp[0]; S.ct = c;
          if (isfinite(S.Et) && S.Et <= S.E - P.c1 * t * S.gd) S.accepted = 1;
          else S.trial = t * P.shrink;
        }
        __syncthreads();
        if (S.accepted || S.trial < P.alpha_min) break;
      }
    }
    if (!S.accepted) {
      if (tid == 0) {
        S.n_fail++;
        S.alpha = fmax(S.alpha * 0.5, P.alpha_min);
        S.f[F_DIR] = S.f[F_Z];
        S.f[F_DIRC] = -1; S.f[F_W] = -1;
        S.need_pz = 0;
        S.do_switch = 0;
        if (S.fp32) {
          // mixed form: repeated failures mean the energy change has reached the
          // FP32 floor; the FP64 iterations take over instead of stopping
          S.done = 0;
          S.do_switch = (S.n_fail >= kMixedFailSwitch || S.alpha <= P.alpha_min);
        } else if (S.alpha <= P.alpha_min || S.n_fail >= P.stall_max) {
          S.stop = kStopStalled; S.done = 1;
        } else {
          S.done = 0;
        }
      }
      __syncthreads();
      if (S.done) break;
      if (S.do_switch && !switch_to_fp64<N, M>(C, S, it)) goto fail;
      continue;
    }
    if (poly) {
      // the accepted state's potential Phi[|w|^2] into the trial buffer: from the
      // parts, or every 32 accepted steps by a convolution of |w|^2 itself (so
      // rounding cannot build up over the updates)
      const int phit = 1 - S.phi_cur;
      double* out = phi_buf(I, phit);
      if ((S.naccept + 1) % 32 == 0) {
        if (tid == 0) { Q.rmode = 4; Q.W = pool_buf(I, S.f[F_W]); Q.cout = out; }
        __syncthreads();
        if (!conv_phases<N, M>(C, 0)) goto fail;
      } else {
        const double* pa = phi_buf(I, S.phi_cur);
        const double* pb = phi_buf(I, 2);
        const double* pc = phi_buf(I, 3);
        const double t = S.trial, sa = S.phisc;
        for (int f = C.T.rank * kThreads + tid; f < I.n; f += C.T.size * kThreads)
          st1(out + f, (sa * ld1(pa + f) - 2.0 * t * ld1(pb + f)) + t * t * ld1(pc + f));
        if (!phase_end0(C)) goto fail;
      }
    }
    // ---- accept: rotate the state
    if (tid == 0) {
      S.n_fail = 0;
      S.naccept++;
      S.f[F_PSIP] = S.f[F_PSI]; S.sc[F_PSIP] = S.sc[F_PSI];
      S.f[F_PSI] = S.f[F_W]; S.sc[F_PSI] = S.ct; S.f[F_W] = -1;
      S.f[F_GP] = S.f[F_G]; S.f[F_G] = -1;
      S.f[F_ZP] = S.f[F_Z]; S.f[F_Z] = -1;
      S.f[F_DIR] = S.f[F_DIRC]; S.f[F_DIRC] = -1;
      S.phi_cur = 1 - S.phi_cur; S.phisc = S.ct * S.ct;
      S.E = S.Et;
      S.alpha = fmin(P.alpha_max, S.trial * P.growth);
    }
    __syncthreads();
    if (!residual_phases<N, M>(C, S)) goto fail;
    if (S.fp32 && S.resid_rel < P.mixed_tol) {
      if (!switch_to_fp64<N, M>(C, S, it)) goto fail;
    }
    if (tid == 0) {
      S.need_pz = 1;
      S.done = 0;
      if (P.record_trace && S.ntrace < P.trace_cap) {
        double* tr = I.trace + 3 * S.ntrace;
        tr[0] = (double)(it + 1); tr[1] = S.E; tr[2] = S.resid_rel; S.ntrace++;
      }
      if (S.resid_rel < S.best_resid) {
        S.best_resid = S.resid_rel;
        S.f[F_BEST] = S.f[F_PSI]; S.sc[F_BEST] = S.sc[F_PSI];
      }
      if (S.fp32) {
        // convergence is declared in FP64 only
      } else if (S.resid_rel < P.res_tol) { S.converged = 1; S.stop = kStopConverged; S.done = 1; }
      else if (it - S.it_ref >= P.window) {
        const double dE = fabs(S.E - S.E_ref) / fmax(1.0, fabs(S.E));
        if (dE < P.etol) { S.converged = 1; S.stop = kStopEnergy; S.done = 1; }
        else { S.E_ref = S.E; S.it_ref = it; }
      }
    }
    __syncthreads();
    if (S.done) break;
    if (S.yield && it + 1 < P.maxit) {
      // hand the GPU back: save the state after this accepted iteration; the host
      // relaunches the unfinished instances with larger teams
      if (C.T.rank == 0 && tid == 0) {
        S.it_next = it + 1;
        *reinterpret_cast<Ctl*>(I.save) = S;
        SolveOut o{};
        o.status = 2;
        o.iters = S.n_iter;
        o.fp64_from = S.fp64_from;   // -1: still in FP32 transforms
        *I.out = o;
      }
      return;
    }
  }
  // ---- result: lowest-residual iterate, then its energy and residual afresh (FP64)
  if (tid == 0) Q.fp32 = 0;
  __syncthreads();
  {
    const int use_best = S.best_resid < S.resid_rel;
    const int fb = use_best ? F_BEST : F_PSI;
    const double2* src = pool_buf(I, S.f[fb]);
    const double sc = S.sc[fb];
    const int sp = S.fp32;     // still FP32 storage if the iterations ended before the hand-over
    for (int f = C.T.rank * kThreads + tid; f < I.n; f += C.T.size * kThreads)
      st2(I.out_c + f, cscale(ldp(src, f, sp), sc));
    if (!phase_end0(C)) goto fail;
    // energy terms of the returned state (and its potential into phi buffer 0)
    if (tid == 0) {
      Q.cin = I.out_c; Q.psi = I.out_c; Q.psc = 1.0;
      for (int q = 0; q < F_NLOG; ++q) if (q != F_A && q != fb) S.f[q] = -1;
      S.f[F_H] = pool_alloc(S);
    }
    __syncthreads();
    if (!energy_phases<N, M>(C, S, 2, 0, nullptr, nullptr, phi_buf(I, 0))) goto fail;
    double comp[8];
    energy_assemble(I, S.tsum, 1.0, comp);
    const double massf = S.tsum[S_N0] * dv;
    if (tid == 0) {
      Q.A = pool_buf(I, S.f[F_A]); Q.H = pool_buf(I, S.f[F_H]);
      Q.phi = kern ? phi_buf(I, 0) : nullptr; Q.phisc = 1.0;
    }
    __syncthreads();
    if (!hpsi_phases<N>(C)) goto fail;
    const double muf = C.tot[0] * dv;
    if (tid == 0) { Q.mu = muf; Q.gin = nullptr; Q.Gout = nullptr; Q.keys_on = 0; Q.win_on = 0; }
    __syncthreads();
    if (!grad_phase<N>(C, 0.0)) goto fail;
    const double raf = sqrt(C.tot[0] * dv);
    if (C.T.rank == 0 && tid == 0) {
      SolveOut o;
      o.iters = S.n_iter; o.stop = S.stop; o.converged = S.converged; o.ntrials = S.ntrials;
      o.ntrace = S.ntrace; o.best_is_final = use_best; o.status = 0; o.pad_ = S.naccept;
      o.E = S.E; o.resid_rel = S.resid_rel; o.resid_abs = S.resid_abs; o.best_resid = S.best_resid;
      o.sigma = S.sigma; o.mu = S.mu; o.alpha = S.alpha; o.maxrho = S.maxrho;
      o.E_final = comp[0]; o.mu_final = muf; o.resid_abs_final = raf;
      o.resid_rel_final = raf / fmax(1.0, fabs(muf)); o.mass_final = massf;
      o.fp64_from = S.fp64_from; o.pad2_ = 0;
      *I.out = o;
      __threadfence();
      if (I.finished) atomicAdd(I.finished, 1);
    }
    return;
  }
fail:
  if (C.T.rank == 0 && tid == 0) {
    SolveOut o{};
    o.stop = kStopError; o.status = 1; o.iters = S.n_iter;
    *I.out = o;
    if (I.finished) atomicAdd(I.finished, 1);
  }
}

// ------------------------------------------------------------- API programs
template <int N, int M>
BGP_D void prog_api(Ctx& C, Ctl& S) {
  const Inst& I = C.I;
  PassArgs& Q = C.Q;
  const int tid = threadIdx.x;
  const bool kern = (I.kind != kNone) && (M > 0);
  double* res = I.res;
  if (tid == 0) {
    Q.psi = I.in_psi; Q.psc = 1.0; Q.cin = I.in_psi;
    Q.cz = Q.cd = Q.cg = 0.0; Q.use_psi = 0; Q.t = 0.0; Q.fp32 = 0;
  }
  __syncthreads();
  if (I.prog == kProgEnergy) {
    double* phi_out = I.out_r ? I.out_r : phi_buf(I, 0);
    if (!energy_phases<N, M>(C, S, 2, 0, nullptr, nullptr, phi_out)) goto fail;
    if (C.T.rank == 0 && tid < kNRec) res[tid] = S.tsum[tid];
    return;
  }
  if (I.prog == kProgConv) {
    if (tid == 0) {
      Q.rmode = 2; Q.rin = I.in_phi;
      Q.Kq = I.which_w ? I.Wq : I.Kq;
      const double Md = (M > 0) ? (double)M : 1.0;
      Q.cscale = I.dv / ((BGP_DIM(I) == 2) ? Md * Md : Md * Md * Md);
      Q.cout = I.out_r;
    }
    __syncthreads();
    if (!conv_phases<N, M>(C)) goto fail;
    return;
  }
  if (I.prog == kProgConvW) {
    // potential of the virial kernel, -G_C dV (W * rho), and its sum against rho
    if (tid == 0) {
      Q.rmode = 0; Q.smode = 0;
      Q.Kq = I.Wq; Q.cscale = I.conv_scale; Q.cout = phi_buf(I, 1);
    }
    __syncthreads();
    if (!conv_phases<N, M>(C, 1)) goto fail;
    if (C.T.rank == 0 && tid == 0) res[0] = C.tot[S_G];
    return;
  }
  if (I.prog == kProgApplyH || I.prog == kProgResidual) {
    const double* phi = nullptr;
    if (kern && I.use_phi == 2) {
      if (tid == 0) {
        Q.rmode = 0; Q.Kq = I.Kq; Q.cscale = I.conv_scale; Q.cout = phi_buf(I, 0);
      }
      __syncthreads();
      if (!conv_phases<N, M>(C)) goto fail;
      phi = phi_buf(I, 0);
    } else if (I.use_phi == 1) {
      phi = I.in_phi;
    }
    double2* H = (I.prog == kProgApplyH) ? I.out_c : pool_buf(I, 1);
    if (tid == 0) { Q.A = pool_buf(I, 0); Q.H = H; Q.phi = phi; Q.phisc = 1.0; }
    __syncthreads();
    if (!hpsi_phases<N>(C)) goto fail;
    const double mu = C.tot[0] * I.dv;
    if (I.prog == kProgApplyH) {
      if (C.T.rank == 0 && tid == 0) { res[0] = mu; res[1] = C.tot[kNSum]; }
      return;
    }
    if (tid == 0) { Q.mu = mu; Q.gin = nullptr; Q.Gout = nullptr; Q.A = pool_buf(I, 2); Q.keys_on = 0; Q.win_on = 0; }
    __syncthreads();
    if (!grad_phase<N>(C, 0.0)) goto fail;
    if (C.T.rank == 0 && tid == 0) { res[0] = mu; res[1] = C.tot[0]; }
    return;
  }
  if (I.prog == kProgPrecond) {
    const double* phi = (I.use_phi == 1) ? I.in_phi : nullptr;
    // max rho of psi (rank 0 also clears the histograms)
    {
      Acc a; a.zero();
      if (C.T.rank == 0) for (int q = tid; q < 8 * 256 + 2; q += kThreads) I.hist[q] = 0u;
      for (int f = C.T.rank * kThreads + tid; f < I.n; f += C.T.size * kThreads)
        a.mx = fmax(a.mx, cabs2(ld2(I.in_psi + f)));
      if (!phase_end<0>(C, a)) goto fail;
    }
    const double maxrho = C.tot[kNSum];
    if (tid == 0) {
      Q.gin = I.in_grad; Q.H = nullptr; Q.Gout = nullptr; Q.A = pool_buf(I, 0);
      Q.phi = phi; Q.phisc = 1.0; Q.thr = 0.05 * maxrho; Q.keys_on = 1; Q.win_on = 0;
      S.win_used = 0;
    }
    __syncthreads();
    if (!grad_phase<N>(C, 0.0)) goto fail;
    if (tid == 0) S.nkeys = C.tot[3];
    __syncthreads();
    double sig;
    if (!median_phases(C, S, I.sp.shift_min, sig)) goto fail;
    const double sigma = fmax(sig, I.sp.shift_min);
    if (tid == 0) { Q.sigma = sigma; Q.Z = I.out_c; Q.A = pool_buf(I, 0); }
    __syncthreads();
    if (!precond_phases<N>(C)) goto fail;
    const double2 ap = cmk(C.tot[0] * I.dv, C.tot[1] * I.dv);
    for (int f = C.T.rank * kThreads + tid; f < I.n; f += C.T.size * kThreads)
      st2(I.out_c + f, csub(ld2(I.out_c + f), cmul(ap, ld2(I.in_psi + f))));
    if (C.T.rank == 0 && tid == 0) { res[0] = sigma; res[1] = sig; res[2] = maxrho; }
    return;
  }
fail:
  if (C.T.rank == 0 && tid == 0) res[kNRec] = 1.0;
}

BGP_NS_END  // namespace bgp
