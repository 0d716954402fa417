// Device side of the ground-state library: per-instance descriptors, the tiled
// line passes (Hamiltonian, energy, preconditioner, long-range convolution),
// the median selection and the persistent team solver.
//
// Layout in HBM. Every instance owns dense row-major complex128 fields of
// n = N^d points (index (i,j[,k]), k fastest), a pool of such fields for the
// solver, two real potential fields, and, with a long-range kernel, scratch for
// the zero-padded transform: 2D  N x (M/2+1) complex, 3D  N x N x (M/2+1) and
// N x M x (M/2+1) complex (M = pad N). The kernel transform is stored as its
// real, even quadrant Kq[(M/2+1)^d].
//
// Work decomposition. A CTA of 4 warps handles a tile of 4 lines of one axis:
// the lines are loaded into shared memory with coalesced accesses (consecutive
// threads on consecutive addresses), each warp transforms one line, and the
// tile is written back coalesced. A team of CTAs owns one instance and moves
// through phases separated by bounded team barriers; every CTA of a team runs
// the same scalar control code on the same reduced values, so the team never
// needs a broadcast.
#pragma once
#include "bgp_common.cuh"
#include "bgp_fft.cuh"

BGP_NS_BEGIN

constexpr double kTwoPi = 6.283185307179586;  // 2*pi rounded to double
constexpr int kNB = 13;                        // solver field pool size
constexpr int kNSum = 16;                      // summed slots of a reduction record
constexpr int kNRec = kNSum + 1;               // + one max slot
constexpr int kSelCap = 256;                   // median: candidates finished in-CTA
constexpr int kWinTarget = 64;                 // median: keys wanted in the window

enum Kind : int { kNone = 0, kNewton = 1, kLog = 2, kQ2d = 3 };

enum Prog : int {
  kProgSolve = 0,
  kProgApplyH = 1,   // out = H psi (phi from in_phi, or computed when use_phi == 2)
  kProgEnergy = 2,   // energy sums of psi (no normalisation) + phi
  kProgResidual = 3, // H psi, mu, ||H psi - mu psi||
  kProgPrecond = 4,  // z = P_T[(k^2/2 + sigma)^-1 grad], sigma
  kProgConv = 5,     // out_phi = scale * (K * rho) on the zero-padded grid
  kProgConvW = 6,    // sum of (potential of W * |psi|^2) |psi|^2 (q2d virial kernel W)
};

enum Stop : int { kStopMaxit = 0, kStopConverged = 1, kStopEnergy = 2, kStopStalled = 3,
                  kStopError = 4 };

// logical solver fields
enum Fld : int { F_PSI = 0, F_PSIP, F_BEST, F_W, F_G, F_GP, F_Z, F_ZP, F_DIR, F_DIRC, F_H, F_A,
                 F_NLOG };

struct SolverParams {
  int maxit, ls_max, stall_max, restart, cg_beta /*0 pr_precond, 1 pr, 2 none*/, window;
  int record_trace, trace_cap;
  int mixed;                      // 1: FP32 transforms until the hand-over to FP64
  double res_tol, etol, alpha0, alpha_min, alpha_max, shift_min, c1, shrink, growth;
  double bb_min, bb_max, bb_mix;
  double mixed_tol;               // hand over once the residual is below this
};

struct SolveOut {
  int iters, stop, converged, ntrials, ntrace, best_is_final, status, pad_;
  double E, resid_rel, resid_abs, best_resid, sigma, mu, alpha, maxrho;
  // the returned state, evaluated afresh (potential recomputed from it)
  double E_final, mu_final, resid_abs_final, resid_rel_final, mass_final;
  int fp64_from, pad2_;           // mixed form: iteration of the hand-over to FP64 (-1: none)
};

// Everything a team needs about its instance.
struct Inst {
  int ndim, N, M, kind;
  int n, Mh, i0, nM;              // nM = N^(d-1) * M rows of the padded scratch
  double dx, dv, kfac, s, tc;
  double beta2, beta3, Omega, G_C;
  double inv_n, conv_scale;       // 1/N^d; -G_C dV / M^d (potential from the K table)
  const double2* twN;
  const double2* twM;
  const float2* twN32;            // the same twiddles rounded to FP32 (mixed form)
  const float2* twM32;
  const double* Kq;               // K^ quadrant
  const double* Wq;               // W^ quadrant (q2d virial kernel), may be null
  // solver storage
  double2* pool;                  // kNB fields of n
  double* phi2;                   // 2 real fields of n
  double2* cb1;                   // conv scratch (2D: N*Mh, 3D: N*N*Mh)
  double2* cb2;                   // conv scratch 3D: N*M*Mh
  unsigned long long* keys;       // n median keys
  unsigned* hist;                 // 8 x 256 histograms + candidate and window counters
  unsigned long long* cand;       // kSelCap median candidates (radix path)
  unsigned long long* wcand;      // kSelCap median candidates (window path)
  double* part;                   // 2 x kNRec x team_size partials
  double* trace;                  // trace_cap x 2 (E, resid_rel)
  double* res;                    // API result record (kNRec x 4)
  unsigned long long* bar;        // team barrier counter
  unsigned long long* prof;       // phase profiler counters (BGP_PROF builds), else null
  int team_first, team_size;
  // segmented solve: saved control state, resume flag, and the yield rule
  void* save;                     // solver control state between launches
  int resume;                     // 1: continue from `save`
  int yield_at;                   // yield once this many instances of the launch finished
  int* finished;                  // instances of this launch that have finished
  // API operands
  int prog, use_phi, which_w;
  const double2* in_psi;          // psi (API) / psi0 (solve)
  const double2* in_grad;         // precond input
  const double* in_phi;           // given potential
  double2* out_c;                 // complex output (H psi, z, final psi)
  double* out_r;                  // real output (phi)
  SolverParams sp;
  SolveOut* out;
};

struct Launch {
  Inst* insts;
  const int* cta_inst;            // CTA -> instance
  int* abort_flag;
};

// ------------------------------------------------------------------ grid helpers
// Twiddle table of the N-lines (or M-lines) in the transform type T.
template <class T> BGP_D const T* twN_of(const Inst& I);
template <> BGP_D const double2* twN_of<double2>(const Inst& I) { return I.twN; }
template <> BGP_D const float2* twN_of<float2>(const Inst& I) { return I.twN32; }

// The grid helpers take an Inst or a Geo (the same field names): passes copy
// the scalars they need into a Geo in registers once, so the per-element code
// does not reload them from shared memory after every store.
struct Geo {
  int ndim, N, n;
  double dx, kfac, s, tc, beta2, beta3, Omega;
};
BGP_D Geo geo_of(const Inst& I) {
  return Geo{BGP_DIM(I), I.N, I.n, I.dx, I.kfac, I.s, I.tc, I.beta2, I.beta3, I.Omega};
}
// The same with the line length a compile-time constant (index arithmetic by
// constants instead of divisions).
template <int NT>
struct GeoT {
  static constexpr int N = NT;
  int ndim, n;
  double dx, kfac, s, tc, beta2, beta3, Omega;
};
template <int NT>
BGP_D GeoT<NT> geo_t(const Inst& I) {
  return GeoT<NT>{BGP_DIM(I), I.n, I.dx, I.kfac, I.s, I.tc, I.beta2, I.beta3, I.Omega};
}

template <class G>
BGP_D double xcoord(const G& g, int i) { return (double)(i - g.N / 2) * g.dx; }
template <class G>
BGP_D double kof(const G& g, int m) {
  const int mm = (m < (g.N + 1) / 2) ? m : m - g.N;
  return kTwoPi * ((double)mm * g.kfac);
}
template <class G>
BGP_D double potential(const G& g, int i, int j, int k) {
  const double x = xcoord(g, i), y = xcoord(g, j);
  double r2 = x * x + y * y;
  if (BGP_DIM(g) == 3) { const double z = xcoord(g, k); r2 = r2 + z * z; }
  if (g.s <= 0.0) return 0.0;
  return (g.s == 2.0) ? g.tc * r2 : g.tc * pow(r2, 0.5 * g.s);
}

// Element (r, c) of tile `t` of the N-lines along axis `ax`: flat index and
// coordinates. Lines along the last axis are contiguous; the others are strided
// and a tile groups kLines neighbours in the last axis.
template <class G>
BGP_D int nline_elem(const G& g, int ax, int t, int r, int c, int& i, int& j, int& k) {
  const int N = g.N;
  if (BGP_DIM(g) == 2) {
    k = 0;
    if (ax == 1) { i = t * kLines + c; j = r; } else { j = t * kLines + c; i = r; }
    return i * N + j;
  }
  const int tpl = N / kLines;
  if (ax == 2) { const int line = t * kLines + c; i = line / N; j = line - i * N; k = r; }
  else if (ax == 1) { i = t / tpl; k = (t - i * tpl) * kLines + c; j = r; }
  else { j = t / tpl; k = (t - j * tpl) * kLines + c; i = r; }
  return (i * N + j) * N + k;
}
BGP_HD int ntiles_axis(const Inst& I) { return BGP_DIM(I) == 2 ? I.N / kLines : (I.N * I.N) / kLines; }

// Coalesced thread -> (r, c) maps for a tile of kLines lines of length L.
template <int L>
BGP_D void map_contig(int e, int& r, int& c) { c = e / L; r = e - c * L; }
template <int L>
BGP_D void map_strided(int e, int& r, int& c) { r = e / kLines; c = e % kLines; }

// ------------------------------------------------------------- reduction records
// Shared reduction scratch of a CTA: (kNSum + 1) x kWarps warp totals, then a
// 256-bin histogram of the gradient pass (128 doubles).
constexpr int kSredDoubles = (kNSum + 1) * kWarps + 128;

struct Acc {
  double s[kNSum];
  double mx;
  BGP_D void zero() {
#pragma unroll
    for (int i = 0; i < kNSum; ++i) s[i] = 0.0;
    mx = 0.0;
  }
};

// Write this CTA's record (block-reduced) into partial slot `slot`.
// Only the first NV summed slots and the max slot are reduced and written.
// Warps reduce their values by shuffles (reduce-scatter for NV >= 4), the warp
// totals meet in shared memory, and thread q adds slot q's eight warp totals in
// warp order. sred must hold (kNSum + 1) * kWarps doubles.
template <int NV>
BGP_D void acc_commit(const Inst& I, const Team& T, Acc& a, int slot, double* sred) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double m = a.mx;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if constexpr (NV >= 4) {
    double v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = (i < NV) ? a.s[i] : 0.0;
    warp_rs16(v, lane);
    __syncthreads();
    const int q = rs16_slot(lane);
    if ((lane & 1) == 0 && q < NV) sred[q * kWarps + w] = v[0];
  } else {
    double v[NV > 0 ? NV : 1];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double x = a.s[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      v[i] = x;
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < NV; ++i) sred[i * kWarps + w] = v[i];
    }
  }
  if (lane == 0) sred[kNSum * kWarps + w] = m;
  __syncthreads();
  const int q = threadIdx.x;
  if (q < NV || q == kNSum) {
    double val = sred[q * kWarps];
#pragma unroll
    for (int k = 1; k < kWarps; ++k) {
      const double x = sred[q * kWarps + k];
      val = (q == kNSum) ? fmax(val, x) : val + x;
    }
    st1(I.part + ((size_t)slot * kNRec + q) * I.team_size + T.rank, val);
  }
}

// After the team barrier: team totals of slot `slot` (identical in every CTA).
template <int NV>
BGP_D void acc_gather(const Inst& I, int slot, double* tot /* smem kNRec */) {
  // G threads per reduced value (slots 0..NV-1 and the max slot; G = 32, 16 or
  // 8, as many as the CTA has for them): each issues all of its partial loads
  // of a round before using any, then the G partial results meet in a fixed
  // shuffle tree, so every CTA forms the same totals.
  constexpr int G = ((NV + 1) * 32 <= kThreads) ? 32 : (((NV + 1) * 16 <= kThreads) ? 16 : 8);
  constexpr int U = (G == 8) ? 16 : 8;   // partial loads of a thread in flight per round
  static_assert((NV + 1) * G <= kThreads, "too many reduced values for one CTA");
  const int tid = threadIdx.x, lane = tid & 31;
  for (int q = tid + NV; q < kNSum; q += kThreads) tot[q] = 0.0;
  const int v = tid / G, g = tid % G;
  const int ts = I.team_size;
  if (v <= NV) {
    const int q = (v == NV) ? kNSum : v;
    const bool mx = (q == kNSum);
    const double* p = I.part + ((size_t)slot * kNRec + q) * ts;
    double x = 0.0;
    for (int r0 = g; r0 < ts; r0 += G * U) {
      double y[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * G;
        y[u] = (r < ts) ? ld1(p + r) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) x = mx ? fmax(x, y[u]) : x + y[u];
    }
    unsigned mask = 0xFFFFFFFFu;
    if constexpr (G < 32) mask = ((1u << G) - 1u) << (lane & ~(G - 1));
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const double z = __shfl_xor_sync(mask, x, o);
      x = mx ? fmax(x, z) : x + z;
    }
    if (g == 0) tot[q] = x;
  }
  __syncthreads();
}

// ------------------------------------------------------------------ pass operands
// Operands of the passes of one phase. They live in shared memory (written by
// thread 0 before the phase) so every thread reads them by broadcast instead of
// holding copies in registers.
struct PassArgs {
  // psi = psc * psi_buf
  const double2* psi;
  double psc;
  // direction: dirc = cz z + cd d + cg g + cpsi psi (terms with zero coefficient not read)
  const double2* dz;
  const double2* dd;
  const double2* dg;
  double cz, cd, cg;
  double2 cpsi;
  int use_psi;
  double t;                      // trial step
  double2* W;                    // trial state w = psi - t dirc
  double2* DIRC;                 // materialised direction
  const double2* src;            // stored state for the later axes
  double2* A;                    // scratch / accumulator field
  double2* H;                    // H psi output
  double2* Gout;                 // gradient output
  const double2* gin;            // given gradient (preconditioner API)
  double2* Z;                    // preconditioned output
  const double* phi;             // potential (scaled by phisc), may be null
  double phisc, mu, thr, sigma;
  // convolution
  int rmode;                     // density source (see rho_at)
  int smode;                     // |w|^2 source of the energy sum
  const double* rin;             // real density input
  const double* phia;            // sum source 8: the current potential (times phisc)
  const double2* cin;            // complex state input (|cin|^2)
  const double* Kq;              // kernel quadrant
  double cscale;                 // output scale
  double* cout;                  // real output
  int sum_on;
  // pass selectors
  int ax, stage, mode, first, write_w, write_dirc, init, keys_on, inverse;
  unsigned* shist;               // CTA histogram (shared memory)
  unsigned long long win_lo, win_hi;  // median window (keys), used when win_on
  int win_on;
  int fp32;                      // FP32 transforms in the mixed-precision passes
};

// Operands of one tile element. A pass first issues every load of a batch of
// elements (`fetch`), then computes and stores (`enter` / `leave`), so no load
// waits behind a store that the compiler cannot prove independent of it.
struct Pre {
  double2 a, b, c;
  double r;
};

BGP_D double2 czero() { return cmk(0.0, 0.0); }

// Solver pool fields in the storage precision of the phase. While the mixed form
// runs in FP32 (sp != 0) a pool field holds complex64: element f of a float2
// view of the field's buffer (its first half). Everything else (the caller's
// fields, the convolution scratch, the potentials) is always complex128 / FP64.
// In the FP64-only builds the FP32 branch is not compiled.
BGP_D double2 ldp(const double2* p, int f, int sp) {
#if BGP_MIXED
  if (sp) {
    const float2 v = __ldcg(reinterpret_cast<const float2*>(p) + f);
    return cmk((double)v.x, (double)v.y);
  }
#endif
  (void)sp;
  return ld2(p + f);
}
BGP_D void stp(double2* p, int f, double2 v, int sp) {
#if BGP_MIXED
  if (sp) {
    float* q = reinterpret_cast<float*>(reinterpret_cast<float2*>(p) + f);
    asm volatile("st.global.cg.v2.f32 [%0], {%1, %2};" ::"l"(q), "f"((float)v.x), "f"((float)v.y));
    return;
  }
#endif
  (void)sp;
  st2(p + f, v);
}
// A value rounded to the storage precision: a trial state and its direction are
// rounded before their norm and energy sums are taken, so that the sums belong to
// the state that is stored (and accepted) in complex64.
BGP_D double2 rnd_sp(double2 v, int sp) {
#if BGP_MIXED
  if (sp) return cmk((double)(float)v.x, (double)(float)v.y);
#endif
  (void)sp;
  return v;
}
BGP_D double2 psi_at(const PassArgs& Q, int f) { return cscale(ldp(Q.psi, f, Q.fp32), Q.psc); }

// Operands of the direction combination  dirc = cz z + cd d + cg g + cpsi psi
// and of the trial state  psi - t dirc, copied into registers by a pass.
struct DirArgs {
  const double2 *psi, *dz, *dd, *dg, *DIRC;
  double psc, cz, cd, cg, t;
  double2 cpsi;
  int use_psi;
  int sp;                        // pool fields stored in FP32 (mixed form)
};
BGP_D DirArgs dir_args(const PassArgs& Q) {
  return DirArgs{Q.psi, Q.dz, Q.dd, Q.dg, Q.DIRC, Q.psc, Q.cz, Q.cd, Q.cg, Q.t, Q.cpsi, Q.use_psi, Q.fp32};
}

// Loads of the direction combination. At most two of the field terms are active
// (cz with cd, cz alone, or cg alone), so they go to P.b (z or g) and P.c (d);
// psi goes to P.a.
BGP_D void dirc_fetch(const DirArgs& D, int f, Pre& P) {
  P.a = cscale(ldp(D.psi, f, D.sp), D.psc);
  P.b = (D.cz != 0.0) ? ldp(D.dz, f, D.sp) : ((D.cg != 0.0) ? ldp(D.dg, f, D.sp) : czero());
  P.c = (D.cd != 0.0) ? ldp(D.dd, f, D.sp) : czero();
}
BGP_D double2 dirc_of(const DirArgs& D, const Pre& P) {
  double2 v = czero();
  if (D.cz != 0.0) v = cscale(P.b, D.cz);
  if (D.cd != 0.0) v = cadd(v, cscale(P.c, D.cd));
  if (D.cz == 0.0 && D.cg != 0.0) v = cadd(v, cscale(P.b, D.cg));
  if (D.use_psi) v = cadd(v, cmul(D.cpsi, P.a));
  return v;
}

// Density sources: 0 |psi|^2, 1 |psi - t dirc|^2 (combination), 2 real input,
// 3 |cin|^2, 4 |W|^2, 5 |psi - t DIRC|^2, 6 Re(conj(psi) dirc), 7 |dirc|^2
// (the linear and quadratic parts of the trial density in t, dirc the
// combination). Sum source 8 (the convolution's last pass only): psi and dirc
// with the current potential Phi_a = phisc * phia, for the pair sums of the
// line search's quartic.
struct RhoArgs {
  DirArgs d;
  const double* rin;
  const double2 *cin, *W;
  const double* phia;
  double phisc;
  int mode;
};
BGP_D RhoArgs rho_args(const PassArgs& Q, int mode) {
  return RhoArgs{dir_args(Q), Q.rin, Q.cin, Q.W, Q.phia, Q.phisc, mode};
}
BGP_D void rho_fetch(const RhoArgs& R, int f, Pre& P) {
  switch (R.mode) {
    case 0: P.a = cscale(ldp(R.d.psi, f, R.d.sp), R.d.psc); break;
    case 1: dirc_fetch(R.d, f, P); break;
    case 2: P.r = ld1(R.rin + f); break;
    case 3: P.a = rnd_sp(ld2(R.cin + f), R.d.sp); break;   // the caller's state: complex128
    case 4: P.a = ldp(R.W, f, R.d.sp); break;
    case 6: case 7: dirc_fetch(R.d, f, P); break;
    case 8: dirc_fetch(R.d, f, P); P.r = R.phia ? R.phisc * ld1(R.phia + f) : 0.0; break;
    default: P.a = cscale(ldp(R.d.psi, f, R.d.sp), R.d.psc); P.b = ldp(R.d.DIRC, f, R.d.sp); break;
  }
}
// the three parts of the trial density |psi - t d|^2 = a - 2 t b + t^2 c (d the
// direction as the first trial pass rounds and stores it)
BGP_D void rho_parts(const RhoArgs& R, const Pre& P, double& a, double& b, double& c) {
  const double2 d = rnd_sp(dirc_of(R.d, P), R.d.sp);
  a = cabs2(P.a);
  b = P.a.x * d.x + P.a.y * d.y;
  c = cabs2(d);
}
BGP_D double rho_of(const RhoArgs& R, const Pre& P) {
  switch (R.mode) {
    case 1: return cabs2(rnd_sp(csub(P.a, cscale(rnd_sp(dirc_of(R.d, P), R.d.sp), R.d.t)), R.d.sp));
    case 2: return P.r;
    case 5: return cabs2(rnd_sp(csub(P.a, cscale(P.b, R.d.t)), R.d.sp));
    case 6: { double a, b, c; rho_parts(R, P, a, b, c); return b; }
    case 7: { double a, b, c; rho_parts(R, P, a, b, c); return c; }
    default: return cabs2(P.a);
  }
}

BGP_NS_END  // namespace bgp
