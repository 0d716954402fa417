/* bgp.h -- C ABI of the B200 ground-state library (libbgp.so).
 *
 * Gross-Pitaevskii(-Poisson) energy functional on uniform 2D/3D grids: the
 * Hamiltonian apply, energy and residual, the zero-padded long-range
 * convolution, the Sobolev preconditioner and the device-resident normalised
 * preconditioned CG solver, for one instance or a batch of instances.
 *
 * Conventions
 *   - Fields are dense row-major arrays of N^d points (index (i,j[,k]), last
 *     index fastest); complex fields are interleaved complex128 (double re, im).
 *   - Every pointer named psi/hpsi/phi/... is a DEVICE pointer owned by the
 *     caller; the library never frees caller memory. Plans own their scratch.
 *   - `stream` is a cudaStream_t (0 = legacy default stream). Calls are
 *     stream-ordered and return after the results they report are on the host.
 *   - Every function returns BGP_OK (0) or a negative BGP_ERR_* code;
 *     bgp_last_error() gives the message of the last failure in this thread.
 *   - A plan is used by one host thread at a time: its scratch, its pass
 *     schedules and the side streams and events of its batched apply belong to
 *     it; different plans may be used from different threads.
 *
 * Reference interfaces replaced (becGPP v1.2.1, paths within that project):
 *   bgp_plan_create    make_grid + _build_kernel_fft       becgpp/grid.py:69-101,
 *                                                            becgpp/interactions.py:112-151
 *   bgp_apply_H        apply_H                             becgpp/operators.py:36-45
 *   bgp_energy         energy_components                   becgpp/operators.py:10-29
 *   bgp_residual       compute_residual                    becgpp/operators.py:48-52
 *   bgp_convolve       kernel_convolution / long_range_phi becgpp/interactions.py:154-171
 *   bgp_precondition   _preconditioner                     becgpp/solvers.py:28-45
 *   bgp_solve          ground_state (loop, lines 48-226); a batch of instances
 *                      replaces the sequential loops of ground_state_multiseed
 *                      (becgpp/solvers.py:238-263) and mode_sweep (becgpp/modes.py:340-386)
 */
#ifndef BGP_H_
#define BGP_H_

#ifdef __cplusplus
extern "C" {
#endif

#define BGP_OK 0
#define BGP_ERR_ARG -1        /* invalid argument (bad size, kernel, pointer)    */
#define BGP_ERR_CUDA -2       /* CUDA runtime error (launch, copy, no device)    */
#define BGP_ERR_OOM -3        /* device allocation failed                        */
#define BGP_ERR_DEVICE -4     /* a bounded device wait gave up (status word set) */
#define BGP_ERR_UNSUPPORTED -5 /* grid size / padding not compiled in            */

#define BGP_KERNEL_NONE 0
#define BGP_KERNEL_NEWTON 1   /* 1/r (2D or 3D)            */
#define BGP_KERNEL_LOG 2      /* -ln r (2D)                */
#define BGP_KERNEL_Q2D 3      /* quasi-2D Gaussian pancake */

#define BGP_STOP_MAXIT 0
#define BGP_STOP_CONVERGED 1
#define BGP_STOP_ENERGY 2
#define BGP_STOP_STALLED 3
#define BGP_STOP_ERROR 4

#define BGP_CG_PR_PRECOND 0
#define BGP_CG_PR 1
#define BGP_CG_NONE 2

typedef struct bgp_plan bgp_plan;

/* One problem instance (becgpp make_grid keys: dimension, Ngrid, L, pad, s,
 * trap_coeff, kernel, l_z; physics: beta2, beta3, Omega, G_C). */
typedef struct {
  int ndim;          /* 2 or 3                                            */
  int N;             /* grid points per axis                             */
  int pad;           /* zero padding of the long-range transform (2)     */
  int kernel;        /* BGP_KERNEL_*                                      */
  double L;          /* half box: domain [-L, L)^d                       */
  double s;          /* trap power                                        */
  double trap_coeff; /* V = trap_coeff * r^s                              */
  double beta2, beta3, Omega, G_C, l_z;
} bgp_instance_desc;

/* Solver settings (becgpp config keys of the same names). */
typedef struct {
  int maxit, linesearch_max, linesearch_stall, cg_restart, cg_beta, conv_window;
  int record_trace, trace_cap;
  int mixed;   /* 0: FP64 throughout; 1: mixed form: the solver's bulk fields stored
                  as complex64 and transformed in FP32, while the norms, energies,
                  inner products, Armijo test and long-range potential stay FP64;
                  hands over to FP64 storage and transforms at mixed_switch_res or
                  after three consecutive failed line searches; convergence is only
                  declared in FP64 */
  double res_tol, energy_tol, step, step_max, precond_shift_min;
  double mixed_switch_res;
} bgp_solver_params;

/* Per-instance outcome of bgp_solve. E, mu, resid_* are those of the last
 * accepted iterate; the returned state is the lowest-residual iterate
 * (best_is_final says whether it differs from the last), and *_final are its
 * energy and residual evaluated afresh on the device. */
typedef struct {
  int iters, stop_reason, converged, ntrials, ntrace, best_is_final, status, naccepted;
  double E, resid_rel, resid_abs, min_resid, sigma, mu, alpha, maxrho;
  /* the returned state evaluated afresh, phi recomputed (compute_residual + energy): */
  double E_final, mu_final, resid_abs_final, resid_rel_final, mass_final;
  int fp64_from, reserved; /* mixed form: iteration at which FP64 took over (-1: never) */
} bgp_solve_result;

/* Energy terms, in the order of energy_components: */
typedef struct {
  double E, Ekin, Etrap, Econtact, Ethree, Erot, Egrav, Lz;
  double mass, r2mean, peak, rperp2, z2;   /* extra sums for observables */
} bgp_energy_terms;

int bgp_version(void);
const char* bgp_last_error(void);

/* Create a plan for n_inst instances (kernel tables are built here, on the
 * device, and synchronously). */
int bgp_plan_create(const bgp_instance_desc* desc, int n_inst, bgp_plan** plan);
int bgp_plan_destroy(bgp_plan* plan);
/* Device bytes held by the plan. */
long long bgp_plan_bytes(const bgp_plan* plan);
/* Solver-kernel launches issued through the plan so far (a solve relaunches
 * its unfinished instances with larger teams as others finish). */
long long bgp_plan_launches(const bgp_plan* plan);

/* Relaunch-schedule autotuner of bgp_solve (no counterpart in the reference).
 * A batched solve is a sequence of persistent launches: a launch yields once a
 * fraction 1/d of its instances has finished and the rest are relaunched with
 * larger teams. With enable = 1 the next three batched solves of the plan try
 * d = 2, 4 and 8 in turn, timed on the device, and later solves use the fastest
 * (the tuner assumes repeated solves of comparable inputs). */
int bgp_plan_autotune(bgp_plan* plan, int enable);
/* The schedule in use: yield divisor d, whether tuning has finished, and the
 * measured milliseconds of the three candidates (ms3 nullable). */
int bgp_plan_schedule(const bgp_plan* plan, int* yield_div, int* tuned, float* ms3);

/* hpsi = H psi. phi_mode 0: no long-range term; 1: use the given phi (real,
 * N^d); 2: compute phi from |psi|^2. mu_out (nullable) gets Re<psi,H psi> dV. */
int bgp_apply_H(bgp_plan* plan, int inst, const void* psi, void* hpsi, const double* phi,
                int phi_mode, double* mu_out, void* stream);

/* H psi of n instances of the plan in one call (no counterpart in the reference,
 * which applies H to one state at a time, becgpp/operators.py:36-45): plain
 * per-axis launches over all n at once (instances of one grid size share a
 * launch), with no persistent kernel and no host synchronisation: it returns
 * once the work is enqueued on `stream`. idx[a]: instance index (each at most
 * once per call); psi[a], hpsi[a]: device fields of that instance (not aliased);
 * phi_mode as in bgp_apply_H (2: the potential is computed from |psi|^2 into the
 * plan's scratch), phi[a] with phi_mode 1; mu_dev (nullable): device array,
 * mu_dev[a] = Re<psi, H psi> dV. Instances of different sizes run as groups on
 * the plan's side streams, forked from and joined to `stream` by events (one
 * capturable call). The first call for a grid size N tunes that
 * size's pass schedule on the call's data (bgp_plan_stream_schedule) and waits
 * for its timing runs. */
int bgp_apply_H_batch(bgp_plan* plan, int n, const int* idx, const void* const* psi, void* const* hpsi,
                      const double* const* phi, int phi_mode, double* mu_dev, void* stream);

/* Pass schedule of the batched apply for line length N (autotuner of the
 * project, no counterpart in the reference): lines per tile (1, 2, 4, 8, 16) and the
 * line FFT's radix order (0: Stockham stages, largest radix first; 1: reversed;
 * 2: radix 4 first; 3: register-resident transform, N = 32 R: an R-point DFT per
 * lane and a 32-point transform across the lanes; 4-7: the same four at twice the
 * resident warps, with half the registers), and the convolution's lines
 * per tile of its contiguous passes (1, 2, 4, 8) and of its strided passes (1, 2,
 * 4, 8, 16; 16 where the tile fits in shared memory) and its radix order (0 or 3);
 * tuned = 0 not yet, 1 tuned, 2 fixed by bgp_plan_stream_set. cand (nullable)
 * receives up to *ncand (lines, order, strided lines, ms) quadruples of the
 * timed candidates (lines < 0: convolution candidates, whose -lines is the
 * contiguous width; strided lines 0 for the H psi candidates); *ncand is set
 * to their number. */
int bgp_plan_stream_schedule(bgp_plan* plan, int N, int* lines, int* radix_order, int* conv_lines,
                             int* conv_strided_lines, int* conv_order, int* tuned, float* cand, int* ncand);
/* Fix the schedule of line length N (lines = 0: tune again on the next call). */
int bgp_plan_stream_set(bgp_plan* plan, int N, int lines, int radix_order, int conv_lines,
                        int conv_strided_lines, int conv_order);

/* Energy terms of psi as given (not normalised); phi_out (nullable, N^d real)
 * receives the long-range potential. */
int bgp_energy(bgp_plan* plan, int inst, const void* psi, double* phi_out,
               bgp_energy_terms* terms, void* stream);

/* Gradient of the energy functional at psi (as given, not normalised); no
 * counterpart in the reference, derived from energy_components
 * (becgpp/operators.py:10-29). terms = the energy terms of bgp_energy;
 * dE_dpsi (nullable, complex N^d) = dE/dpsi* = H psi dV (torch's complex
 * gradient of a real E is twice this); dparams[5] = dE/d(beta2, beta3, G_C,
 * Omega, l_z). dE/dG_C = Egrav/G_C (0 without a long-range kernel); dE/dl_z
 * uses dK/dl_z = -(K + W)/l_z with the q2d virial kernel W (0 unless q2d).
 * At a converged ground state these are the parameter sensitivities of the
 * ground-state energy (Hellmann-Feynman). */
int bgp_energy_grad(bgp_plan* plan, int inst, const void* psi, bgp_energy_terms* terms,
                    void* dE_dpsi, double* dparams, void* stream);

/* out3 = {resid_abs, mu, resid_rel} with phi recomputed from psi. */
int bgp_residual(bgp_plan* plan, int inst, const void* psi, double* out3, void* stream);

/* out = scale * (K * rho) on the zero-padded grid, scale = dV: the discrete
 * free-space convolution (which 0: interaction kernel, 1: q2d virial kernel). */
int bgp_convolve(bgp_plan* plan, int inst, const double* rho, double* out, int which,
                 void* stream);

/* z = P_T[(k^2/2 + sigma)^-1 grad]; sigma_out = the shift used. phi nullable. */
int bgp_precondition(bgp_plan* plan, int inst, const void* grad, const void* psi,
                     const double* phi, double shift_min, void* z, double* sigma_out,
                     void* stream);

/* Solve every instance of the plan in one persistent launch. psi0[i] and
 * psi_out[i] are device pointers (may be equal). trace (nullable, host) gets
 * trace_cap x 3 doubles per instance: (iteration, E, resid_rel). */
int bgp_solve(bgp_plan* plan, const void* const* psi0, void* const* psi_out,
              const bgp_solver_params* params, bgp_solve_result* results, double* trace,
              void* stream);

/* H psi without a plan and without any device allocation (no counterpart in
 * the reference). For callers that cannot call cudaMalloc: a host framework
 * that owns the device-memory budget and forbids its plugins to allocate, or a
 * time-critical loop that cannot afford cudaMalloc's device-wide
 * synchronisation. The scratch field and the twiddle table are fixed static
 * device arrays shared by every call, so at most 262144 grid points (2D up to
 * 512^2, 3D up to 64^3); larger grids return BGP_ERR_ARG. phi is the
 * long-range potential (N^d real) or NULL for none; hpsi must not alias psi.
 * Calls that overlap on the GPU race on the shared scratch and on the shared
 * twiddle table (each call rewrites it for its N) and must be serialised by
 * the caller. The first call on a device looks up the arrays' addresses and
 * keeps them for the life of the device's primary context; make it before any
 * stream capture, and make no call after cudaDeviceReset. Enqueued on
 * `stream`; returns without waiting. */
int bgp_apply_H_noalloc(const bgp_instance_desc* desc, const void* psi, void* hpsi,
                        const double* phi, void* stream);

/* Thomas-Fermi reference density of instance `inst` on the device
 * (becgpp/thomasfermi.py:65-120): nonlocal = 1 runs the relaxed fixed point of
 * the compressed TF density with the plan's long-range kernel (`iters` steps at
 * most, mixing `relax`, stop when sum |n_new - n| dV < 1e-9); nonlocal = 0 solves
 * the local inverted profile once. Each step's chemical potential is found by
 * the reference's bracket expansion and 90 bisection halvings, every one a
 * full-grid sum on the device (no host round trip per halving). V_eff uses the
 * given Omega. n_out: device N^d doubles (the density, unit mass). info[5] =
 * {mu (NaN: no bracket), converged, final dn, steps taken, device status}. */
int bgp_tf_density(bgp_plan* plan, int inst, int nonlocal, double Omega, int iters, double relax,
                   double* n_out, double* info, void* stream);

/* Density diagnostics on a device field rho of N^d doubles on the grid of half
 * box L (plans not needed). Synchronous: results are on the host on return.
 *   bgp_density_center   mass = sum rho dV and centre of mass       becgpp/fields.py:9-14
 *   bgp_mass_quantiles   radii around `center` (NULL: the centre of   becgpp/fields.py:17-30
 *                        mass) enclosing the fractions of max(rho,0) dV: the
 *                        distance of the first point, in distance order,
 *                        whose running mass reaches the fraction
 *   bgp_radial_profile   mean of f over the shells [edges[b],         becgpp/fields.py:37-57
 *                        edges[b+1]) around `center` (the last shell takes
 *                        everything beyond; NaN where empty; bins <= 2048) */
int bgp_density_center(int ndim, int N, double L, const double* rho, double* mass_out,
                       double* center_out, void* stream);
int bgp_mass_quantiles(int ndim, int N, double L, const double* rho, const double* center,
                       const double* fractions, int nf, double* radii_out, void* stream);
int bgp_radial_profile(int ndim, int N, double L, const double* f, const double* center,
                       const double* edges, int bins, double* prof_out, void* stream);

/* Resample a complex field from the N_old^d grid of half box L_old onto the
 * N_new^d grid of half box L_new by multilinear interpolation between the old
 * nodes, zero outside them (the interpolation of resample_state,
 * becgpp/grid.py:140-161; the caller normalises). Enqueued on `stream`. */
int bgp_resample(int ndim, int N_old, double L_old, const void* psi_old, int N_new, double L_new,
                 void* psi_new, void* stream);

/* Vortex count of a 2D field psi (complex128, N x N, element (i, j) at i N + j,
 * x_i = (i - N/2) dx, dx = 2L/N; a 3D state passes its z = 0 midplane): the
 * plaquettes whose wrapped phase increments sum to +-2 pi, inside the droplet
 * (Gaussian-smoothed density of width min(2 sqrt(pi/|Omega|), max(R/3, 2 dx))
 * above thresh_frac of its maximum, first corner within the 99 % mass radius R
 * around the centre of mass); out[4] = {Nv, Nplus, Nminus, Nnet}, all zero when
 * the mass or R is not positive. Replaces becgpp/vortex.py:10-48
 * (_count_vortices_2d). Synchronises `stream`. */
int bgp_vortex_count(int N, double L, const void* psi, double Omega, double thresh_frac, int* out,
                     void* stream);
/* Lowest-Landau-level weight of a 2D field: sum over m <= mcap of
 * |<phi_m, psi / |psi|>|^2 with phi_m ~ r^m e^(-r^2/2) e^(i m theta) normalised on
 * the grid (theta negated for Omega < 0), mcap from <r^2> and Mmax as the
 * reference; *out clamped to [0, 1]. Replaces becgpp/vortex.py:61-84
 * (lll_weight). Synchronises `stream`. */
int bgp_lll_weight(int N, double L, const void* psi, double Omega, int Mmax, double* out, void* stream);

/* Host-only helpers (no GPU needed): e^x K0(x), e^x K1(x) as used by the q2d
 * kernel table, and whether a grid size is compiled in. */
double bgp_k0e(double x);
double bgp_k1e(double x);
int bgp_size_supported(int ndim, int N, int pad, int kernel);

#ifdef __cplusplus
}
#endif
#endif /* BGP_H_ */
