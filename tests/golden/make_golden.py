"""Generate the golden fixtures under tests/golden/ by running becGPP v1.2.1 itself.

Run where the reference source tree is readable; its path is the required first
argument. The fixtures are committed, so the machines that run the GPU tests never
need the reference. matplotlib is not needed by any fixture, so a
stand-in module is registered before the import (becgpp/figures.py imports it at
module load).

    python tests/golden/make_golden.py REF_DIR            # small fixtures (~2 min)
    python tests/golden/make_golden.py REF_DIR --big      # benchmark-configuration runs (~40 min)
    python tests/golden/make_golden.py REF_DIR --grads    # energy gradients (~1 min)
    python tests/golden/make_golden.py REF_DIR --stopstats  # c1 stop reasons over 40 seeds (~1 min)
    python tests/golden/make_golden.py REF_DIR --bigops     # operators at benchmark sizes (~2 min)
    python tests/golden/make_golden.py REF_DIR --tf         # Thomas-Fermi references

Outputs
  ops.npz         operator cases: psi, H psi, phi, energy terms, residual, observables,
                  preconditioner output, for 2D / quasi2D / 3D and every kernel
  kernels.npz     kernel transforms K^ (real part) of small grids, all kernel kinds
  seeds.npz       reference seeds (gaussian / tf / flat-top tf / triangular)
  solves.npz      small ground-state solves: psi0, final psi, observables, E trace
  baseline_runs.json  (--big) the benchmark configurations' final observables
  diag.npz/json       (--diag) vortex count / LLL weight of synthetic states, diagnostics()
                      of solved states, run() in single and sweep mode
  grads.npz       (--grads) torch autograd through the reference's energy_components:
                  dE/dpsi and dE/d(beta2, beta3, G_C, Omega); central differences in l_z;
                  and ground-state energies at shifted parameters (Hellmann-Feynman check)
"""
import json
import math
import os
import sys
import tempfile
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference(ref_dir):
    os.environ.setdefault("GPP_OUTDIR", tempfile.mkdtemp(prefix="golden_out_"))
    try:
        import matplotlib  # noqa: F401
    except ImportError:
        class _Any:
            def __getattr__(self, name):
                return _Any()

            def __call__(self, *a, **k):
                return _Any()

            def __iter__(self):
                return iter((_Any(), _Any()))

        def _attr(name):
            if name.startswith("__"):
                raise AttributeError(name)
            return _Any()

        mpl = types.ModuleType("matplotlib")
        mpl.use = lambda *a, **k: None
        mpl.__getattr__ = _attr
        plt = types.ModuleType("matplotlib.pyplot")

        class _RC(dict):
            def update(self, *a, **k):
                pass

        plt.rcParams = _RC()
        plt.__getattr__ = _attr
        mpl.pyplot = plt
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = plt
    sys.path.insert(0, ref_dir)
    import becgpp  # noqa: F401
    return becgpp


def _np(t):
    return t.detach().cpu().numpy()


def _cfg(becgpp, **kw):
    base = dict(mode="single", show_inline=False, save_figs=False, save_ckpt=False)
    base.update(kw)
    return becgpp.default_cfg(**base)


# operator cases: the physics sets of the reference's audit tests plus quartic trap,
# a 3*2^k grid and a 3D case on an odd-factor grid
OPS = {
    "cq_rot": dict(dimension="2D", beta2=30, beta3=5, Omega=0.4, L=6, Ngrid=48),
    "newton2d_rot": dict(dimension="2D", beta2=30, G_C=3, kernel="newton", Omega=0.3, L=6, Ngrid=48),
    "log2d": dict(dimension="2D", beta2=30, G_C=3, kernel="log", L=6, Ngrid=48),
    "q2d": dict(dimension="quasi2D", beta2=30, G_C=3, kernel="q2d", l_z=0.5, L=6, Ngrid=48),
    "newton3d_rot": dict(dimension="3D", beta2=20, beta3=2, G_C=3, kernel="newton", Omega=0.5,
                         Ngrid=24, L=5),
    "quartic": dict(dimension="2D", s=4, trap_coeff=0.25, beta2=10, L=6, Ngrid=32),
    "harm64": dict(dimension="2D", beta2=100, L=8, Ngrid=64),
    "q2d_rot64": dict(dimension="quasi2D", beta2=50, G_C=10, kernel="q2d", l_z=0.5, Omega=0.3,
                      L=8, Ngrid=64),
}

KERNELS = {
    "newton2d": dict(dimension="2D", G_C=1.0, kernel="newton", L=4, Ngrid=16),
    "log2d": dict(dimension="2D", G_C=1.0, kernel="log", L=4, Ngrid=16),
    "q2d": dict(dimension="quasi2D", G_C=1.0, kernel="q2d", l_z=0.5, L=4, Ngrid=16),
    "q2d_small_lz": dict(dimension="quasi2D", G_C=1.0, kernel="q2d", l_z=0.1, L=4, Ngrid=16),
    "newton3d": dict(dimension="3D", G_C=1.0, kernel="newton", L=4, Ngrid=8),
}

SEEDS = {
    "gauss": dict(dimension="2D", beta2=100, L=8, Ngrid=64, seed="gaussian", seed_noise=1e-3, rng=0),
    "gauss_wind": dict(dimension="2D", beta2=100, L=8, Ngrid=64, seed="gaussian", seed_winding=2, rng=3),
    "tf_parabola": dict(dimension="2D", beta2=100, L=8, Ngrid=64, seed="tf", rng=1),
    "tf_flattop": dict(dimension="2D", beta2=-200, beta3=1e3, L=20, Ngrid=64, seed="tf", rng=2),
    "triangular": dict(dimension="2D", beta2=200, Omega=0.9, L=10, Ngrid=96, seed="triangular", rng=0),
    "gauss3d": dict(dimension="3D", beta2=10, L=5, Ngrid=24, seed="gaussian", seed_noise=1e-3, rng=0),
}

SOLVES = {
    "harm48": dict(dimension="2D", beta2=50, L=6, Ngrid=48, seed="gaussian", seed_noise=1e-3,
                   res_tol=1e-8, maxit=3000),
    "cq_rot48": dict(dimension="2D", beta2=30, beta3=5, Omega=0.4, L=6, Ngrid=48, seed="tf",
                     res_tol=1e-8, maxit=3000),
    "newton2d48": dict(dimension="2D", beta2=30, G_C=3, kernel="newton", Omega=0.3, L=6, Ngrid=48,
                       seed="gaussian", res_tol=1e-8, maxit=3000),
    "log2d48": dict(dimension="2D", beta2=30, G_C=3, kernel="log", L=6, Ngrid=48, seed="gaussian",
                    res_tol=1e-8, maxit=3000),
    "q2d48": dict(dimension="quasi2D", beta2=30, G_C=3, kernel="q2d", l_z=0.5, L=6, Ngrid=48,
                  seed="gaussian", res_tol=1e-8, maxit=3000),
    "newton3d24": dict(dimension="3D", beta2=20, beta3=2, G_C=3, kernel="newton", Omega=0.5,
                       Ngrid=24, L=5, seed="gaussian", res_tol=1e-7, maxit=2000),
    "free2d": dict(dimension="2D", beta2=0.0, L=6, Ngrid=48, res_tol=1e-7, maxit=600, seed="tf"),
    "free3d": dict(dimension="3D", beta2=0.0, L=6, Ngrid=32, res_tol=1e-7, maxit=600, seed="tf"),
    "free_soft": dict(dimension="2D", beta2=0.0, trap_coeff=0.125, L=9, Ngrid=48, res_tol=1e-7,
                      maxit=600, seed="tf"),
    "free_rot": dict(dimension="2D", beta2=0.0, Omega=0.6, L=6, Ngrid=48, res_tol=1e-7, maxit=600,
                     seed="tf"),
    "stall": dict(dimension="2D", beta2=0.0, L=6, Ngrid=48, res_tol=1e-12, energy_tol=1e-9,
                  conv_window=200, maxit=1000, seed="tf"),
    "maxit5": dict(dimension="2D", beta2=50.0, L=6, Ngrid=48, res_tol=1e-14, maxit=5, seed="tf"),
    "pr48": dict(dimension="2D", beta2=50, L=6, Ngrid=48, seed="gaussian", seed_noise=1e-3,
                 res_tol=1e-8, maxit=3000, cg_beta="pr"),
    "none48": dict(dimension="2D", beta2=50, L=6, Ngrid=48, seed="gaussian", seed_noise=1e-3,
                   res_tol=1e-8, maxit=3000, cg_beta="none"),
    "droplet64": dict(dimension="2D", beta2=-200, beta3=1e3, L=20, Ngrid=64, seed="gaussian",
                      res_tol=1e-8, maxit=3000, rng=1),
    "quartic32": dict(dimension="2D", s=4, trap_coeff=0.25, beta2=10, L=6, Ngrid=32, seed="tf",
                      res_tol=1e-8, maxit=3000),
}

OBS_KEYS = ("E", "mu", "Lz", "virial_rel", "virial", "virial_lr_term", "Ekin", "Etrap", "Econtact",
            "Ethree", "Erot", "Egrav", "rrms", "peak", "resid_rel", "resid_abs", "min_resid",
            "iters", "preconditioner_shift")


def _random_state(torch, G, seed=1):
    # the reference's audit-test state: Gaussian envelope with 30% noise
    g = torch.Generator().manual_seed(seed)
    env = torch.exp(-0.5 * G["R2"])
    sh = G["R2"].shape
    re = env * (1.0 + 0.3 * torch.randn(sh, generator=g))
    im = 0.3 * env * torch.randn(sh, generator=g)
    return (re + 1j * im).to(torch.complex128)


def small(becgpp):
    import torch
    from becgpp.interactions import _build_kernel_fft
    from becgpp.solvers import _preconditioner
    from becgpp.operators import compute_residual
    out = {}
    meta = {}
    for name, kw in OPS.items():
        c = _cfg(becgpp, **kw)
        G = becgpp.make_grid(c)
        dv = G["dx"] ** G["ndim"]
        psi = _random_state(torch, G)
        psi = psi / torch.sqrt((psi.abs() ** 2).sum() * dv)
        H = becgpp.apply_H(psi, G, c)
        comp = becgpp.energy_components(psi, G, c["beta2"], c["beta3"], c["Omega"], c["G_C"])
        ra, mu, rr = compute_residual(psi, G, c)
        obs = becgpp.observables(psi, G, c)
        mu_t = (psi.conj() * H).sum().real * dv
        grad = H - mu_t * psi
        z, sigma = _preconditioner(grad, psi, G, c, comp["phi"])
        out[f"{name}/psi"] = _np(psi)
        out[f"{name}/H"] = _np(H)
        out[f"{name}/phi"] = _np(comp["phi"])
        out[f"{name}/z"] = _np(z)
        meta[name] = dict(cfg={k: c[k] for k in kw}, sigma=float(sigma), resid=[ra, mu, rr],
                          energy={k: float(comp[k]) for k in ("E", "Ekin", "Etrap", "Econtact",
                                                              "Ethree", "Erot", "Egrav", "Lz")},
                          observables={k: float(v) for k, v in obs.items()
                                       if isinstance(v, (int, float))})
    np.savez_compressed(os.path.join(HERE, "ops.npz"), **out)
    with open(os.path.join(HERE, "ops.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)

    kern = {}
    kmeta = {}
    for name, kw in KERNELS.items():
        G = becgpp.make_grid(_cfg(becgpp, **kw))
        Kf, M = _build_kernel_fft(G, "K")
        kern[f"{name}/K"] = _np(Kf.real)
        kern[f"{name}/Kimag_max"] = np.array(float(Kf.imag.abs().max()))
        if G["kernel"] == "q2d":
            Wf, _ = _build_kernel_fft(G, "W")
            kern[f"{name}/W"] = _np(Wf.real)
        kmeta[name] = dict(cfg=kw, M=int(M))
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **kern)
    with open(os.path.join(HERE, "kernels.json"), "w") as f:
        json.dump(kmeta, f, indent=1, sort_keys=True)

    seeds = {}
    for name, kw in SEEDS.items():
        c = _cfg(becgpp, **kw)
        G = becgpp.make_grid(c)
        seeds[name] = _np(becgpp.make_seed(G, c))
    np.savez_compressed(os.path.join(HERE, "seeds.npz"), **seeds)
    with open(os.path.join(HERE, "seeds.json"), "w") as f:
        json.dump(SEEDS, f, indent=1, sort_keys=True)

    sol = {}
    smeta = {}
    for name, kw in SOLVES.items():
        c = _cfg(becgpp, record_trace=True, **kw)
        G = becgpp.make_grid(c)
        psi0 = becgpp.make_seed(G, c)
        t = time.time()
        psi, G, obs = becgpp.ground_state(c, G=G, psi0=psi0.clone(), verbose=False)
        wall = time.time() - t
        sol[f"{name}/psi0"] = _np(psi0)
        sol[f"{name}/psi"] = _np(psi)
        sol[f"{name}/trace_E"] = np.array([r[2] for r in obs["trace"]])
        sol[f"{name}/trace_res"] = np.array([r[3] for r in obs["trace"]])
        smeta[name] = dict(cfg=kw, obs={k: (float(obs[k]) if k != "iters" else int(obs[k]))
                                        for k in OBS_KEYS},
                           stop_reason=obs["stop_reason"], converged=bool(obs["converged"]),
                           wall_s=wall)
        print(name, smeta[name]["obs"]["E"], obs["stop_reason"], obs["iters"], f"{wall:.1f}s",
              flush=True)
    np.savez_compressed(os.path.join(HERE, "solves.npz"), **sol)
    with open(os.path.join(HERE, "solves.json"), "w") as f:
        json.dump(smeta, f, indent=1, sort_keys=True)


# gradient cases: the physics of the operator cases (a scaled-down quasi-2D rotating
# pancake first: q2d l_z=0.5, Omega=0.3, beta2=50, G_C=10)
GRADS = ("q2d_rot64", "newton3d_rot", "cq_rot", "log2d", "newton2d_rot", "q2d")
# ground state whose energy is differentiated by central differences of solves
HF_CASE = dict(dimension="quasi2D", beta2=50, G_C=10, kernel="q2d", l_z=0.5, Omega=0.3, L=6,
               Ngrid=48, seed="gaussian", res_tol=1e-10, maxit=6000)
HF_STEPS = dict(beta2=1e-3, G_C=1e-3, Omega=1e-4, l_z=1e-4)


def grads(becgpp):
    """Autograd through the reference's FP64 energy functional (psi, beta2, beta3,
    G_C, Omega) and central differences for l_z (the reference's kernel table is
    not differentiable in l_z); ground-state energies at shifted parameters."""
    import torch
    from becgpp.interactions import clear_kernel_cache
    out, meta = {}, {}
    for name in GRADS:
        kw = OPS[name]
        c = _cfg(becgpp, **kw)
        G = becgpp.make_grid(c)
        psi = _random_state(torch, G)
        dv = G["dx"] ** G["ndim"]
        psi = (psi / torch.sqrt((psi.abs() ** 2).sum() * dv)).detach().requires_grad_(True)
        pars = {k: torch.tensor(float(c[k]), dtype=torch.float64, requires_grad=True)
                for k in ("beta2", "beta3", "G_C", "Omega")}
        E = becgpp.energy_components(psi, G, pars["beta2"], pars["beta3"], pars["Omega"],
                                     pars["G_C"])["E"]
        E.backward()
        out[f"{name}/psi"] = _np(psi)
        out[f"{name}/dpsi"] = _np(psi.grad)
        m = dict(cfg=kw, E=float(E), dparams={k: float(v.grad) if v.grad is not None else 0.0
                                              for k, v in pars.items()})
        if G["kernel"] == "q2d":
            h = 1e-6
            Es = []
            for lz in (kw["l_z"] + h, kw["l_z"] - h):
                clear_kernel_cache()
                cl = _cfg(becgpp, **dict(kw, l_z=lz))
                Gl = becgpp.make_grid(cl)
                Es.append(float(becgpp.energy_components(psi.detach(), Gl, c["beta2"], c["beta3"],
                                                         c["Omega"], c["G_C"])["E"]))
            clear_kernel_cache()
            m["dparams"]["l_z"] = (Es[0] - Es[1]) / (2 * h)
            m["l_z_fd_step"] = h
        meta[name] = m
        print(name, m["E"], m["dparams"], flush=True)
    # Hellmann-Feynman: ground-state energy at shifted parameters
    c = _cfg(becgpp, **HF_CASE)
    G = becgpp.make_grid(c)
    psi0 = becgpp.make_seed(G, c)
    psi, _, obs = becgpp.ground_state(c, G=G, psi0=psi0.clone(), verbose=False)
    out["hf/psi0"] = _np(psi0)
    out["hf/psi"] = _np(psi)
    hf = dict(cfg=HF_CASE, E=float(obs["E"]), resid_rel=float(obs["resid_rel"]), fd={})
    for k, h in HF_STEPS.items():
        Es = []
        for sgn in (1, -1):
            clear_kernel_cache()
            cs = _cfg(becgpp, **dict(HF_CASE, **{k: HF_CASE[k] + sgn * h}))
            Gs = becgpp.make_grid(cs)
            _, _, o = becgpp.ground_state(cs, G=Gs, psi0=psi.clone(), verbose=False)
            Es.append(float(o["E"]))
        hf["fd"][k] = dict(h=h, dE=(Es[0] - Es[1]) / (2 * h), E_plus=Es[0], E_minus=Es[1])
        print("hf", k, hf["fd"][k], flush=True)
    clear_kernel_cache()
    meta["hf"] = hf
    np.savez_compressed(os.path.join(HERE, "grads.npz"), **out)
    with open(os.path.join(HERE, "grads.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


def big(becgpp, only=None):
    """The benchmark configurations, run through the reference's CPU path."""
    import torch
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from becgpp_b200.workloads import baseline_instances
    path = os.path.join(HERE, "baseline_runs.json")
    done = json.load(open(path)) if os.path.isfile(path) else {}
    for inst in baseline_instances():
        name = inst["name"]
        if name in done or (only and not name.startswith(only)):
            continue
        c = _cfg(becgpp, **inst["cfg"])
        G = becgpp.make_grid(c)
        psi0 = becgpp.make_seed(G, c)
        if inst.get("phase_noise", 0.0):
            g = torch.Generator().manual_seed(inst["phase_seed"])
            psi0 = psi0 * torch.exp(1j * inst["phase_noise"] * torch.randn(psi0.shape, generator=g,
                                                                           dtype=torch.float64))
        t = time.time()
        psi, G, obs = becgpp.ground_state(c, G=G, psi0=psi0.clone(), verbose=False)
        wall = time.time() - t
        done[name] = dict(cfg=inst["cfg"], obs={k: (float(obs[k]) if k != "iters" else int(obs[k]))
                                                for k in OBS_KEYS},
                          stop_reason=obs["stop_reason"], converged=bool(obs["converged"]),
                          wall_s=wall, threads=torch.get_num_threads())
        print(name, done[name]["obs"]["E"], obs["stop_reason"], obs["iters"], f"{wall:.1f}s",
              flush=True)
        with open(path, "w") as f:
            json.dump(done, f, indent=1, sort_keys=True)


# operator cases at the sizes the benchmark configurations run at (c1 128^2, c2
# 384^2 rotating, c4 droplets at 128^2 and 256^2, c5 quasi-2D 256^2, c3 128^3 with
# the 256^3 padded newton transform). The state is _random_state of the grid, which
# the GPU test regenerates from the same CPU generator, so only samples and
# checksums of the outputs are stored: the values at BIG_SAMPLES random points, the
# max-norm and 2-norm of each field, and its projections on BIG_PROJ seeded random
# complex weight vectors (any error anywhere in a field moves a projection).
BIG_OPS = {
    "c1_128": dict(dimension="2D", beta2=100, L=16, Ngrid=128),
    "c2_384_rot": dict(dimension="2D", beta2=200, Omega=0.9, L=12, Ngrid=384),
    "c4_128_droplet": dict(dimension="2D", beta2=-200, beta3=1000, L=20, Ngrid=128),
    "c4_256_droplet": dict(dimension="2D", beta2=-200, beta3=1000, L=20, Ngrid=256),
    "c5_256_q2d": dict(dimension="quasi2D", beta2=50, G_C=10, kernel="q2d", l_z=0.5, Omega=0.3,
                       L=16, Ngrid=256),
    "c3_128_newton": dict(dimension="3D", beta2=10, G_C=20, kernel="newton", L=16, Ngrid=128),
}
BIG_SAMPLES = 8192
BIG_PROJ = 3


def big_weights(n, case_index):
    """Sample indices and projection weights of a big-operator case (shared with
    the GPU test): numpy's seeded generator, so both sides draw the same."""
    rng = np.random.default_rng(1000 + case_index)
    idx = np.sort(rng.choice(n, size=min(BIG_SAMPLES, n), replace=False))
    w = rng.standard_normal((BIG_PROJ, n)) + 1j * rng.standard_normal((BIG_PROJ, n))
    return idx, w


def field_summary(x, idx, w):
    """Samples, max-norm, 2-norm and projections of a field (flattened)."""
    f = np.asarray(x).reshape(-1)
    return dict(samples=f[idx], maxabs=float(np.abs(f).max()), norm2=float(np.sqrt((np.abs(f) ** 2).sum())),
                proj=w @ f.astype(np.complex128))


def bigops(becgpp):
    import torch
    from becgpp.solvers import _preconditioner
    from becgpp.operators import compute_residual
    arr, meta = {}, {}
    for ci, (name, kw) in enumerate(BIG_OPS.items()):
        t = time.time()
        c = _cfg(becgpp, **kw)
        G = becgpp.make_grid(c)
        dv = G["dx"] ** G["ndim"]
        psi = _random_state(torch, G)
        psi = psi / torch.sqrt((psi.abs() ** 2).sum() * dv)
        H = becgpp.apply_H(psi, G, c)
        comp = becgpp.energy_components(psi, G, c["beta2"], c["beta3"], c["Omega"], c["G_C"])
        ra, mu, rr = compute_residual(psi, G, c)
        mu_t = (psi.conj() * H).sum().real * dv
        z, sigma = _preconditioner(H - mu_t * psi, psi, G, c, comp["phi"])
        n = psi.numel()
        idx, w = big_weights(n, ci)
        arr[f"{name}/idx"] = idx
        m = dict(cfg=kw, n=n, case_index=ci, sigma=float(sigma), resid=[ra, float(mu), rr],
                 energy={k: float(comp[k]) for k in ("E", "Ekin", "Etrap", "Econtact", "Ethree", "Erot",
                                                     "Egrav", "Lz")})
        for fname, fld in (("psi", psi), ("H", H), ("phi", comp["phi"]), ("z", z)):
            sm = field_summary(_np(fld), idx, w)
            arr[f"{name}/{fname}/samples"] = sm.pop("samples")
            arr[f"{name}/{fname}/proj"] = sm.pop("proj")
            m[fname] = sm
        meta[name] = m
        print(name, f"{time.time() - t:.1f}s", m["energy"]["E"], flush=True)
    np.savez_compressed(os.path.join(HERE, "bigops.npz"), **arr)
    with open(os.path.join(HERE, "bigops.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


# Thomas-Fermi references (becgpp/thomasfermi.py:65-156): the nonlocal fixed point
# (quasi-2D pancake of the benchmark's c5 configuration, a 3D newton case), the local
# inverted profile (the rotating c2 configuration) and the droplet flat top
TF_CASES = {
    "tf_q2d256": dict(dimension="quasi2D", beta2=50, G_C=10, kernel="q2d", l_z=0.5, Omega=0.3, L=16,
                      Ngrid=256),
    "tf_newton3d48": dict(dimension="3D", beta2=10, G_C=20, kernel="newton", L=8, Ngrid=48),
    "tf_local384": dict(dimension="2D", beta2=200, Omega=0.9, L=12, Ngrid=384),
    "tf_flattop256": dict(dimension="2D", beta2=-200, beta3=1000, L=20, Ngrid=256),
}


def tf(becgpp):
    import torch
    from becgpp.thomasfermi import extract_tf
    arr, meta = {}, {}
    for ci, (name, kw) in enumerate(TF_CASES.items()):
        t = time.time()
        c = _cfg(becgpp, **kw)
        G = becgpp.make_grid(c)
        r = extract_tf(c, G)
        n = r["n"].numel()
        idx, w = big_weights(n, 100 + ci)
        sm = field_summary(_np(r["n"]), idx, w)
        arr[f"{name}/idx"] = idx
        arr[f"{name}/n/samples"] = sm.pop("samples")
        arr[f"{name}/n/proj"] = sm.pop("proj")
        meta[name] = dict(cfg=kw, n=n, case_index=100 + ci, kind=r["kind"], mu=float(r["mu"]),
                          R90=float(r["R90"]), R99=float(r["R99"]), converged=bool(r["converged"]),
                          final_dn=float(r["final_dn"]), field=sm, wall_s=time.time() - t)
        print(name, meta[name]["kind"], meta[name]["mu"], f"{meta[name]['wall_s']:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "tf.npz"), **arr)
    with open(os.path.join(HERE, "tf.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


def stopstats(becgpp, n=40):
    """The reference's own stop reasons over n seeded variants of the 2D harmonic
    configuration c1 (rng 0..n-1): near res_tol the choice between 'converged'
    and 'line_search_stalled' is decided by round-off, so the distribution is
    the thing to compare, not one seed's outcome."""
    import torch
    torch.set_num_threads(1)   # small grids: one thread is faster than many
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from becgpp_b200.workloads import c1
    rows = []
    for rng in range(n):
        c = _cfg(becgpp, **dict(c1()[0]["cfg"], rng=rng))
        G = becgpp.make_grid(c)
        _, _, obs = becgpp.ground_state(c, G=G, psi0=becgpp.make_seed(G, c), verbose=False)
        rows.append(dict(rng=rng, E=float(obs["E"]), resid_rel=float(obs["resid_rel"]),
                         stop_reason=obs["stop_reason"], iters=int(obs["iters"])))
        print(rows[-1], flush=True)
    with open(os.path.join(HERE, "stop_stats.json"), "w") as f:
        json.dump({"workload": "c1", "rows": rows}, f, indent=1)


# diagnostics: synthetic vortex states (their count and LLL weight are known by
# construction), reference diagnostics() of solved states, and the reference's
# run() for one single-mode and one sweep-mode configuration
DIAG_SOLVES = ("cq_rot48", "free_rot", "newton2d48")
DIAG_RUNS = {
    "single_rot": dict(mode="single", dimension="2D", beta2=30, beta3=5, Omega=0.4, L=6, Ngrid=48,
                       seed="gaussian", nseeds=2),
    "sweep_b2": dict(mode="sweep", dimension="2D", beta3=5, Omega=0.3, L=6, Ngrid=48, seed="tf",
                     sweep_param="beta2", sweep_values=[20.0, 30.0, 40.0], sweep_continuation=True),
    "sweep_fresh": dict(mode="sweep", dimension="2D", beta2=-200, beta3=1000, L=8, Ngrid=64,
                        seed="gaussian", sweep_param="rng", sweep_values=[0, 1, 2, 3],
                        sweep_continuation=False, res_tol=1e-9),
}
VORTICES = ((1.0, 0.5, 1), (-1.2, 0.3, 1), (0.2, -1.1, 1), (0.9, -0.9, -1))


def _vortex_state(torch, G, vortices):
    z = torch.complex(G["X"], G["Y"])
    psi = torch.exp(-0.5 * G["R2"]).to(torch.complex128)
    for x, y, q in vortices:
        zk = complex(x, y)
        psi = psi * ((z - zk) if q > 0 else (z - zk).conj())
    return psi


def diag(becgpp):
    import torch
    from becgpp.vortex import lll_weight, vortex_diagnostic
    arr, meta = {}, {}
    # synthetic states: 2D with 3 + 1 vortices, the same extended along z, a pure LLL state
    c2 = _cfg(becgpp, dimension="2D", L=6, Ngrid=64, Omega=0.8)
    G2 = becgpp.make_grid(c2)
    c3 = _cfg(becgpp, dimension="3D", L=6, Ngrid=32, Omega=0.8)
    G3 = becgpp.make_grid(c3)
    states = {
        "mixed2d": (c2, G2, _vortex_state(torch, G2, VORTICES)),
        "lll2d": (c2, G2, _vortex_state(torch, G2, [v for v in VORTICES if v[2] > 0])),
        "mixed3d": (c3, G3, _vortex_state(torch, G3, VORTICES)),
    }
    for name, (c, G, psi) in states.items():
        arr[f"{name}/psi"] = _np(psi)
        meta[name] = dict(cfg=dict(dimension=c["dimension"], L=c["L"], Ngrid=c["Ngrid"], Omega=c["Omega"]),
                          vortex={k: int(v) for k, v in vortex_diagnostic(psi, G, c["Omega"]).items()},
                          w_LLL=float(lll_weight(psi, G, 60, c["Omega"])))
    # diagnostics of the reference's solved states (solves.npz)
    sol, smeta = np.load(os.path.join(HERE, "solves.npz")), json.load(open(os.path.join(HERE, "solves.json")))
    for name in DIAG_SOLVES:
        c = _cfg(becgpp, **smeta[name]["cfg"])
        G = becgpp.make_grid(c)
        psi = torch.as_tensor(sol[f"{name}/psi"])
        d = becgpp.diagnostics(psi, G, c)
        meta[f"diag/{name}"] = dict(cfg=smeta[name]["cfg"], diag={k: (v if isinstance(v, (bool, str)) else float(v))
                                                                   for k, v in d.items()
                                                                   if isinstance(v, (bool, str, int, float))})
    # sweep helpers: box sizing and bi/trilinear resampling between grids
    from becgpp.grid import auto_grid, resample_state
    for name, kw in (("droplet2d", dict(dimension="2D", beta2=-200, beta3=1000)),
                     ("droplet3d", dict(dimension="3D", beta2=-200, beta3=1000)),
                     ("longrange", dict(dimension="2D", beta2=40, G_C=5, kernel="newton")),
                     ("plain", dict(dimension="2D", beta2=30))):
        L, N, R = auto_grid(_cfg(becgpp, **kw))
        meta[f"autogrid/{name}"] = dict(cfg=kw, L=L, N=N, R=R)
    for name, (ca, cb) in (("2d", (dict(dimension="2D", L=6, Ngrid=48), dict(dimension="2D", L=7, Ngrid=64))),
                           ("3d", (dict(dimension="3D", L=5, Ngrid=24), dict(dimension="3D", L=6, Ngrid=32)))):
        Ga, Gb = becgpp.make_grid(_cfg(becgpp, **ca)), becgpp.make_grid(_cfg(becgpp, **cb))
        psi = _vortex_state(torch, Ga, VORTICES[:2])
        arr[f"resample/{name}/psi"] = _np(psi)
        arr[f"resample/{name}/out"] = _np(resample_state(psi, Ga, Gb))
        meta[f"resample/{name}"] = dict(a=ca, b=cb)
    # run(): single (two seeds) and two sweeps
    for name, kw in DIAG_RUNS.items():
        c = _cfg(becgpp, **kw)
        out = becgpp.run(c)
        rows = out if isinstance(out, list) else [out]
        keep = ("E", "mu", "Lz", "iters", "stop_reason", "converged", "Nv", "R90", "branch", "seed_used",
                "resid_rel", "w_LLL", "virial_rel")
        meta[f"run/{name}"] = dict(cfg=kw, rows=[{k: (r[k] if isinstance(r[k], (bool, str)) else float(r[k]))
                                                  for k in keep if k in r} for r in rows])
        print(name, [r.get("E") for r in rows], flush=True)
    np.savez_compressed(os.path.join(HERE, "diag.npz"), **arr)
    with open(os.path.join(HERE, "diag.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args:
        sys.exit("usage: make_golden.py REF_DIR [--big [--only=NAME] | --grads | --diag | --stopstats | --bigops | --tf]")
    ref = args[0]
    becgpp = _import_reference(ref)
    if "--grads" in sys.argv:
        grads(becgpp)
    elif "--stopstats" in sys.argv:
        stopstats(becgpp)
    elif "--bigops" in sys.argv:
        bigops(becgpp)
    elif "--tf" in sys.argv:
        tf(becgpp)
    elif "--diag" in sys.argv:
        diag(becgpp)
    elif "--big" in sys.argv:
        only = next((a.split("=", 1)[1] for a in sys.argv if a.startswith("--only=")), None)
        big(becgpp, only)
    else:
        small(becgpp)
