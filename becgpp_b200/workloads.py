"""Named workloads: the five reference configurations the solver is measured on.

Each instance is a plain config dict (keys of ``CFG_DEFAULTS``) plus, where the
workload asks for it, a seeded phase-noise factor multiplied into the seed on
the host: ``psi0 *= exp(i * phase_noise * N(0,1))`` drawn from a CPU
``torch.Generator`` seeded with ``phase_seed``.

* ``c1``  2D harmonic trap, beta2=100, N=128, L=16, Gaussian seed (noise 1e-3).
* ``c2``  2D rotating condensate Omega=0.9, beta2=200, N=384, L=12; three seeds
  (triangular, tf, gaussian; rng 0,1,2) with 1e-3 phase noise.
* ``c3``  3D self-gravitating condensate, beta2=10, G_C=20 (1/r), N=128 padded to
  256, L=16, Gaussian seed.
* ``c4``  cubic-quintic droplet sweep: beta2 in linspace(-400,-50,16), beta3=1e3,
  L=20, 4 seeds each (tf, gaussian, tf, gaussian; rng 0..3); even sweep index on
  a 128^2 grid, odd on 256^2: 64 instances in one batch.
* ``c5``  quasi-2D pancake, q2d kernel l_z=0.5, Omega=0.3, beta2=50, G_C=10,
  N=256, L=16, Gaussian seed.
"""
import numpy as np

_COMMON = dict(mode="single", show_inline=False, save_figs=False, save_ckpt=False)


def c1():
    return [dict(name="c1", cfg=dict(_COMMON, dimension="2D", s=2, Omega=0.0, beta2=100.0, beta3=0.0,
                                     G_C=0.0, kernel="none", Ngrid=128, L=16.0, seed="gaussian",
                                     seed_noise=1e-3, rng=0, res_tol=1e-8))]


def c2():
    kinds = ("triangular", "tf", "gaussian")
    return [dict(name=f"c2_s{j}", phase_noise=1e-3, phase_seed=j,
                 cfg=dict(_COMMON, dimension="2D", s=2, Omega=0.9, beta2=200.0, beta3=0.0, G_C=0.0,
                          kernel="none", Ngrid=384, L=12.0, seed=kinds[j], seed_noise=1e-3, rng=j,
                          res_tol=1e-8, maxit=20000))
            for j in range(3)]


def c3():
    return [dict(name="c3", cfg=dict(_COMMON, dimension="3D", s=2, Omega=0.0, beta2=10.0, beta3=0.0,
                                     G_C=20.0, kernel="newton", Ngrid=128, L=16.0, pad=2,
                                     seed="gaussian", seed_noise=1e-3, rng=0, res_tol=1e-8,
                                     maxit=3000))]


def c4():
    out = []
    for b, b2 in enumerate(np.linspace(-400.0, -50.0, 16)):
        for j in range(4):
            out.append(dict(name=f"c4_b{b:02d}_s{j}",
                            cfg=dict(_COMMON, dimension="2D", s=2, Omega=0.0, beta2=float(b2),
                                     beta3=1e3, G_C=0.0, kernel="none",
                                     Ngrid=(128 if b % 2 == 0 else 256), L=20.0,
                                     seed=("tf", "gaussian")[j % 2], rng=j, res_tol=1e-8,
                                     maxit=20000)))
    return out


def c5():
    return [dict(name="c5", cfg=dict(_COMMON, dimension="quasi2D", s=2, Omega=0.3, beta2=50.0,
                                     beta3=0.0, G_C=10.0, kernel="q2d", l_z=0.5, Ngrid=256, L=16.0,
                                     seed="gaussian", rng=0, res_tol=1e-8, maxit=20000))]


WORKLOADS = dict(c1=c1, c2=c2, c3=c3, c4=c4, c5=c5)


def baseline_instances(order=("c4", "c1", "c5", "c3", "c2")):
    out = []
    for w in order:
        out.extend(WORKLOADS[w]())
    return out
