"""Thomas-Fermi reference densities, computed on the device.

Which reference applies follows becgpp/thomasfermi.py:83-152:

=============================  =========================================  ==========================
kind                           when                                       density
=============================  =========================================  ==========================
``nonlocal_compressed``        long-range kernel on (G_C != 0) and not    relaxed fixed point of
                               both b2 <= 0 and b3 <= 0                   mu = V_eff + b2 n + b3 n^2
                                                                          + phi[n], unit mass
``local_flattop``              local, b2 < 0 < b3 (self-bound droplet)    rho0 = -3 b2 / (4 b3) inside
                                                                          the radius of unit mass
``repulsive_parabola`` /       local, confined (max V_eff > 1e-12) and    inverted profile, mu by
``local_trapped_repulsive``    b2 > 0 (or b2 = 0 < b3)                    bisection on unit mass
None                           anything else
=============================  =========================================  ==========================

with V_eff = V - Omega^2 (x^2 + y^2) / 2. The fixed point and the inverted
profile run in libbgp (``bgp_tf_density``): every chemical-potential
bisection step is a full-grid sum on the device and the long-range potential
is the plan's zero-padded convolution, so a step costs one convolution and one
cooperative launch, with no host round trip per halving. The flat top is
closed-form. Radii R90, R99 are the device mass quantiles (``fields``).

Seeds need the reference's local densities element for element and build
them on the host themselves (``seeds.host_tf_density``).
"""
import ctypes
import math

import torch

from . import _lib
from .fields import mass_quantiles

_TF_CACHE = {}


def effective_potential_max(G, cfg):
    """max over the grid of V_eff = tc r^s - Omega^2 (x^2 + y^2) / 2 (decides
    whether a local repulsive gas is confined)."""
    Om = float(cfg.get("Omega", 1.0))
    R2 = G["R2"]
    s, tc = float(G["s"]), float(G.get("trap_coeff", 0.5))
    V = tc * R2 ** (s / 2.0) if s > 0 else torch.zeros_like(R2)
    return float((V - 0.5 * Om * Om * (G["X"] ** 2 + G["Y"] ** 2)).max())


def reference_kind(cfg, G):
    """The Thomas-Fermi reference that applies to these parameters, or None."""
    b2, b3, gc = float(cfg["beta2"]), float(cfg["beta3"]), float(cfg["G_C"])
    if G["kernel"] != "none" and abs(gc) > 1e-15:
        return None if (b2 <= 0 and b3 <= 0) else "nonlocal_compressed"
    if b2 < 0 < b3:
        return "local_flattop"
    if (b2 > 0 or (b2 == 0 and b3 > 0)) and effective_potential_max(G, cfg) > 1e-12:
        return "repulsive_parabola" if b3 <= 0 else "local_trapped_repulsive"
    return None


def _key(cfg, G):
    r = lambda v: round(float(v), 10)
    return ("tf", G["kernel"], r(cfg["beta2"]), r(cfg["beta3"]), r(cfg["G_C"]), r(cfg["Omega"]), int(G["N"]),
            r(G["L"]), int(G["ndim"]), r(G["s"]), r(G.get("trap_coeff", 0.5)), r(G.get("l_z", 0.0)), int(G["pad"]))


def _flattop(cfg, G):
    """Zero-pressure droplet: density rho0 = -3 b2 / (4 b3) on the ball of unit
    mass, R = (pi rho0)^-1/2 (2D) or (3 / (4 pi rho0))^1/3 (3D); the discrete
    density is renormalised to unit mass on the grid."""
    b2, b3 = float(cfg["beta2"]), float(cfg["beta3"])
    rho0 = -3.0 * b2 / (4.0 * b3)
    R = 1.0 / math.sqrt(math.pi * rho0) if G["ndim"] == 2 else (3.0 / (4.0 * math.pi * rho0)) ** (1.0 / 3.0)
    n = torch.where(torch.sqrt(G["R2"]) <= R, torch.full_like(G["R2"], rho0), torch.zeros_like(G["R2"]))
    n = n / (n.sum() * G["dx"] ** G["ndim"])
    return dict(n=n, mu=b2 * rho0 + b3 * rho0 * rho0, rho0=rho0, R=R, converged=True, final_dn=0.0)


def _device_density(cfg, G, nonlocal_, iters, relax):
    from .grid import plan_for
    plan = plan_for(G, cfg)
    n = torch.empty(tuple(G["R2"].shape), dtype=torch.float64, device="cuda")
    info = (ctypes.c_double * 5)()
    _lib.check(_lib.lib().bgp_tf_density(plan.handle, 0, 1 if nonlocal_ else 0, float(cfg.get("Omega", 1.0)),
                                         int(iters), float(relax), _lib.ptr(n), info, _lib.stream_ptr()),
               "bgp_tf_density")
    mu = info[0]
    if not math.isfinite(mu):
        return None
    return dict(n=n, mu=mu, rho0=float("nan"), converged=bool(info[1]), final_dn=info[2], steps=int(info[3]))


def extract_tf(cfg, G, iters=400, relax=0.4):
    """Thomas-Fermi reference for the current parameters (becgpp/thomasfermi.py:65-156):
    dict(kind, n, R90, R99, mu, rho0, converged, final_dn[, R]) or None."""
    _lib.require_cuda()
    key = _key(cfg, G)
    use_cache = cfg.get("tf_cache", True)
    if use_cache and key in _TF_CACHE:
        return _TF_CACHE[key]
    kind = reference_kind(cfg, G)
    if kind is None:
        return None
    if kind == "local_flattop":
        tf = _flattop(cfg, G)
    else:
        tf = _device_density(cfg, G, kind == "nonlocal_compressed", iters, relax)
        if tf is None:
            return None
    R90, R99 = mass_quantiles(tf["n"], G, (0.90, 0.99))
    tf.update(kind=kind, R90=R90, R99=R99)
    if use_cache:
        _TF_CACHE[key] = tf
    return tf


def clear_tf_cache():
    _TF_CACHE.clear()
