"""Thomas-Fermi reference density (seeds and diagnostics).

Definitions of becgpp/thomasfermi.py:21-156: nonlocal compressed TF by a
relaxed fixed point (G_C != 0), zero-pressure flat top (b2 < 0 < b3), inverted
profile (repulsive, trapped), or None. The local cases run on a CPU copy of the
grid (so seeds built on them equal the reference's CPU seeds); the nonlocal
fixed point runs on the device, its potential from the library's zero-padded
convolution.
"""
import math

import torch

from .fields import mass_quantiles

_TF_CACHE = {}
_GRID_CACHE = {}


def cpu_grid(G):
    """CPU FP64 coordinates of grid G, built with the operations of make_grid."""
    key = (G["ndim"], G["N"], float(G["L"]), float(G["s"]), float(G.get("trap_coeff", 0.5)))
    if key in _GRID_CACHE:
        return _GRID_CACHE[key]
    N, L, s, ndim = int(G["N"]), float(G["L"]), float(G["s"]), int(G["ndim"])
    dx = 2.0 * L / N
    x = (torch.arange(N, dtype=torch.float64) - N // 2) * dx
    if ndim == 2:
        X, Y = torch.meshgrid(x, x, indexing="ij")
        coords = (X, Y)
        R2 = X ** 2 + Y ** 2
    else:
        X, Y, Z = torch.meshgrid(x, x, x, indexing="ij")
        coords = (X, Y, Z)
        R2 = X ** 2 + Y ** 2 + Z ** 2
    tc = float(G.get("trap_coeff", 0.5))
    V = tc * R2 ** (s / 2.0) if s > 0 else torch.zeros_like(R2)
    Gc = dict(G)
    Gc.update(coords=coords, X=X, Y=Y, R2=R2, V=V, dx=dx)
    if len(_GRID_CACHE) > 8:
        _GRID_CACHE.clear()
    _GRID_CACHE[key] = Gc
    return Gc


def tf_effective_potential(Gc, cfg):
    """V - Omega^2 (x^2 + y^2) / 2: the centrifugal term acts in the plane only."""
    O = float(cfg.get("Omega", 1.0))
    return Gc["V"] - 0.5 * O * O * (Gc["X"] ** 2 + Gc["Y"] ** 2)


def _invert_local(mu, Veff, b2, b3):
    """Upper physical root rho >= 0 of b3 rho^2 + b2 rho = mu - Veff (zero where
    no real root exists)."""
    rhs = mu - Veff
    if b3 > 1e-30:
        disc = b2 * b2 + 4.0 * b3 * rhs
        root = (-b2 + torch.sqrt(torch.clamp(disc, min=0.0))) / (2.0 * b3)
        return torch.where(disc > 0.0, torch.clamp(root, min=0.0), torch.zeros_like(rhs))
    if abs(b2) > 1e-30:
        return torch.clamp(rhs / b2, min=0.0)
    return torch.zeros_like(rhs)


def _bisect_mu_for_norm(f_rho, dv, lo, hi, steps=90):
    guard = 0
    while (f_rho(hi).sum() * dv).item() < 1.0:
        hi = lo + 2.0 * (hi - lo) + 1e-9
        guard += 1
        if guard > 200:
            return float("nan")
    for _ in range(steps):
        mid = 0.5 * (lo + hi)
        if (f_rho(mid).sum() * dv).item() < 1.0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def extract_tf(cfg, G, iters=400, relax=0.4):
    """Thomas-Fermi reference for the current parameters: dict with the density n
    (CPU tensor), R90, R99, mu, kind, or None."""
    from .interactions import long_range_phi
    b2, b3, gc = float(cfg["beta2"]), float(cfg["beta3"]), float(cfg["G_C"])
    Gc = cpu_grid(G)
    dv = Gc["dx"] ** Gc["ndim"]
    Veff = tf_effective_potential(Gc, cfg)
    nonlocal_on = G["kernel"] != "none" and abs(gc) > 1e-15
    key = ("tf", G["kernel"], round(b2, 10), round(b3, 10), round(gc, 10),
           round(float(cfg["Omega"]), 10), int(G["N"]), round(float(G["L"]), 10), int(G["ndim"]),
           round(float(G["s"]), 10), round(float(G.get("trap_coeff", 0.5)), 10),
           round(float(G.get("l_z", 0.0)), 10), int(G["pad"]))
    if cfg.get("tf_cache", True) and key in _TF_CACHE:
        return _TF_CACHE[key]
    tf = None
    if nonlocal_on and b2 <= 0 and b3 <= 0:
        tf = None
    elif nonlocal_on:
        # the fixed point runs where the grid's tensors live (the device on a GPU
        # box): each iteration is one zero-padded convolution and a 90-step
        # bisection over the whole grid
        dev = G["X"].device
        sigma = 0.15 * float(G["L"])
        n = torch.exp(-Gc["R2"].to(dev) / (2 * sigma ** 2))
        n = n / (n.sum() * dv)
        Veff = Veff.to(dev)
        conv, dn, mu = False, float("inf"), float("nan")
        for _ in range(int(iters)):
            phi = long_range_phi(n, G, gc)
            base = Veff + phi
            f = lambda m: _invert_local(m, base, b2, b3)
            mu = _bisect_mu_for_norm(f, dv, base.min().item(), base.max().item() + abs(b2) + abs(b3) + 1.0)
            if not math.isfinite(mu):
                break
            n_new = f(mu)
            ssum = (n_new.sum() * dv).item()
            if ssum <= 0:
                break
            n_new = n_new / ssum
            dn = (n_new - n).abs().sum().item() * dv
            n = (1 - relax) * n + relax * n_new
            n = n / (n.sum() * dv)
            if dn < 1e-9:
                conv = True
                break
        if math.isfinite(mu):
            n = n.cpu()
            R90, R99 = mass_quantiles(n, Gc, (0.90, 0.99))
            tf = dict(kind="nonlocal_compressed", n=n, R90=R90, R99=R99, mu=mu, rho0=float("nan"),
                      converged=conv, final_dn=dn)
    else:
        confined = bool(torch.max(Veff).item() > 1e-12)
        if b2 < 0 and b3 > 0:
            rho0 = -3.0 * b2 / (4.0 * b3)
            mu = b2 * rho0 + b3 * rho0 ** 2
            R = 1.0 / math.sqrt(math.pi * rho0) if G["ndim"] == 2 else (3.0 / (4.0 * math.pi * rho0)) ** (1.0 / 3.0)
            rr = torch.sqrt(Gc["R2"])
            n = torch.where(rr <= R, torch.full_like(rr, rho0), torch.zeros_like(rr))
            n = n / (n.sum() * dv)
            R90, R99 = mass_quantiles(n, Gc, (0.90, 0.99))
            tf = dict(kind="local_flattop", n=n, R90=R90, R99=R99, mu=mu, rho0=rho0, R=R,
                      converged=True, final_dn=0.0)
        elif confined and (b2 > 0 or (b2 == 0 and b3 > 0)):
            f = lambda m: _invert_local(m, Veff, b2, b3)
            mu = _bisect_mu_for_norm(f, dv, Veff.min().item(), Veff.max().item() + abs(b2) + abs(b3) + 1.0)
            n = f(mu)
            n = n / (n.sum() * dv)
            R90, R99 = mass_quantiles(n, Gc, (0.90, 0.99))
            kind = "repulsive_parabola" if b3 <= 0 else "local_trapped_repulsive"
            tf = dict(kind=kind, n=n, R90=R90, R99=R99, mu=mu, rho0=float("nan"), converged=True,
                      final_dn=0.0)
    if tf is not None and cfg.get("tf_cache", True):
        _TF_CACHE[key] = tf
    return tf
