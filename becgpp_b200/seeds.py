"""Initial states, generated on the host (CPU, FP64) and moved to the device.

Gaussian, Thomas-Fermi and triangular vortex-lattice seeds with the
definitions of becgpp/seeds.py:11-103. They are drawn from torch's CPU
generator (``torch.manual_seed(rng)``) on a CPU copy of the grid built with the
same operations as ``make_grid``, so a seed equals the reference's CPU seed
for the same configuration element for element. Seed generation is one-time
input preparation, not part of the solve.
"""
import math

import numpy as np
import torch

from .thomasfermi import extract_tf, reference_kind

_GRID_CACHE = {}


def cpu_grid(G):
    """CPU FP64 coordinates (X, Y[, Z]), R2 and trap V of grid G, formed with
    the tensor operations of becgpp/grid.py:74-91 so seeds drawn on it equal the
    reference's element for element."""
    key = (G["ndim"], G["N"], float(G["L"]), float(G["s"]), float(G.get("trap_coeff", 0.5)))
    if key in _GRID_CACHE:
        return _GRID_CACHE[key]
    N, L, s, ndim = int(G["N"]), float(G["L"]), float(G["s"]), int(G["ndim"])
    dx = 2.0 * L / N
    x = (torch.arange(N, dtype=torch.float64) - N // 2) * dx
    coords = torch.meshgrid(*([x] * ndim), indexing="ij")
    R2 = coords[0] ** 2 + coords[1] ** 2 + (coords[2] ** 2 if ndim == 3 else 0.0)
    tc = float(G.get("trap_coeff", 0.5))
    V = tc * R2 ** (s / 2.0) if s > 0 else torch.zeros_like(R2)
    Gc = dict(G, coords=coords, X=coords[0], Y=coords[1], R2=R2, V=V, dx=dx)
    if len(_GRID_CACHE) > 8:
        _GRID_CACHE.clear()
    _GRID_CACHE[key] = Gc
    return Gc


def host_tf_density(cfg, G):
    """Thomas-Fermi density of the seeds: dict(n, converged) or None.

    Seeds must equal the reference's element for element. For the local
    references that needs the reference's own CPU tensor arithmetic: a
    chemical potential found with another summation order can differ in the
    last bit, which moves points across the edge of the support and changes
    sqrt(n) there by far more than round-off. So the flat top and the inverted
    profile are formed here with the operations, in the order, of
    becgpp/thomasfermi.py:21-62 and 121-150. The nonlocal density comes from the
    device fixed point (thomasfermi.extract_tf); seeds built on it equal the
    reference's to the fixed point's convergence, not bit for bit."""
    kind = reference_kind(cfg, G)
    if kind is None:
        return None
    if kind == "nonlocal_compressed":
        tf = extract_tf(cfg, G)
        return None if tf is None else dict(n=tf["n"].cpu(), converged=tf["converged"])
    Gc = cpu_grid(G)
    dv = Gc["dx"] ** Gc["ndim"]
    b2, b3 = float(cfg["beta2"]), float(cfg["beta3"])
    if kind == "local_flattop":
        rho0 = -3.0 * b2 / (4.0 * b3)
        R = 1.0 / math.sqrt(math.pi * rho0) if Gc["ndim"] == 2 else (3.0 / (4.0 * math.pi * rho0)) ** (1.0 / 3.0)
        rr = torch.sqrt(Gc["R2"])
        n = torch.where(rr <= R, torch.full_like(rr, rho0), torch.zeros_like(rr))
        return dict(n=n / (n.sum() * dv), converged=True)
    Om = float(cfg.get("Omega", 1.0))
    veff = Gc["V"] - 0.5 * Om * Om * (Gc["X"] ** 2 + Gc["Y"] ** 2)

    def density(mu):
        rhs = mu - veff
        if b3 > 1e-30:
            disc = b2 * b2 + 4.0 * b3 * rhs
            root = (-b2 + torch.sqrt(torch.clamp(disc, min=0.0))) / (2.0 * b3)
            return torch.where(disc > 0.0, torch.clamp(root, min=0.0), torch.zeros_like(rhs))
        return torch.clamp(rhs / b2, min=0.0)

    def mass(mu):
        return (density(mu).sum() * dv).item()

    lo, hi = veff.min().item(), veff.max().item() + abs(b2) + abs(b3) + 1.0
    for _ in range(201):                 # widen the upper end until it holds unit mass
        if mass(hi) >= 1.0:
            break
        hi = lo + 2.0 * (hi - lo) + 1e-9
    else:
        return None
    for _ in range(90):
        mid = 0.5 * (lo + hi)
        if mass(mid) < 1.0:
            lo = mid
        else:
            hi = mid
    n = density(0.5 * (lo + hi))
    return dict(n=n / (n.sum() * dv), converged=True)


def _norm(p, Gc):
    return torch.sqrt((p.abs() ** 2).sum() * Gc["dx"] ** Gc["ndim"])


def gaussian_seed(G, cfg):
    Gc = cpu_grid(G)
    torch.manual_seed(cfg["rng"])
    env = torch.exp(-0.5 * Gc["R2"])
    noise = 1.0 + cfg.get("seed_noise", 1e-2) * torch.randn_like(env)
    psi = (env * noise).to(torch.complex128)
    m = int(cfg.get("seed_winding", 0))
    if m != 0:
        psi = psi * torch.exp(1j * m * torch.atan2(Gc["Y"], Gc["X"]))
    return psi / _norm(psi, Gc)


def tf_seed(G, cfg):
    Gc = cpu_grid(G)
    tf = host_tf_density(cfg, G)
    if tf is None or tf.get("n") is None:
        return gaussian_seed(G, cfg)
    amp = torch.sqrt(torch.clamp(tf["n"], min=0.0))
    torch.manual_seed(cfg["rng"])
    noise = 1.0 + cfg.get("seed_noise", 1e-2) * torch.randn_like(amp)
    pn = cfg.get("seed_phase_noise", 5e-2) * torch.randn_like(amp)
    psi = (amp * noise).to(torch.complex128) * torch.exp(1j * pn)
    m = int(cfg.get("seed_winding", 0))
    if m != 0:
        psi = psi * torch.exp(1j * m * torch.atan2(Gc["Y"], Gc["X"]))
    return psi / _norm(psi, Gc)


def _inplane_radius(n, Gc, frac=0.90):
    w = (torch.clamp(n, min=0.0) * Gc["dx"] ** Gc["ndim"]).reshape(-1)
    rperp = torch.sqrt(Gc["X"] ** 2 + Gc["Y"] ** 2).reshape(-1)
    order = torch.argsort(rperp)
    cum = torch.cumsum(w[order], dim=0)
    jj = int(torch.searchsorted(cum, float(frac) * cum[-1]).clamp(max=cum.numel() - 1).item())
    return rperp[order[jj]].item()


def triangular_seed(G, cfg):
    """Triangular (Abrikosov) vortex lattice on the TF envelope; straight vortex
    lines along z in 3D; winding sign(Omega)."""
    O = float(cfg.get("Omega", 0.0))
    if abs(O) < 0.3:
        return tf_seed(G, cfg)
    tf = host_tf_density(cfg, G)
    if tf is None or not tf.get("converged", False):
        return tf_seed(G, cfg)
    Gc = cpu_grid(G)
    n = tf["n"]
    amp = torch.sqrt(torch.clamp(n, min=0.0))
    wsign = -1.0 if O < 0 else 1.0
    O = abs(O)
    av = math.sqrt(2.0 * math.pi / (math.sqrt(3.0) * O))
    dy = math.sqrt(3.0) * av / 2.0
    Rperp = _inplane_radius(n, Gc, 0.90)
    Rv = max(av, 0.98 * Rperp)
    rng = np.random.default_rng(int(cfg.get("rng", 0)))
    torch.manual_seed(int(cfg.get("rng", 0)))
    angle = float(rng.uniform(0.0, math.pi / 3.0))
    shift = rng.uniform(-0.25, 0.25, size=2) * av
    ca, sa = math.cos(angle), math.sin(angle)
    pos = []
    jmax = int(math.ceil(Rv / dy)) + 2
    imax = int(math.ceil(Rv / av)) + 3
    for jj in range(-jmax, jmax + 1):
        for ii in range(-imax, imax + 1):
            x0 = (ii + 0.5 * (jj & 1)) * av + shift[0]
            y0 = jj * dy + shift[1]
            xx = ca * x0 - sa * y0
            yy = sa * x0 + ca * y0
            if xx * xx + yy * yy < Rv * Rv:
                pos.append((xx, yy))
    phase = torch.zeros_like(amp)
    core = torch.ones_like(amp)
    xi = 0.25 * av
    for xx, yy in pos:
        dxt = Gc["X"] - xx
        dyt = Gc["Y"] - yy
        dist = torch.sqrt(dxt * dxt + dyt * dyt)
        phase = phase + wsign * torch.atan2(dyt, dxt)
        core = core * torch.tanh(dist / max(xi, 1e-12))
    noise = cfg.get("seed_noise", 1e-2) * torch.randn_like(amp)
    psi = (amp * core * (1.0 + noise)).to(torch.complex128) * torch.exp(1j * phase)
    return psi / _norm(psi, Gc)


def make_seed(G, cfg, device=None):
    """Seed of kind cfg['seed'] (gaussian | tf | triangular), on `device`
    (default: the CUDA device when present)."""
    kind = cfg.get("seed", "tf")
    if kind == "triangular":
        p = triangular_seed(G, cfg)
    elif kind == "tf":
        p = tf_seed(G, cfg)
    else:
        p = gaussian_seed(G, cfg)
    dev = device or ("cuda" if torch.cuda.is_available() else "cpu")
    return p.to(dev)


def phase_noise(psi, amplitude, seed):
    """psi * exp(i amplitude N(0,1)) with a CPU generator seeded by `seed`."""
    g = torch.Generator().manual_seed(int(seed))
    ph = amplitude * torch.randn(tuple(psi.shape), generator=g, dtype=torch.float64)
    return psi * torch.exp(1j * ph).to(psi.device)
