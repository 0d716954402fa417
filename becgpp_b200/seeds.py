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

from .thomasfermi import extract_tf, cpu_grid


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
    tf = extract_tf(cfg, G)
    if tf is None or tf.get("n") is None:
        return gaussian_seed(G, cfg)
    amp = torch.sqrt(torch.clamp(tf["n"].cpu(), min=0.0))
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
    tf = extract_tf(cfg, G)
    if tf is None or not tf.get("converged", False):
        return tf_seed(G, cfg)
    Gc = cpu_grid(G)
    n = tf["n"].cpu()
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
