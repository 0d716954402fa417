"""Vortex count and lowest-Landau-level weight of a solved state (post-solve
diagnostics, not on the solver path). Same definitions as becgpp/vortex.py:10-84,
computed with torch on the state's own device:

- a vortex is a plaquette of the (i, j) grid whose wrapped phase increments
  around its four edges sum to +-2 pi, counted inside the droplet: the cell's
  Gaussian-smoothed density (width min(2 sqrt(pi/|Omega|), max(R/3, 2 dx)))
  above 0.15 of its maximum and its corner within R, the radius around the
  centre of mass that holds 99 % of the mass. In 3D the z = 0 midplane is
  counted (straight vortex lines along z).
- the LLL weight is sum_m |<phi_m, psi>|^2 over the normalised states
  phi_m ~ z^m exp(-r^2/2) (conj(z)^m for Omega < 0), m up to a cap that grows
  with <r^2>.
"""
import math

import torch

from .grid import dV, norm_of

_NONE = dict(Nv=0, Nplus=0, Nminus=0, Nnet=0)


def _wrap(d):
    """Phase difference folded into [-pi, pi)."""
    return torch.remainder(d + math.pi, 2.0 * math.pi) - math.pi


def _windings(theta):
    """Winding number of every plaquette: corners (i,j) -> (i+1,j) -> (i+1,j+1)
    -> (i,j+1) -> (i,j)."""
    c = (theta[:-1, :-1], theta[1:, :-1], theta[1:, 1:], theta[:-1, 1:])
    total = _wrap(c[1] - c[0])
    for a, b in ((c[1], c[2]), (c[2], c[3]), (c[3], c[0])):
        total = total + _wrap(b - a)
    return torch.round(total / (2.0 * math.pi))


def _radius_holding(rad, w, frac):
    """Smallest sampled radius whose disc holds `frac` of the weights w."""
    order = torch.argsort(rad.reshape(-1))
    cum = torch.cumsum(w.reshape(-1)[order], 0)
    j = int(torch.searchsorted(cum, frac * cum[-1]).clamp(max=cum.numel() - 1).item())
    return rad.reshape(-1)[order[j]].item()


def count_vortices_2d(psi2d, X, Y, dx, Omega=1.0, dens_thresh_frac=0.15):
    """Phase windings of one 2D field inside its droplet: {Nv, Nplus, Nminus, Nnet}."""
    psi2d = psi2d.contiguous()
    rho = psi2d.abs() ** 2
    da = dx * dx
    mass = (rho.sum() * da).item()
    if mass <= 0:
        return dict(_NONE)
    xc = (X * rho).sum().item() * da / mass
    yc = (Y * rho).sum().item() * da / mass
    R = _radius_holding(torch.sqrt((X - xc) ** 2 + (Y - yc) ** 2), rho * da, 0.99)
    if not math.isfinite(R) or R <= 0:
        return dict(_NONE)
    wind = _windings(torch.angle(psi2d))
    n = psi2d.shape[0]
    k = 2.0 * math.pi * torch.fft.fftfreq(n, d=dx).to(psi2d.device)
    k2 = k[:, None] ** 2 + k[None, :] ** 2
    ell = min(2.0 * math.sqrt(math.pi / max(abs(Omega), 1e-9)), max(R / 3.0, 2.0 * dx))
    smooth = torch.fft.ifftn(torch.fft.fftn(rho) * torch.exp(-0.5 * ell ** 2 * k2)).real.clamp(min=0.0)
    cell = 0.25 * (smooth[:-1, :-1] + smooth[1:, :-1] + smooth[1:, 1:] + smooth[:-1, 1:])
    corner_r = torch.sqrt((X[:-1, :-1] - xc) ** 2 + (Y[:-1, :-1] - yc) ** 2)
    inside = (cell > dens_thresh_frac * smooth.max()) & (corner_r < R)
    nplus = int(((wind >= 1) & inside).sum().item())
    nminus = int(((wind <= -1) & inside).sum().item())
    return dict(Nv=nplus + nminus, Nplus=nplus, Nminus=nminus, Nnet=nplus - nminus)


def vortex_diagnostic(psi, G, Omega=1.0, dens_thresh_frac=0.15):
    """Vortex count of psi (2D; 3D at the z = 0 midplane)."""
    if G["ndim"] == 2:
        return count_vortices_2d(psi, G["X"], G["Y"], G["dx"], Omega, dens_thresh_frac)
    m = G["N"] // 2
    return count_vortices_2d(psi[:, :, m], G["X"][:, :, m], G["Y"][:, :, m], G["dx"], Omega,
                             dens_thresh_frac)


def lll_weight(psi, G, Mmax=60, Omega=1.0):
    """Weight of psi in the lowest Landau level of the rotating harmonic trap
    (2D only; NaN otherwise)."""
    if G["ndim"] != 2:
        return float("nan")
    dv = dV(G)
    pn = psi / norm_of(psi, G)
    R2 = G["R2"]
    logr = torch.log(torch.clamp(torch.sqrt(R2), min=1e-300))
    phase = torch.atan2(G["Y"], G["X"]) * (1.0 if Omega >= 0 else -1.0)
    r2mean = (R2 * pn.abs() ** 2).sum().item() * dv
    want = int(math.ceil(r2mean + 10.0 * math.sqrt(max(r2mean, 1.0)) + 30.0))
    mcap = min(max(int(Mmax), want), max(int(Mmax), int((0.80 * G["L"]) ** 2)))
    total = 0.0
    for m in range(mcap + 1):
        if m == 0:
            amp = torch.exp(-0.5 * R2) / math.sqrt(math.pi)
        else:
            amp = torch.exp(m * logr - 0.5 * R2 - 0.5 * (math.log(math.pi) + math.lgamma(m + 1.0)))
        basis = amp.to(torch.complex128) * torch.exp(1j * m * phase)
        basis = basis / norm_of(basis, G)
        total += ((basis.conj() * pn).sum() * dv).abs().item() ** 2
    return min(max(total, 0.0), 1.0)
