"""Derivatives of the Gross-Pitaevskii energy functional on the device.

The reference has no derivative API; these follow from its energy functional
(becgpp/operators.py:10-29):

    dE/dpsi*   = H psi dV                       (apply_H, becgpp/operators.py:36-45)
    dE/dbeta2  = 1/2 sum |psi|^4 dV
    dE/dbeta3  = 1/3 sum |psi|^6 dV
    dE/dG_C    = Egrav / G_C                    (phi is linear in G_C)
    dE/dOmega  = -L_z
    dE/dl_z    = -(Egrav + E_W) / l_z           (q2d: dK/dl_z = -(K + W)/l_z with the
                                                 virial kernel W, becgpp/interactions.py:64-74)

All of them come from one call of ``bgp_energy_grad`` (energy sums, one H psi and,
for q2d, one convolution with W), the backward pass of :class:`EnergyFunction`.
At a converged ground state psi (normalised, stationary on the unit sphere) the
same numbers are the derivatives of the ground-state energy with respect to the
parameters (Hellmann-Feynman): :func:`ground_state_sensitivities`.
"""
import ctypes

import torch

from . import _lib
from .grid import dV, plan_for

PARAMS = ("beta2", "beta3", "G_C", "Omega", "l_z")


def _phys_grid(G, beta2, beta3, G_C, Omega, l_z):
    """Grid dictionary and physics dict for a plan at these parameter values."""
    Gx = dict(G)
    if l_z is not None:
        Gx["l_z"] = float(l_z)
    cfg = dict(beta2=float(beta2), beta3=float(beta3), G_C=float(G_C), Omega=float(Omega))
    return Gx, cfg


def energy_and_grad(psi, G, beta2, beta3, G_C, Omega, l_z=None, want_psi_grad=True):
    """E, its terms, dE/dpsi* (= H psi dV, or None) and dE/d(beta2, beta3, G_C,
    Omega, l_z) at psi (as given, not normalised)."""
    _lib.require_cuda()
    psi = psi.to(device="cuda", dtype=torch.complex128).contiguous()
    Gx, phys = _phys_grid(G, beta2, beta3, G_C, Omega, l_z)
    plan = plan_for(Gx, phys)
    terms = _lib.EnergyTerms()
    dparams = (ctypes.c_double * 5)()
    dpsi = torch.empty_like(psi) if want_psi_grad else None
    _lib.check(_lib.lib().bgp_energy_grad(plan.handle, 0, _lib.ptr(psi), ctypes.byref(terms),
                                          _lib.ptr(dpsi), dparams, _lib.stream_ptr()),
               "bgp_energy_grad")
    t = {k: getattr(terms, k) for k, _ in _lib.EnergyTerms._fields_}
    return t, dpsi, dict(zip(PARAMS, list(dparams)))


class EnergyFunction(torch.autograd.Function):
    """E(psi, beta2, beta3, G_C, Omega, l_z) with a hand-written backward.

    forward returns E as a 0-dim float64 tensor; backward returns torch's
    gradient convention for a complex input of a real function,
    2 dE/dpsi* = 2 H psi dV, and dE/d(parameter) for each parameter tensor."""

    @staticmethod
    def forward(ctx, psi, beta2, beta3, G_C, Omega, l_z, G):
        lz = None if l_z is None else float(l_z)
        terms, dpsi, dp = energy_and_grad(psi, G, float(beta2), float(beta3), float(G_C),
                                          float(Omega), lz, want_psi_grad=ctx.needs_input_grad[0])
        ctx.save_for_backward(dpsi if dpsi is not None else torch.empty(0))
        ctx.dparams = dp
        ctx.has_psi = dpsi is not None
        ctx.devices = [t.device if torch.is_tensor(t) else None for t in (beta2, beta3, G_C, Omega, l_z)]
        return torch.tensor(terms["E"], dtype=torch.float64, device=psi.device)

    @staticmethod
    def backward(ctx, gE):
        (dpsi,) = ctx.saved_tensors
        g_psi = (2.0 * gE) * dpsi if ctx.has_psi else None
        out = [g_psi]
        for name, dev in zip(PARAMS, ctx.devices):
            v = ctx.dparams[name]
            out.append(gE * torch.tensor(v, dtype=torch.float64, device=gE.device) if dev is not None
                       else None)
        out.append(None)  # G
        return tuple(out)


def _as_param(x):
    if torch.is_tensor(x):
        return x
    return torch.tensor(float(x), dtype=torch.float64)


def energy(psi, G, beta2, beta3, G_C, Omega, l_z=None):
    """Differentiable energy of psi: gradients flow to psi and to every
    parameter given as a tensor with requires_grad."""
    if l_z is None and G.get("kernel") == "q2d":
        l_z = float(G["l_z"])
    lz = None if l_z is None else _as_param(l_z)
    return EnergyFunction.apply(psi, _as_param(beta2), _as_param(beta3), _as_param(G_C),
                                _as_param(Omega), lz, G)


def ground_state_sensitivities(psi, G, cfg):
    """dE_gs/d(beta2, beta3, G_C, Omega, l_z) at a converged ground state psi
    (Hellmann-Feynman: the explicit parameter derivatives of E at fixed psi)."""
    _, _, dp = energy_and_grad(psi, G, cfg["beta2"], cfg["beta3"], cfg["G_C"], cfg["Omega"],
                               G.get("l_z") if G.get("kernel") == "q2d" else None,
                               want_psi_grad=False)
    return dp


def hpsi_identity_error(psi, G, cfg):
    """max |dE/dpsi* - H psi dV| / max |H psi dV| (the backward against apply_H)."""
    from .operators import apply_H
    _, dpsi, _ = energy_and_grad(psi, G, cfg["beta2"], cfg["beta3"], cfg["G_C"], cfg["Omega"],
                                 G.get("l_z") if G.get("kernel") == "q2d" else None)
    ref = apply_H(psi, G, cfg) * dV(G)
    return float((dpsi - ref).abs().max() / ref.abs().max())
