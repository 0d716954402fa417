"""Vortex count and lowest-Landau-level weight of a solved state (post-solve
diagnostics, becgpp/vortex.py:10-84), computed by the library's device kernels
(``bgp_vortex_count``, ``bgp_lll_weight``):

- a vortex is a plaquette of the (i, j) grid whose wrapped phase increments
  around its four edges sum to +-2 pi, counted inside the droplet: the cell's
  Gaussian-smoothed density (width min(2 sqrt(pi/|Omega|), max(R/3, 2 dx)))
  above 0.15 of its maximum and its corner within R, the radius around the
  centre of mass that holds 99 % of the mass. In 3D the z = 0 midplane is
  counted (straight vortex lines along z).
- the LLL weight is sum_m |<phi_m, psi>|^2 over the normalised states
  phi_m ~ z^m exp(-r^2/2) (conj(z)^m for Omega < 0), m up to a cap that grows
  with <r^2>; NaN for a 3D state.
"""
import ctypes

import numpy as np
import torch

from . import _lib


def _plane(psi, G):
    """The 2D field the diagnostics read: psi itself, or the z = 0 midplane of a
    3D state, as a contiguous complex128 CUDA tensor."""
    _lib.require_cuda()
    t = psi.detach() if torch.is_tensor(psi) else torch.as_tensor(np.asarray(psi))
    if int(G["ndim"]) == 3:
        t = t[:, :, int(G["N"]) // 2]
    return t.to(device="cuda", dtype=torch.complex128).contiguous()


def vortex_diagnostic(psi, G, Omega=1.0, dens_thresh_frac=0.15):
    """Vortex count of psi (2D; 3D at the z = 0 midplane): {Nv, Nplus, Nminus, Nnet}."""
    p = _plane(psi, G)
    out = (ctypes.c_int * 4)()
    _lib.check(_lib.lib().bgp_vortex_count(int(G["N"]), float(G["L"]), _lib.ptr(p), float(Omega),
                                           float(dens_thresh_frac), out, _lib.stream_ptr()), "bgp_vortex_count")
    return dict(Nv=out[0], Nplus=out[1], Nminus=out[2], Nnet=out[3])


def lll_weight(psi, G, Mmax=60, Omega=1.0):
    """Weight of psi in the lowest Landau level of the rotating harmonic trap
    (2D only; NaN otherwise)."""
    if int(G["ndim"]) != 2:
        return float("nan")
    p = _plane(psi, G)
    w = ctypes.c_double()
    _lib.check(_lib.lib().bgp_lll_weight(int(G["N"]), float(G["L"]), _lib.ptr(p), float(Omega), int(Mmax),
                                         ctypes.byref(w), _lib.stream_ptr()), "bgp_lll_weight")
    return w.value
