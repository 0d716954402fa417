"""Long-range interaction: the free-space convolution with the cell-averaged kernel.

``kernel_convolution`` and ``long_range_phi`` keep the signatures of
becgpp/interactions.py:154-171. The kernel tables (4x4(x4) Gauss-Legendre cell
averages, exact self cell, transform) are built on the device when a plan is
created and cached with it; ``clear_kernel_cache`` frees them.
"""
import math

import numpy as np
import torch

from . import _lib
from .grid import plan_for, clear_plans


def _rho_dev(rho):
    _lib.require_cuda()
    return rho.to(device="cuda", dtype=torch.float64).contiguous()


def kernel_convolution(rho, G, which="K"):
    """Discrete free-space convolution (K * rho)(r_i) = sum_j K_ij rho_j dV on the
    zero-padded grid; which = "K" (interaction kernel) or "W" (q2d virial kernel)."""
    if G["kernel"] == "none":
        raise ValueError("kernel_convolution needs a long-range kernel (G['kernel'] != 'none')")
    r = _rho_dev(rho)
    # the table depends on the grid only; any nonzero G_C selects the kernel
    plan = plan_for(G, dict(beta2=0.0, beta3=0.0, Omega=0.0, G_C=1.0))
    out = torch.empty_like(r)
    code = 1 if which == "W" else 0
    _lib.check(_lib.lib().bgp_convolve(plan.handle, 0, _lib.ptr(r), _lib.ptr(out), code,
                                       _lib.stream_ptr()), "bgp_convolve")
    return out


def long_range_phi(rho, G, gc):
    """phi = -G_C (K * rho), free-space boundary conditions."""
    if G["kernel"] == "none" or abs(gc) <= 1e-15:
        return torch.zeros_like(rho)
    return -gc * kernel_convolution(rho, G, "K")


def q2d_kernel(u, l_z):
    """Quasi-2D Newton kernel e^x K0(x) / (sqrt(2 pi) l_z), x = u^2 / (4 l_z^2)
    (becgpp/interactions.py:64-67), evaluated with the library's e^x K0."""
    f = _lib.lib().bgp_k0e
    ut = torch.as_tensor(u, dtype=torch.float64)
    x = (ut * ut / (4.0 * l_z * l_z)).cpu().numpy().reshape(-1)
    v = np.array([f(float(xi)) for xi in x]).reshape(tuple(ut.shape))
    return torch.as_tensor(v / (math.sqrt(2.0 * math.pi) * l_z), dtype=torch.float64, device=ut.device)


def clear_kernel_cache():
    """Free the cached plans and their kernel transforms."""
    clear_plans()
