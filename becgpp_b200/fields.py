"""Density-field diagnostics (post-solve): centre of mass, mass-quantile radii,
radial profile and droplet edge, computed by libbgp's device kernels
(``bgp_density_center``, ``bgp_mass_quantiles``, ``bgp_radial_profile``).

The definitions are the reference's (becgpp/fields.py:9-66): the centre of
mass is sum(x rho) dV / sum(rho) dV; the quantile radius for a fraction f is
the distance of the first grid point, in order of distance from the centre,
at which the running mass of max(rho, 0) dV reaches f times the total; the
radial profile is the mean of a field over equal shells out to the box edge.
The kernels find the quantile point by radix selection on the distances'
bits instead of sorting the grid (see csrc/bgp_diag.cu). Inputs may live on
the CPU or the device; they are moved to the device as contiguous FP64.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib


def _field(x):
    _lib.require_cuda()
    t = x.detach() if torch.is_tensor(x) else torch.as_tensor(np.asarray(x))
    if t.is_complex():
        t = t.real
    return t.to(device="cuda", dtype=torch.float64).contiguous()


def _geom(G):
    return int(G["ndim"]), int(G["N"]), float(G["L"])


def center_of_mass(rho, G):
    """(x, y[, z]) centre of mass of rho; zeros when the mass is not positive."""
    f = _field(rho)
    ndim, N, L = _geom(G)
    mass = ctypes.c_double()
    c = (ctypes.c_double * 3)()
    _lib.check(_lib.lib().bgp_density_center(ndim, N, L, _lib.ptr(f), ctypes.byref(mass), c,
                                             _lib.stream_ptr()), "bgp_density_center")
    return tuple(c[a] for a in range(ndim))


def mass_quantiles(rho, G, fractions=(0.50, 0.90, 0.99), center=None):
    """Radii around `center` (default: the centre of mass) that enclose the given
    fractions of the mass of max(rho, 0)."""
    f = _field(rho)
    ndim, N, L = _geom(G)
    fr = [float(x) for x in fractions]
    out = (ctypes.c_double * len(fr))()
    cptr = None
    if center is not None:
        cptr = (ctypes.c_double * 3)(*[float(v) for v in center][:3])
    _lib.check(_lib.lib().bgp_mass_quantiles(ndim, N, L, _lib.ptr(f), cptr, (ctypes.c_double * len(fr))(*fr),
                                             len(fr), out, _lib.stream_ptr()), "bgp_mass_quantiles")
    return [out[q] for q in range(len(fr))]


def mass_radius(rho, G, fraction=0.99, center=None):
    return mass_quantiles(rho, G, (fraction,), center=center)[0]


def radial_average(field, G, bins=None, rmax=None, center=None):
    """(bin centres, mean of `field` per shell) around `center` (default the
    origin), shells of equal width out to `rmax` (default L); NaN where a shell
    holds no grid point. The default shell count is rmax / (2 dx), within
    [20, 400]."""
    f = _field(field)
    ndim, N, L = _geom(G)
    rmax = L if rmax is None else float(rmax)
    if bins is None:
        bins = int(min(400, max(20, rmax / (2.0 * G["dx"]))))
    edges = np.linspace(0, rmax, bins + 1)
    ctr = 0.5 * (edges[1:] + edges[:-1])
    c = (ctypes.c_double * 3)(*([float(v) for v in center] if center is not None else [0.0] * ndim)[:3])
    prof = (ctypes.c_double * bins)()
    _lib.check(_lib.lib().bgp_radial_profile(ndim, N, L, _lib.ptr(f), c, edges.ctypes.data_as(
        ctypes.POINTER(ctypes.c_double)), bins, prof, _lib.stream_ptr()), "bgp_radial_profile")
    return ctr, np.array(prof[:bins], dtype=np.float64)


def droplet_radius(rho, G, frac=1e-2):
    """Outermost shell centre (around the centre of mass) whose mean density is
    above `frac` times the profile's peak; NaN for an empty profile."""
    ctr, prof = radial_average(rho, G, center=center_of_mass(rho, G))
    finite = prof[np.isfinite(prof)]
    if finite.size == 0:
        return float("nan")
    peak = float(finite.max())
    if not math.isfinite(peak) or peak <= 0:
        return float("nan")
    above = np.nonzero(np.nan_to_num(prof, nan=-np.inf) > frac * peak)[0]
    return float(ctr[above[-1]]) if above.size else float("nan")
