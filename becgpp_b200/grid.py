"""Grid description, plans and small grid helpers.

``make_grid(cfg)`` returns the same dictionary as becgpp/grid.py:69-101
(coordinates, wave numbers, trap on the device, scalars dx, N, L, kernel...),
so code written against the reference's ``G`` keeps working. The CUDA library
recomputes coordinates, wave numbers and the trap from indices inside its
kernels; these tensors are for callers and diagnostics.

A ``Plan`` owns a libbgp plan (device scratch and kernel tables) for a list of
instances; ``plan_for(G, cfg)`` caches single-instance plans by their grid and
physics.
"""
import ctypes
import math
from collections import OrderedDict

import torch

from . import _lib
from ._lib import InstanceDesc, KERNEL_CODES

DEV = "cuda" if torch.cuda.is_available() else "cpu"


def geometry(cfg):
    """(ndim, quasi) of ``cfg['dimension']``: "2D", "3D" or "quasi2D" (case-insensitive)."""
    g = str(cfg.get("dimension", "2D")).strip().lower()
    if g == "2d":
        return 2, False
    if g == "3d":
        return 3, False
    if g == "quasi2d":
        return 2, True
    raise ValueError(f"unknown dimension {cfg.get('dimension')!r}; use '2D', '3D' or 'quasi2D'")


def resolve_kernel(cfg):
    """(kind, tag): kind in newton | log | q2d | none, as becgpp/grid.py:23-55."""
    ndim, quasi = geometry(cfg)
    k = str(cfg.get("kernel", "auto")).lower()
    if abs(float(cfg.get("G_C", 0.0))) <= 1e-15 or k == "none":
        return "none", 0
    lz = float(cfg.get("l_z", 0.0))
    if k == "auto":
        if ndim == 3:
            k = "newton"
        elif quasi:
            k = "q2d" if lz > 0 else "newton"
        else:
            k = "log"
    if k == "newton":
        return "newton", 1
    if k == "log":
        if ndim != 2:
            raise ValueError("kernel='log' is two-dimensional only")
        return "log", 0
    if k == "q2d":
        if ndim != 2:
            raise ValueError("kernel='q2d' needs dimension '2D' or 'quasi2D'")
        if lz <= 0:
            raise ValueError("kernel='q2d' needs an axial width l_z > 0")
        return "q2d", 0
    raise ValueError(f"unknown kernel {k!r}")


def memory_estimate_gb(ndim, N, pad, kernel):
    """Device memory of one solve with this library: 13 complex fields, 2 real
    potentials and median keys, plus the padded transform scratch and the
    kernel-table quadrant with a long-range term."""
    n = float(N) ** ndim
    b = 13 * 16 * n + 2 * 8 * n + 8 * n
    if kernel != "none":
        M = pad * N
        mh = M // 2 + 1
        b += 16 * (N * mh if ndim == 2 else N * N * mh + N * M * mh) + 8 * mh ** ndim
    return b / 1e9


def make_grid(cfg):
    """Grid dictionary of becgpp/grid.py:69-101 (device tensors, FP64)."""
    ndim, quasi = geometry(cfg)
    L, N, s = float(cfg["L"]), int(cfg["Ngrid"]), float(cfg["s"])
    kkind, kexp = resolve_kernel(cfg)
    dx = 2.0 * L / N
    dev = DEV
    x = (torch.arange(N, device=dev, dtype=torch.float64) - N // 2) * dx
    k1 = 2 * math.pi * torch.fft.fftfreq(N, d=dx, dtype=torch.float64).to(dev)
    if ndim == 2:
        X, Y = torch.meshgrid(x, x, indexing="ij")
        coords = (X, Y)
        R2 = X ** 2 + Y ** 2
        KX, KY = torch.meshgrid(k1, k1, indexing="ij")
        kcoords = (KX, KY)
        K2 = KX ** 2 + KY ** 2
    else:
        X, Y, Z = torch.meshgrid(x, x, x, indexing="ij")
        coords = (X, Y, Z)
        R2 = X ** 2 + Y ** 2 + Z ** 2
        KX, KY, KZ = torch.meshgrid(k1, k1, k1, indexing="ij")
        kcoords = (KX, KY, KZ)
        K2 = KX ** 2 + KY ** 2 + KZ ** 2
    tc = float(cfg.get("trap_coeff", 0.5))
    V = tc * R2 ** (s / 2.0) if s > 0 else torch.zeros_like(R2)
    pad = max(2, int(cfg.get("pad", 2)))
    mem = memory_estimate_gb(ndim, N, pad, kkind)
    if mem > float(cfg.get("mem_warn_gb", 12.0)):
        print(f"[warn] estimated device memory ~{mem:.0f} GB for N={N} ({ndim}D, kernel={kkind}, "
              f"pad={pad})")
    return dict(ndim=ndim, quasi=quasi, coords=coords, kcoords=kcoords,
                X=coords[0], Y=coords[1], KX=kcoords[0], KY=kcoords[1],
                R2=R2, V=V, K2=K2, s=s, trap_coeff=tc, dx=dx, N=N, L=L,
                kernel=kkind, kexp=kexp, l_z=float(cfg.get("l_z", 0.0)), pad=pad,
                mem_estimate_gb=mem)


def dV(G):
    return G["dx"] ** G["ndim"]


def norm_of(p, G):
    return torch.sqrt((p.abs() ** 2).sum() * dV(G))


def auto_grid(cfg):
    """Half-box L and grid N from a radius estimate, for sweeps that resize the
    box per point (becgpp/grid.py:119-137): the long-range radius b2 / (2 G_C),
    the quantum-droplet density -3 b2 / (4 b3) (b2 < 0 < b3), else 4; L = 2.5 R
    (at least 6), dx ~ R/20 in [0.01, 0.1], N a multiple of 32 in [128, cap]."""
    b2, b3, gc = float(cfg["beta2"]), float(cfg["beta3"]), float(cfg["G_C"])
    ndim, _ = geometry(cfg)
    if gc > 1e-15 and b2 > 0:
        R = 0.5 * b2 / gc
    elif b2 < 0 and b3 > 0:
        rho0 = max(-3.0 * b2 / (4.0 * b3), 1e-6)
        R = 1.0 / math.sqrt(math.pi * rho0) if ndim == 2 else (3.0 / (4.0 * math.pi * rho0)) ** (1.0 / 3.0)
    else:
        R = 4.0
    L = max(6.0, 2.5 * R)
    dx = min(0.10, max(R / 20.0, 0.01))
    n = int(math.ceil(2.0 * L / dx))
    cap = 512 if ndim == 2 else 224
    return float(L), int(min(cap, max(128, 32 * math.ceil(n / 32)))), R


def resample_state(psi_old, G_old, G_new):
    """psi_old interpolated (bi/trilinear between the old nodes, zero outside
    them) onto the nodes of G_new by libbgp's device kernel (bgp_resample), and
    normalised there; None when that fails (becgpp/grid.py:140-161)."""
    _lib.require_cuda()
    if G_old["ndim"] != G_new["ndim"]:
        raise ValueError("resample_state needs grids of the same dimension")
    src = psi_old.to(device="cuda", dtype=torch.complex128).contiguous()
    n_new = int(G_new["N"])
    out = torch.empty((n_new,) * int(G_new["ndim"]), dtype=torch.complex128, device="cuda")
    rc = _lib.lib().bgp_resample(int(G_old["ndim"]), int(G_old["N"]), float(G_old["L"]), _lib.ptr(src),
                                 n_new, float(G_new["L"]), _lib.ptr(out), _lib.stream_ptr())
    if rc != 0:
        if b"degenerate" in _lib.lib().bgp_last_error():
            return None
        _lib.check(rc, "bgp_resample")
    nn = norm_of(out, G_new)
    if not torch.isfinite(nn) or nn.item() <= 1e-14:
        return None
    return out / nn


# --------------------------------------------------------------------------- plans
def instance_desc(G, cfg):
    """C descriptor of one instance from a grid dictionary and the physics in cfg."""
    d = InstanceDesc()
    d.ndim = int(G["ndim"])
    d.N = int(G["N"])
    d.pad = int(G["pad"])
    d.kernel = KERNEL_CODES[G["kernel"]]
    d.L = float(G["L"])
    d.s = float(G["s"])
    d.trap_coeff = float(G.get("trap_coeff", 0.5))
    d.beta2 = float(cfg["beta2"])
    d.beta3 = float(cfg["beta3"])
    d.Omega = float(cfg["Omega"])
    d.G_C = float(cfg["G_C"]) if G["kernel"] != "none" else 0.0
    d.l_z = float(G.get("l_z", 0.0))
    return d


def desc_key(d):
    return tuple(getattr(d, f) for f, _ in InstanceDesc._fields_)


class Plan:
    """A libbgp plan for a list of instance descriptors (device scratch and tables)."""

    def __init__(self, descs):
        _lib.require_cuda()
        self.descs = list(descs)
        arr = (InstanceDesc * len(self.descs))(*self.descs)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().bgp_plan_create(arr, len(self.descs), ctypes.byref(h)), "bgp_plan_create")
        self.handle = h

    @property
    def bytes(self):
        return int(_lib.lib().bgp_plan_bytes(self.handle))

    @property
    def launches(self):
        return int(_lib.lib().bgp_plan_launches(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().bgp_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_PLANS = OrderedDict()
_MAX_PLANS = 4


def plan_for(G, cfg):
    """Cached single-instance plan for grid G with the physics of cfg."""
    d = instance_desc(G, cfg)
    key = desc_key(d)
    p = _PLANS.get(key)
    if p is None:
        while len(_PLANS) >= _MAX_PLANS:
            _PLANS.popitem(last=False)[1].close()
        p = Plan([d])
        _PLANS[key] = p
    else:
        _PLANS.move_to_end(key)
    return p


def clear_plans():
    """Free the cached plans (device scratch and kernel tables)."""
    while _PLANS:
        _PLANS.popitem()[1].close()
