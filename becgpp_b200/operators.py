"""Energy functional, Hamiltonian, residual and observables on the CUDA library.

Same names, arguments and return values as becgpp/operators.py:10-103; every
field operation runs in libbgp (FP64). Scalars come back as 0-dim float64
tensors where the reference returns tensors, and as Python floats where it
calls ``.item()``.
"""
import ctypes
import math

import torch

from . import _lib
from .grid import dV, plan_for


def _dev_c128(p):
    _lib.require_cuda()
    return p.to(device="cuda", dtype=torch.complex128).contiguous()


def _physics(beta2, beta3, Omega, G_C):
    return dict(beta2=float(beta2), beta3=float(beta3), Omega=float(Omega), G_C=float(G_C))


def _energy_terms(p, G, phys, want_phi=True):
    p = _dev_c128(p)
    plan = plan_for(G, phys)
    kern = G["kernel"] != "none" and abs(phys["G_C"]) > 1e-15
    phi = torch.zeros(p.shape, dtype=torch.float64, device=p.device)
    t = _lib.EnergyTerms()
    _lib.check(_lib.lib().bgp_energy(plan.handle, 0, _lib.ptr(p), _lib.ptr(phi) if kern else None,
                                     ctypes.byref(t), _lib.stream_ptr()), "bgp_energy")
    return t, phi


def energy_components(p, G, beta2, beta3, Omega, G_C):
    """E and its terms for state p as given (not normalised) and the long-range
    potential phi (becgpp/operators.py:10-29)."""
    t, phi = _energy_terms(p, G, _physics(beta2, beta3, Omega, G_C))
    f = lambda v: torch.tensor(v, dtype=torch.float64)
    return dict(E=f(t.E), Ekin=f(t.Ekin), Etrap=f(t.Etrap), Econtact=f(t.Econtact),
                Ethree=f(t.Ethree), Erot=f(t.Erot), Egrav=f(t.Egrav), Lz=f(t.Lz), phi=phi)


def energy_t(p, G, beta2, beta3, Omega, G_C):
    return energy_components(p, G, beta2, beta3, Omega, G_C)["E"]


def apply_H(psi, G, cfg, phi=None):
    """H psi = -1/2 lap psi + (V + b2 |psi|^2 + b3 |psi|^4 + phi) psi - Omega L_z psi
    (becgpp/operators.py:36-45). ``phi`` may carry the long-range potential of
    this psi; otherwise it is computed from |psi|^2 when the kernel is on."""
    psi = _dev_c128(psi)
    plan = plan_for(G, cfg)
    out = torch.empty_like(psi)
    kern = G["kernel"] != "none" and abs(float(cfg["G_C"])) > 1e-15
    if phi is not None and not (isinstance(phi, (int, float)) and phi == 0):
        ph = phi.to(device=psi.device, dtype=torch.float64).contiguous() if torch.is_tensor(phi) else None
        if ph is None:
            ph = torch.full(psi.shape, float(phi), dtype=torch.float64, device=psi.device)
        mode = 1
    else:
        ph = None
        mode = 2 if kern else 0
    P = ctypes.c_void_p * 1
    _lib.check(_lib.lib().bgp_apply_H_batch(plan.handle, 1, (ctypes.c_int * 1)(0), P(psi.data_ptr()),
                                            P(out.data_ptr()), P(ph.data_ptr()) if ph is not None else None,
                                            mode, None, _lib.stream_ptr()), "bgp_apply_H_batch")
    return out


class HamiltonianBatch:
    """H psi of a fixed list of instances (grids and physics may differ) in one
    call: libbgp's batched apply (bgp_apply_H_batch), per-axis launches over all
    instances of a grid size at once, enqueued on the current stream without a
    host synchronisation. The first apply tunes each grid size's pass schedule.

    cfgs: config dicts; grids: matching grid dictionaries (default make_grid)."""

    def __init__(self, cfgs, grids=None):
        from .grid import Plan, instance_desc, make_grid
        self.cfgs = [dict(c) for c in cfgs]
        self.grids = list(grids) if grids is not None else [make_grid(c) for c in self.cfgs]
        self.plan = Plan([instance_desc(G, c) for G, c in zip(self.grids, self.cfgs)])
        self.n = len(self.cfgs)
        self._idx = (ctypes.c_int * self.n)(*range(self.n))

    def apply(self, psis, out=None, phis=None, mu=None):
        """out[i] = H psis[i]. phis: None (potential computed from |psi|^2 where
        the kernel is on) or a list of potentials; mu: optional device float64
        tensor of n entries receiving Re<psi, H psi> dV."""
        psis = [_dev_c128(p) for p in psis]
        outs = out if out is not None else [torch.empty_like(p) for p in psis]
        P = ctypes.c_void_p * self.n
        ph = None
        mode = 2
        if phis is not None:
            ph = P(*[q.data_ptr() for q in phis])
            mode = 1
        _lib.check(_lib.lib().bgp_apply_H_batch(self.plan.handle, self.n, self._idx,
                                                P(*[p.data_ptr() for p in psis]), P(*[o.data_ptr() for o in outs]),
                                                ph, mode, _lib.ptr(mu), _lib.stream_ptr()), "bgp_apply_H_batch")
        return outs

    def schedule(self, N):
        """Pass schedule of grid size N: lines per tile and radix order of the H psi
        passes; lines per tile of the convolution's contiguous and strided passes
        and its radix order; whether tuned; and the timed candidates as (lines,
        order, strided lines, ms), lines < 0 for a convolution candidate (its
        contiguous width negated)."""
        ln, v, cl, csl, cv, tu, nc = (ctypes.c_int() for _ in range(7))
        cap = 96
        nc.value = cap
        cand = (ctypes.c_float * (4 * cap))()
        _lib.check(_lib.lib().bgp_plan_stream_schedule(self.plan.handle, int(N), ctypes.byref(ln), ctypes.byref(v),
                                                       ctypes.byref(cl), ctypes.byref(csl), ctypes.byref(cv),
                                                       ctypes.byref(tu), cand, ctypes.byref(nc)),
                   "bgp_plan_stream_schedule")
        rows = [(int(cand[4 * q]), int(cand[4 * q + 1]), int(cand[4 * q + 2]), round(float(cand[4 * q + 3]), 4))
                for q in range(min(nc.value, cap))]
        return {"lines": ln.value, "radix_order": v.value, "conv_lines": cl.value, "conv_strided_lines": csl.value,
                "conv_order": cv.value, "tuned": tu.value, "candidates_ms": rows}

    def set_schedule(self, N, lines, radix_order=0, conv_lines=8, conv_order=0, conv_strided_lines=None):
        """Fix the schedule of grid size N (lines = 0: tune again on the next
        apply); the strided convolution passes default to conv_lines."""
        csl = conv_lines if conv_strided_lines is None else conv_strided_lines
        _lib.check(_lib.lib().bgp_plan_stream_set(self.plan.handle, int(N), int(lines), int(radix_order),
                                                  int(conv_lines), int(csl), int(conv_order)), "bgp_plan_stream_set")

    def close(self):
        self.plan.close()


def compute_residual(psi, G, cfg):
    """(||H psi - mu psi||, mu, resid / max(1, |mu|)) with phi recomputed
    (becgpp/operators.py:48-52)."""
    psi = _dev_c128(psi)
    plan = plan_for(G, cfg)
    out = (ctypes.c_double * 3)()
    _lib.check(_lib.lib().bgp_residual(plan.handle, 0, _lib.ptr(psi), out, _lib.stream_ptr()),
               "bgp_residual")
    return float(out[0]), float(out[1]), float(out[2])


def observables(p, G, cfg):
    """E, mu, L_z, rrms, peak, the virial identity and the energy terms
    (becgpp/operators.py:55-103)."""
    from .interactions import kernel_convolution
    gc = float(cfg["G_C"])
    phys = _physics(cfg["beta2"], cfg["beta3"], cfg["Omega"], gc)
    t, _ = _energy_terms(p, G, phys)
    d, s, dv = float(G["ndim"]), float(G["s"]), dV(G)
    mass = t.mass
    mu = t.E + t.Econtact + 2.0 * t.Ethree + t.Egrav
    kind = G["kernel"]
    if kind == "none" or abs(gc) <= 1e-15:
        T_lr = 0.0
    elif kind == "newton":
        T_lr = t.Egrav
    elif kind == "log":
        T_lr = -0.5 * gc * mass * mass
    else:
        pd = _dev_c128(p)
        rho = (pd.real ** 2 + pd.imag ** 2).contiguous()
        T_lr = 0.5 * gc * float(torch.dot(rho.reshape(-1), kernel_convolution(rho, G, "W").reshape(-1))) * dv
    virial = (2.0 * t.Ekin - s * t.Etrap + d * t.Econtact + 2.0 * d * t.Ethree) + T_lr
    vscale = sum(abs(v) for v in (t.Ekin, t.Etrap, t.Econtact, t.Ethree, t.Egrav)) + abs(T_lr)
    O = float(cfg["Omega"])
    binding_ref = 1.0 if (abs(abs(O) - 1.0) < 1e-12 and s == 2 and G["ndim"] == 2) else float("nan")
    out = dict(E=t.E, mu=mu, Lz=t.Lz, rrms=math.sqrt(max(t.r2mean, 0.0)), peak=t.peak,
               E_bind=(t.E - binding_ref) if math.isfinite(binding_ref) else float("nan"),
               virial=virial, virial_rel=abs(virial) / max(1.0, vscale), virial_lr_term=T_lr)
    for k in ("Ekin", "Etrap", "Econtact", "Ethree", "Erot", "Egrav"):
        out[k] = getattr(t, k)
    if G["ndim"] == 3:
        out["R_perp_rms"] = math.sqrt(max(t.rperp2, 0.0))
        out["R_z_rms"] = math.sqrt(max(t.z2, 0.0))
        out["oblateness"] = (out["R_perp_rms"] / math.sqrt(2.0)) / max(out["R_z_rms"], 1e-30)
    else:
        out["R_perp_rms"] = out["R_z_rms"] = float("nan")
        out["oblateness"] = float("nan")
    return out
