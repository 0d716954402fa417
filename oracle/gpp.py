"""CPU oracle for the Gross-Pitaevskii ground-state hot path (TEST INFRASTRUCTURE).

This module is test infrastructure, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline / reference arm of
``bench.py`` may import it. The CUDA library in ``becgpp_b200`` never calls it.

It restates, in plain numpy/scipy FP64, the algorithm of becGPP v1.2.1 for the
Hamiltonian apply and the normalised preconditioned CG around it. Each function
names the reference lines it follows (paths relative to the becGPP project).
Parity is pinned against fixtures produced by the reference itself
(``tests/golden/make_golden.py``) and against the reference's known answers
(non-interacting energies, analytic Gaussian potentials).

FFTs use ``scipy.fft`` (pocketfft, like torch's CPU path); ``workers`` sets the
host threads the transforms may use.
"""
from __future__ import annotations

import math
import time

import numpy as np
import scipy.fft as sfft
from scipy import special as sspecial

WORKERS = -1          # host threads for scipy.fft (-1 = all)

# 4-point Gauss-Legendre rule on [-1, 1] (becgpp/interactions.py:32-35): the
# standard nodes/weights, identical in value to the reference's table.
GL_NODES = (-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526)
GL_WTS = (0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538)
# exact self-cell averages (becgpp/interactions.py:41-43); the 3D constant is the
# reference's 10-digit value, kept so the kernel tables agree entry for entry.
SELF_NEWTON_2D = 4.0 * math.asinh(1.0)
SELF_NEWTON_3D = 2.3800773640
SELF_LOG_2D_CONST = 1.5 + 0.5 * math.log(2.0) - 0.25 * math.pi


def fftn(a):
    return sfft.fftn(a, workers=WORKERS)


def ifftn(a):
    return sfft.ifftn(a, workers=WORKERS)


# ----------------------------------------------------------------------------- grid
def geometry(cfg):
    """(ndim, quasi) of ``cfg['dimension']`` (becgpp/grid.py:10-20)."""
    g = str(cfg.get("dimension", "2D")).strip().lower()
    table = {"2d": (2, False), "3d": (3, False), "quasi2d": (2, True)}
    if g not in table:
        raise ValueError(f"unknown dimension {cfg.get('dimension')!r}")
    return table[g]


def resolve_kernel(cfg):
    """Kernel kind for the configured geometry (becgpp/grid.py:23-55)."""
    ndim, quasi = geometry(cfg)
    k = str(cfg.get("kernel", "auto")).lower()
    if abs(float(cfg.get("G_C", 0.0))) <= 1e-15 or k == "none":
        return "none"
    lz = float(cfg.get("l_z", 0.0))
    if k == "auto":
        k = "newton" if ndim == 3 else (("q2d" if lz > 0 else "newton") if quasi else "log")
    if k == "log" and ndim != 2:
        raise ValueError("kernel='log' is two-dimensional only")
    if k == "q2d" and (ndim != 2 or lz <= 0):
        raise ValueError("kernel='q2d' needs 2D and l_z > 0")
    if k not in ("newton", "log", "q2d"):
        raise ValueError(f"unknown kernel {k!r}")
    return k


def make_grid(cfg):
    """Uniform grid, wave numbers, trap (becgpp/grid.py:69-101).

    x_i = (i - N//2) dx, dx = 2L/N; k = 2 pi fftfreq(N, dx) with the Nyquist
    frequency negative; V = trap_coeff * R2**(s/2)."""
    ndim, quasi = geometry(cfg)
    L, N, s = float(cfg["L"]), int(cfg["Ngrid"]), float(cfg["s"])
    dx = 2.0 * L / N
    x = (np.arange(N, dtype=np.float64) - N // 2) * dx
    k1 = 2 * math.pi * np.fft.fftfreq(N, d=dx)
    coords = np.meshgrid(*([x] * ndim), indexing="ij")
    kcoords = np.meshgrid(*([k1] * ndim), indexing="ij")
    R2 = sum(c ** 2 for c in coords)
    K2 = sum(k ** 2 for k in kcoords)
    tc = float(cfg.get("trap_coeff", 0.5))
    V = tc * R2 ** (s / 2.0) if s > 0 else np.zeros_like(R2)
    return dict(ndim=ndim, quasi=quasi, coords=tuple(coords), kcoords=tuple(kcoords),
                X=coords[0], Y=coords[1], KX=kcoords[0], KY=kcoords[1], R2=R2, V=V, K2=K2,
                s=s, trap_coeff=tc, dx=dx, N=N, L=L, kernel=resolve_kernel(cfg),
                l_z=float(cfg.get("l_z", 0.0)), pad=max(2, int(cfg.get("pad", 2))))


def dV(G):
    return G["dx"] ** G["ndim"]


def norm_of(p, G):
    return math.sqrt(float(np.sum(np.abs(p) ** 2)) * dV(G))


def Lz_op(p, G):
    """-i (X d_y p - Y d_x p) by spectral derivatives (becgpp/grid.py:112-116)."""
    fp = fftn(p)
    dpx = ifftn(1j * G["KX"] * fp)
    dpy = ifftn(1j * G["KY"] * fp)
    return -1j * (G["X"] * dpy - G["Y"] * dpx)


# ------------------------------------------------------------------ long-range kernels
def q2d_kernel(u, l_z):
    """Quasi-2D Newton kernel e^x K0(x)/(sqrt(2 pi) l_z), x = u^2/4l_z^2
    (becgpp/interactions.py:64-67)."""
    x = u * u / (4.0 * l_z * l_z)
    return sspecial.k0e(x) / (math.sqrt(2.0 * math.pi) * l_z)


def q2d_virial_kernel(u, l_z):
    """W(u) = u dK/du = 2x (e^x K0 - e^x K1)/(sqrt(2 pi) l_z)
    (becgpp/interactions.py:70-74)."""
    x = u * u / (4.0 * l_z * l_z)
    xs = np.maximum(x, 1e-300)
    return 2.0 * xs * (sspecial.k0e(xs) - sspecial.k1e(xs)) / (math.sqrt(2.0 * math.pi) * l_z)


def polar_self_cell_2d(f, dx, n=48):
    """Average of a radial kernel over the square cell [-dx/2, dx/2]^2 by an
    n x n Gauss-Legendre rule in polar coordinates over the 8 symmetric
    triangles, with r = R t^2 (becgpp/interactions.py:77-94)."""
    t, wt = np.polynomial.legendre.leggauss(n)
    th = 0.5 * (math.pi / 4.0) * (t + 1.0)
    wth = 0.5 * (math.pi / 4.0) * wt
    tt = 0.5 * (t + 1.0)
    wtt = 0.5 * wt
    total = 0.0
    for thj, wj in zip(th, wth):
        R = 0.5 * dx / math.cos(thj)
        r = R * tt ** 2
        jac = 2.0 * R * R * tt ** 3
        total += wj * float(np.sum(f(r) * jac * wtt))
    return 8.0 * total / (dx * dx)


def _point_kernel(which, kind, l_z, r2):
    if which == "W":
        return q2d_virial_kernel(np.sqrt(r2), l_z)
    if kind == "newton":
        return 1.0 / np.sqrt(r2)
    if kind == "log":
        return -0.5 * np.log(r2)
    if kind == "q2d":
        return q2d_kernel(np.sqrt(r2), l_z)
    raise ValueError(kind)


_KCACHE: dict = {}


def kernel_table(G, which="K"):
    """Real-space cell-averaged kernel on the M^d wrap-around grid
    (becgpp/interactions.py:112-147): 4^d-point GL average of the point kernel
    over each cell, offsets dj = j (j <= M//2) else j - M, and the exact
    self-cell value at the origin."""
    N, dx, ndim, pad = G["N"], G["dx"], G["ndim"], G["pad"]
    M = pad * N
    j = np.arange(M, dtype=np.float64)
    dj = np.where(j <= M // 2, j, j - M) * dx
    D = np.meshgrid(*([dj] * ndim), indexing="ij")
    ker = np.zeros_like(D[0])
    kind, lz = G["kernel"], G["l_z"]
    if ndim == 2:
        for u, wu in zip(GL_NODES, GL_WTS):
            for v, wv in zip(GL_NODES, GL_WTS):
                r2 = (D[0] + 0.5 * dx * u) ** 2 + (D[1] + 0.5 * dx * v) ** 2
                ker += 0.25 * wu * wv * _point_kernel(which, kind, lz, r2)
        if which == "W":
            ker[0, 0] = polar_self_cell_2d(lambda r: q2d_virial_kernel(r, lz), dx)
        elif kind == "newton":
            ker[0, 0] = SELF_NEWTON_2D / dx
        elif kind == "log":
            ker[0, 0] = -math.log(dx) + SELF_LOG_2D_CONST
        else:
            ker[0, 0] = polar_self_cell_2d(lambda r: q2d_kernel(r, lz), dx)
    else:
        if kind != "newton":
            raise ValueError("only the Newton kernel is available in 3D")
        for u, wu in zip(GL_NODES, GL_WTS):
            for v, wv in zip(GL_NODES, GL_WTS):
                for w, ww in zip(GL_NODES, GL_WTS):
                    r2 = ((D[0] + 0.5 * dx * u) ** 2 + (D[1] + 0.5 * dx * v) ** 2
                          + (D[2] + 0.5 * dx * w) ** 2)
                    ker += (wu * wv * ww / 8.0) / np.sqrt(r2)
        ker[0, 0, 0] = SELF_NEWTON_3D / dx
    return ker


def kernel_fft(G, which="K"):
    """FFT of the kernel table, cached per grid (becgpp/interactions.py:112-151)."""
    key = (which, G["kernel"], G["ndim"], G["N"], round(G["dx"], 14), G["pad"], round(G["l_z"], 14))
    if key not in _KCACHE:
        _KCACHE[key] = fftn(kernel_table(G, which).astype(np.complex128))
    return _KCACHE[key]


def kernel_convolution(rho, G, which="K"):
    """dV * crop(ifft(fft(pad0(rho)) * Khat)).real, pad offset (M-N)//2
    (becgpp/interactions.py:154-164)."""
    N, ndim = G["N"], G["ndim"]
    Kf = kernel_fft(G, which)
    M = Kf.shape[0]
    i0 = (M - N) // 2
    sl = tuple(slice(i0, i0 + N) for _ in range(ndim))
    rp = np.zeros((M,) * ndim, dtype=np.complex128)
    rp[sl] = rho
    conv = ifftn(fftn(rp) * Kf).real
    return dV(G) * conv[sl]


def long_range_phi(rho, G, gc):
    """phi = -G_C (K * rho) (becgpp/interactions.py:167-171)."""
    if G["kernel"] == "none" or abs(gc) <= 1e-15:
        return np.zeros_like(rho)
    return -gc * kernel_convolution(rho, G, "K")


# ------------------------------------------------------------------------ operators
def energy_components(p, G, beta2, beta3, Omega, G_C):
    """Energy terms and the long-range potential of state p
    (becgpp/operators.py:10-29)."""
    dv = dV(G)
    rho = np.abs(p) ** 2
    fp = fftn(p)
    Ekin = 0.5 * float(np.sum(G["K2"] * np.abs(fp) ** 2)) * dv / p.size
    Etrap = float(np.sum(G["V"] * rho)) * dv
    Econtact = 0.5 * beta2 * float(np.sum(rho ** 2)) * dv
    Ethree = (beta3 / 3.0) * float(np.sum(rho ** 3)) * dv
    Lz = float(np.sum((np.conj(p) * Lz_op(p, G)).real)) * dv
    Erot = -Omega * Lz
    if G["kernel"] != "none" and abs(G_C) > 1e-15:
        phi = long_range_phi(rho, G, G_C)
        Egrav = 0.5 * float(np.sum(phi * rho)) * dv
    else:
        phi = np.zeros_like(rho)
        Egrav = 0.0
    E = Ekin + Etrap + Econtact + Ethree + Erot + Egrav
    return dict(E=E, Ekin=Ekin, Etrap=Etrap, Econtact=Econtact, Ethree=Ethree,
                Erot=Erot, Egrav=Egrav, Lz=Lz, phi=phi)


def apply_H(psi, G, cfg, phi=None):
    """H psi = ifft(k^2/2 fft psi) + (V + b2 rho + b3 rho^2 + phi) psi - Omega Lz psi
    (becgpp/operators.py:36-45)."""
    b2, b3, O, gc = cfg["beta2"], cfg["beta3"], cfg["Omega"], cfg["G_C"]
    kin = ifftn(0.5 * G["K2"] * fftn(psi))
    rho = np.abs(psi) ** 2
    if phi is None:
        phi = long_range_phi(rho, G, gc) if (G["kernel"] != "none" and abs(gc) > 1e-15) else 0.0
    return kin + (G["V"] + b2 * rho + b3 * rho ** 2 + phi) * psi - O * Lz_op(psi, G)


def energy_grad(psi, G, cfg):
    """Derivatives of the energy of energy_components (becgpp/operators.py:10-29)
    at psi: dE/dpsi* = H psi dV (apply_H, becgpp/operators.py:36-45) and
    dE/d(beta2, beta3, G_C, Omega, l_z): 1/2 sum rho^2 dV, 1/3 sum rho^3 dV,
    Egrav/G_C, -L_z and, for the q2d kernel, -(Egrav + E_W)/l_z with E_W the energy
    of the virial kernel's potential (dK/dl_z = -(K + W)/l_z, becgpp/interactions.py:64-74)."""
    b2, b3, O, gc = cfg["beta2"], cfg["beta3"], cfg["Omega"], cfg["G_C"]
    dv = dV(G)
    c = energy_components(psi, G, b2, b3, O, gc)
    rho = np.abs(psi) ** 2
    kern = G["kernel"] != "none" and abs(gc) > 1e-15
    d = dict(beta2=0.5 * float(np.sum(rho ** 2)) * dv, beta3=float(np.sum(rho ** 3)) * dv / 3.0,
             G_C=(c["Egrav"] / gc) if kern else 0.0, Omega=-c["Lz"], l_z=0.0)
    if kern and G["kernel"] == "q2d":
        phiW = -gc * kernel_convolution(rho, G, "W")
        EW = 0.5 * float(np.sum(phiW * rho)) * dv
        d["l_z"] = -(c["Egrav"] + EW) / G["l_z"]
    return apply_H(psi, G, cfg, phi=c["phi"]) * dv, d


def compute_residual(psi, G, cfg):
    """(||H psi - mu psi||, mu, resid/max(1,|mu|)) (becgpp/operators.py:48-52)."""
    Hp = apply_H(psi, G, cfg)
    dv = dV(G)
    mu = float(np.sum((np.conj(psi) * Hp).real)) * dv
    r = math.sqrt(float(np.sum(np.abs(Hp - mu * psi) ** 2)) * dv)
    return r, mu, r / max(1.0, abs(mu))


def observables(p, G, cfg):
    """E, mu, L_z, rrms, peak and the virial identity (becgpp/operators.py:55-103)."""
    b2, b3, O, gc = cfg["beta2"], cfg["beta3"], cfg["Omega"], cfg["G_C"]
    d, s, dv = float(G["ndim"]), float(G["s"]), dV(G)
    c = energy_components(p, G, b2, b3, O, gc)
    rho = np.abs(p) ** 2
    mass = float(np.sum(rho)) * dv
    E = c["E"]
    mu = E + c["Econtact"] + 2.0 * c["Ethree"] + c["Egrav"]
    kind = G["kernel"]
    if kind == "none" or abs(gc) <= 1e-15:
        T_lr = 0.0
    elif kind == "newton":
        T_lr = c["Egrav"]
    elif kind == "log":
        T_lr = -0.5 * gc * mass * mass
    else:
        T_lr = 0.5 * gc * float(np.sum(rho * kernel_convolution(rho, G, "W"))) * dv
    virial = (2.0 * c["Ekin"] - s * c["Etrap"] + d * c["Econtact"] + 2.0 * d * c["Ethree"]) + T_lr
    vscale = sum(abs(c[k]) for k in ("Ekin", "Etrap", "Econtact", "Ethree", "Egrav")) + abs(T_lr)
    r2mean = float(np.sum(G["R2"] * rho)) * dv
    out = dict(E=E, mu=mu, Lz=c["Lz"], rrms=math.sqrt(max(r2mean, 0.0)), peak=float(rho.max()),
               virial=virial, virial_rel=abs(virial) / max(1.0, vscale), virial_lr_term=T_lr)
    for k in ("Ekin", "Etrap", "Econtact", "Ethree", "Erot", "Egrav"):
        out[k] = c[k]
    return out


# --------------------------------------------------------------------------- solver
def _inner_re(u, v, dv):
    return float(np.sum((np.conj(u) * v).real)) * dv


def _proj_tangent(v, psi, dv):
    return v - psi * (np.sum(np.conj(psi) * v) * dv)


def lower_median(vals):
    """Lower middle element of a 1-D sample, the value torch.median returns."""
    m = vals.size
    k = (m - 1) // 2
    return float(np.partition(vals, k)[k])


def preconditioner(grad, psi, G, cfg, phi=None):
    """z = P_T[ifft(fft(grad) / (k^2/2 + sigma))] with sigma the lower median of
    V + 2 b2 rho + 3 b3 rho^2 (+ phi) over rho > 0.05 max rho, floored at
    precond_shift_min (becgpp/solvers.py:28-45)."""
    rho = np.abs(psi) ** 2
    b2, b3, gc = cfg["beta2"], cfg["beta3"], cfg["G_C"]
    local = G["V"] + 2.0 * b2 * rho + 3.0 * b3 * rho ** 2
    if G["kernel"] != "none" and abs(gc) > 1e-15:
        local = local + (phi if phi is not None else long_range_phi(rho, G, gc))
    vals = local[rho > 0.05 * rho.max()]
    floor = float(cfg.get("precond_shift_min", 0.5))
    sigma = lower_median(vals) if vals.size else floor
    sigma = max(sigma, floor)
    z = ifftn(fftn(grad) / (0.5 * G["K2"] + sigma))
    return _proj_tangent(z, psi, dV(G)), sigma


def ground_state(cfg, psi0, G=None, verbose=False):
    """Riemannian preconditioned CG on the unit sphere (becgpp/solvers.py:48-235):
    Sobolev preconditioner, Polak-Ribiere beta (pr_precond | pr | none) with
    restart, Barzilai-Borwein trial step mixed 50/50 into alpha, Armijo
    backtracking (c1 = 1e-4, halving), stall exit, windowed energy stop and the
    lowest-residual iterate. Returns (psi, obs)."""
    if G is None:
        G = make_grid(cfg)
    dv = dV(G)
    psi = np.asarray(psi0, dtype=np.complex128)
    psi = psi / norm_of(psi, G)
    maxit = int(cfg["maxit"])
    res_tol = float(cfg["res_tol"])
    etol = float(cfg.get("energy_tol", 1e-9))
    alpha = float(cfg.get("step", 1.0))
    alpha_min, alpha_max = 1e-8, float(cfg.get("step_max", 3.0))
    ls_max = int(cfg.get("linesearch_max", 8))
    stall_max = max(1, int(cfg.get("linesearch_stall", 10)))
    c1, shrink, growth = 1e-4, 0.5, 1.1
    bb_min, bb_max, bb_mix = 0.05, alpha_max, 0.5
    restart = int(cfg.get("cg_restart", 30))
    cg_beta = str(cfg.get("cg_beta", "pr_precond")).lower()
    if cg_beta not in ("pr", "pr_precond", "none"):
        raise ValueError(f"cg_beta must be 'pr', 'pr_precond' or 'none', got {cg_beta!r}")
    window = int(cfg.get("conv_window", 2000))
    b2, b3, O, gc = cfg["beta2"], cfg["beta3"], cfg["Omega"], cfg["G_C"]

    def energy_phi(p):
        c = energy_components(p, G, b2, b3, O, gc)
        return c["E"], c["phi"]

    def residual(p, phi):
        Hp = apply_H(p, G, cfg, phi=phi)
        mu = float(np.sum(np.conj(p) * Hp).real) * dv
        g = Hp - mu * p
        ra = math.sqrt(float(np.sum(np.abs(g) ** 2)) * dv)
        return g, mu, ra, ra / max(1.0, abs(mu))

    E, phi = energy_phi(psi)
    t0 = time.time()
    trace = [(0.0, 0, E, float("nan"))]
    grad, mu, _, resid_rel = residual(psi, phi)
    z, sigma = preconditioner(grad, psi, G, cfg, phi)
    direction = z.copy()
    z_prev = z
    converged, stop = False, "maxit"
    psi_prev, grad_prev = psi, grad
    best_resid, best_psi = resid_rel, psi.copy()
    E_ref, it_ref = E, 0
    n_fail = n_iter = 0
    ntrials = 0
    for it in range(maxit):
        n_iter = it + 1
        z, sigma = preconditioner(grad, psi, G, cfg, phi)
        if it == 0 or cg_beta == "none" or (restart > 0 and it % restart == 0):
            beta = 0.0
        else:
            y = grad - grad_prev
            if cg_beta == "pr_precond":
                den = max(_inner_re(z_prev, grad_prev, dv), 1e-300)
                beta = max(0.0, _inner_re(z, y, dv) / den)
            else:
                den = max(_inner_re(grad_prev, grad_prev, dv), 1e-300)
                beta = max(0.0, _inner_re(grad, y, dv) / den)
            if not math.isfinite(beta):
                beta = 0.0
        dirc = _proj_tangent(z + beta * direction, psi, dv)
        gd = _inner_re(grad, dirc, dv)
        if gd <= 0:
            dirc = z
            gd = _inner_re(grad, dirc, dv)
        if gd <= 0:
            dirc = _proj_tangent(grad, psi, dv)
            gd = _inner_re(grad, dirc, dv)
        if it > 0:
            svec, yvec = psi - psi_prev, grad - grad_prev
            sy = _inner_re(svec, yvec, dv)
            if sy > 1e-30 and math.isfinite(sy):
                bb = _inner_re(svec, svec, dv) / sy
                if math.isfinite(bb):
                    alpha = (1.0 - bb_mix) * alpha + bb_mix * min(max(bb, bb_min), bb_max)
        alpha = min(max(alpha, alpha_min), alpha_max)
        accepted = False
        trial = alpha
        for _ in range(ls_max):
            psi_t = psi - trial * dirc
            psi_t = psi_t / norm_of(psi_t, G)
            Et, phi_t = energy_phi(psi_t)
            ntrials += 1
            if math.isfinite(Et) and Et <= E - c1 * trial * gd:
                accepted = True
                break
            trial *= shrink
            if trial < alpha_min:
                break
        if not accepted:
            n_fail += 1
            alpha = max(alpha * 0.5, alpha_min)
            direction = z.copy()
            if alpha <= alpha_min or n_fail >= stall_max:
                stop = "line_search_stalled"
                break
            continue
        n_fail = 0
        psi_prev, grad_prev, z_prev = psi, grad, z
        psi, E, phi = psi_t, Et, phi_t
        alpha = min(alpha_max, trial * growth)
        direction = dirc
        grad, mu, _, resid_rel = residual(psi, phi)
        trace.append((time.time() - t0, it + 1, E, resid_rel))
        if resid_rel < best_resid:
            best_resid, best_psi = resid_rel, psi.copy()
        if resid_rel < res_tol:
            converged, stop = True, "converged"
            break
        if it - it_ref >= window:
            if abs(E - E_ref) / max(1.0, abs(E)) < etol:
                converged, stop = True, "energy_converged"
                break
            E_ref, it_ref = E, it
    if best_resid < resid_rel:
        psi = best_psi
    resid_abs, _, resid_rel = compute_residual(psi, G, cfg)
    converged = bool(converged or resid_rel < res_tol)
    obs = observables(psi, G, cfg)
    obs.update(iters=n_iter, walltime=time.time() - t0, resid_abs=resid_abs, resid_rel=resid_rel,
               min_resid=best_resid, converged=converged, stop_reason=stop,
               preconditioner_shift=sigma, trace=trace, trials=ntrials)
    return psi, obs


def seed_cycle(Omega):
    """Seed kinds tried by multi-seed selection (becgpp/solvers.py:242-244)."""
    return ("triangular", "tf", "gaussian") if abs(float(Omega)) >= 0.3 else ("tf", "gaussian")


# ----------------------------------------------------------------- density diagnostics
def _coords(G):
    x = (np.arange(G["N"]) - G["N"] // 2) * G["dx"]
    return np.meshgrid(*([x] * G["ndim"]), indexing="ij")


def center_of_mass(rho, G):
    """sum(x rho) dV / (sum rho dV) per axis, zeros for a non-positive mass
    (becgpp/fields.py:9-14)."""
    dv = dV(G)
    mass = float(rho.sum()) * dv
    if mass <= 0:
        return tuple(0.0 for _ in range(G["ndim"]))
    return tuple(float((c * rho).sum()) * dv / mass for c in _coords(G))


def mass_quantiles(rho, G, fractions=(0.50, 0.90, 0.99), center=None):
    """Distance of the first point, in order of distance from the centre, whose
    running mass of max(rho, 0) dV reaches f times the total (becgpp/fields.py:17-30)."""
    w = (np.clip(rho, 0.0, None) * dV(G)).reshape(-1)
    if center is None:
        center = center_of_mass(rho, G)
    r = np.sqrt(sum((c - center[i]) ** 2 for i, c in enumerate(_coords(G)))).reshape(-1)
    order = np.argsort(r, kind="stable")
    cum = np.cumsum(w[order])
    out = []
    for f in fractions:
        j = min(int(np.searchsorted(cum, float(f) * cum[-1], side="left")), cum.size - 1)
        out.append(float(r[order[j]]))
    return out


def radial_average(field, G, bins=None, rmax=None, center=None):
    """Mean of `field` over equal shells out to rmax (default L), NaN where empty
    (becgpp/fields.py:37-57)."""
    coords = _coords(G)
    center = center if center is not None else tuple(0.0 for _ in coords)
    r = np.sqrt(sum((c - center[i]) ** 2 for i, c in enumerate(coords)))
    rmax = G["L"] if rmax is None else rmax
    if bins is None:
        bins = int(min(400, max(20, rmax / (2.0 * G["dx"]))))
    edges = np.linspace(0, rmax, bins + 1)
    idx = np.clip(np.digitize(r.ravel(), edges) - 1, 0, bins - 1)
    f = np.asarray(field).ravel()
    prof = np.full(bins, np.nan)
    for b in range(bins):
        m = idx == b
        if m.any():
            prof[b] = f[m].mean()
    return 0.5 * (edges[1:] + edges[:-1]), prof


def _wrap_phase(d):
    """Phase difference folded into [-pi, pi) (becgpp/vortex.py, the floored
    remainder of d + pi by 2 pi, minus pi)."""
    return np.remainder(d + math.pi, 2.0 * math.pi) - math.pi


def vortex_count_2d(psi2d, N, L, Omega=1.0, dens_thresh_frac=0.15):
    """Plaquette winding count inside the droplet (becgpp/vortex.py:10-48):
    {Nv, Nplus, Nminus, Nnet} of an N x N field on x_i = (i - N/2) dx."""
    G = dict(N=N, ndim=2, dx=2.0 * L / N, L=L)
    psi2d = np.asarray(psi2d, dtype=np.complex128)
    rho = np.abs(psi2d) ** 2
    da = G["dx"] ** 2
    none = dict(Nv=0, Nplus=0, Nminus=0, Nnet=0)
    mass = float(rho.sum()) * da
    if mass <= 0:
        return none
    center = center_of_mass(rho, G)
    R = mass_quantiles(rho, G, (0.99,), center)[0]
    if not math.isfinite(R) or R <= 0:
        return none
    th = np.angle(psi2d)
    c = (th[:-1, :-1], th[1:, :-1], th[1:, 1:], th[:-1, 1:])
    tot = _wrap_phase(c[1] - c[0])
    for a, b in ((c[1], c[2]), (c[2], c[3]), (c[3], c[0])):
        tot = tot + _wrap_phase(b - a)
    wind = np.round(tot / (2.0 * math.pi))
    k = 2.0 * math.pi * np.fft.fftfreq(N, d=G["dx"])
    k2 = k[:, None] ** 2 + k[None, :] ** 2
    ell = min(2.0 * math.sqrt(math.pi / max(abs(Omega), 1e-9)), max(R / 3.0, 2.0 * G["dx"]))
    smooth = np.clip(np.real(np.fft.ifftn(np.fft.fftn(rho) * np.exp(-0.5 * ell ** 2 * k2))), 0.0, None)
    cell = 0.25 * (smooth[:-1, :-1] + smooth[1:, :-1] + smooth[1:, 1:] + smooth[:-1, 1:])
    X, Y = _coords(G)
    corner_r = np.sqrt((X[:-1, :-1] - center[0]) ** 2 + (Y[:-1, :-1] - center[1]) ** 2)
    inside = (cell > dens_thresh_frac * smooth.max()) & (corner_r < R)
    nplus = int(((wind >= 1) & inside).sum())
    nminus = int(((wind <= -1) & inside).sum())
    return dict(Nv=nplus + nminus, Nplus=nplus, Nminus=nminus, Nnet=nplus - nminus)


def lll_weight_2d(psi2d, N, L, Mmax=60, Omega=1.0):
    """Weight of psi in the lowest Landau level, sum_m |<phi_m, psi/|psi|>|^2 over
    grid-normalised phi_m ~ r^m exp(-r^2/2) e^(i m theta) (becgpp/vortex.py:61-84)."""
    G = dict(N=N, ndim=2, dx=2.0 * L / N, L=L)
    dv = G["dx"] ** 2
    psi2d = np.asarray(psi2d, dtype=np.complex128)
    pn = psi2d / math.sqrt(float((np.abs(psi2d) ** 2).sum()) * dv)
    X, Y = _coords(G)
    R2 = X ** 2 + Y ** 2
    logr = np.log(np.clip(np.sqrt(R2), 1e-300, None))
    phase = np.arctan2(Y, X) * (1.0 if Omega >= 0 else -1.0)
    r2mean = float((R2 * np.abs(pn) ** 2).sum()) * dv
    want = int(math.ceil(r2mean + 10.0 * math.sqrt(max(r2mean, 1.0)) + 30.0))
    mcap = min(max(int(Mmax), want), max(int(Mmax), int((0.80 * L) ** 2)))
    total = 0.0
    for m in range(mcap + 1):
        if m == 0:
            amp = np.exp(-0.5 * R2) / math.sqrt(math.pi)
        else:
            amp = np.exp(m * logr - 0.5 * R2 - 0.5 * (math.log(math.pi) + math.lgamma(m + 1.0)))
        basis = amp * np.exp(1j * m * phase)
        basis = basis / math.sqrt(float((np.abs(basis) ** 2).sum()) * dv)
        total += abs(complex((np.conj(basis) * pn).sum()) * dv) ** 2
    return min(max(total, 0.0), 1.0)


def resample_state(psi_old, G_old, G_new):
    """Bi/trilinear interpolation of psi_old between the old nodes onto the new
    nodes (zero outside the old nodes), normalised on the new grid; None when
    degenerate. Restates torch's grid_sample(align_corners=True, zeros padding)
    as becgpp/grid.py:140-161 calls it: the first old node maps to index 0, the
    last to N_old - 1."""
    d = G_old["ndim"]
    n_old, dx_old = int(G_old["N"]), float(G_old["dx"])
    x0 = -(n_old // 2) * dx_old
    x1 = x0 + (n_old - 1) * dx_old
    if not x1 > x0:
        return None
    xn = (np.arange(G_new["N"]) - G_new["N"] // 2) * G_new["dx"]
    ix = ((2.0 * (xn - x0) / (x1 - x0) - 1.0 + 1.0) / 2.0) * (n_old - 1)
    lo = np.floor(ix).astype(int)
    w1 = ix - lo
    out = np.zeros((G_new["N"],) * d, dtype=np.complex128)
    for corner in range(1 << d):
        w = np.ones((G_new["N"],) * d)
        ok = np.ones((G_new["N"],) * d, dtype=bool)
        idx = []
        for a in range(d):
            hi = (corner >> (d - 1 - a)) & 1
            ia = lo + hi
            wa = w1 if hi else 1.0 - w1
            shape = [1] * d
            shape[a] = -1
            w = w * wa.reshape(shape)
            ok = ok & ((ia >= 0) & (ia < n_old)).reshape(shape)
            idx.append(np.clip(ia, 0, n_old - 1).reshape(shape))
        vals = psi_old[tuple(np.broadcast_arrays(*idx))]
        out += np.where(ok, w * vals, 0.0)
    nn = math.sqrt(float((np.abs(out) ** 2).sum()) * G_new["dx"] ** d)
    if not math.isfinite(nn) or nn <= 1e-14:
        return None
    return out / nn
