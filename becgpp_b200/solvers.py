"""Ground-state solver on the device: normalised preconditioned CG.

``ground_state`` keeps the signature and return value of
becgpp/solvers.py:48-235; the whole iteration (preconditioner with its median
shift, Polak-Ribiere beta, Barzilai-Borwein step, Armijo search, stop tests,
lowest-residual iterate) runs in one persistent launch of libbgp with all
state on the device. ``ground_state_multiseed`` (becgpp/solvers.py:238-263)
solves its seeds as one batch; ``BatchSolver`` solves any list of instances
(grids may differ) in one launch.
"""
import ctypes
import time

import torch

from . import _lib
from ._lib import CG_BETA_CODES, STOP_NAMES, SolverParams, SolveResult
from .grid import Plan, instance_desc, make_grid, plan_for
from .operators import compute_residual, observables
from .seeds import make_seed

SOLVER_KEYS = ("maxit", "res_tol", "energy_tol", "conv_window", "step", "step_max",
                "linesearch_max", "linesearch_stall", "precond_shift_min", "cg_beta", "cg_restart",
                "record_trace", "precision", "mixed_switch_res")


def solver_params(cfg, trace_cap=None):
    cg = str(cfg.get("cg_beta", "pr_precond")).lower()
    if cg not in CG_BETA_CODES:
        raise ValueError(f"cg_beta must be 'pr', 'pr_precond' or 'none', got {cg!r}")
    p = SolverParams()
    p.maxit = int(cfg["maxit"])
    p.linesearch_max = int(cfg.get("linesearch_max", 8))
    p.linesearch_stall = max(1, int(cfg.get("linesearch_stall", 10)))
    p.cg_restart = int(cfg.get("cg_restart", 30))
    p.cg_beta = CG_BETA_CODES[cg]
    p.conv_window = int(cfg.get("conv_window", 2000))
    p.record_trace = 1 if cfg.get("record_trace", False) else 0
    p.trace_cap = int(trace_cap if trace_cap is not None else (p.maxit + 1 if p.record_trace else 0))
    p.res_tol = float(cfg["res_tol"])
    p.energy_tol = float(cfg.get("energy_tol", 1e-9))
    p.step = float(cfg.get("step", 1.0))
    p.step_max = float(cfg.get("step_max", 3.0))
    p.precond_shift_min = float(cfg.get("precond_shift_min", 0.5))
    prec = str(cfg.get("precision", "fp64")).lower()
    if prec not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {prec!r}")
    p.mixed = 1 if prec == "mixed" else 0
    p.mixed_switch_res = float(cfg.get("mixed_switch_res", 1e-5))
    return p


def _c128(p):
    _lib.require_cuda()
    return p.to(device="cuda", dtype=torch.complex128).contiguous()


class BatchSolver:
    """Solve a fixed list of instances together: one plan (scratch and kernel
    tables built once), one persistent launch sequence per ``solve`` call.
    With ``autotune`` the first three solves try the relaunch schedules and the
    later ones use the fastest (``schedule()``).

    cfgs: config dicts (physics and grid may differ between instances; the
    solver keys must agree). grids: matching grid dictionaries (default
    make_grid of each cfg)."""

    def __init__(self, cfgs, grids=None, autotune=False):
        self.cfgs = [dict(c) for c in cfgs]
        self.grids = list(grids) if grids is not None else [make_grid(c) for c in self.cfgs]
        ref = {k: self.cfgs[0].get(k) for k in SOLVER_KEYS}
        for c in self.cfgs[1:]:
            if {k: c.get(k) for k in SOLVER_KEYS} != ref:
                raise ValueError("all instances of one batch need the same solver settings")
        self.params = solver_params(self.cfgs[0])
        self.plan = Plan([instance_desc(G, c) for G, c in zip(self.grids, self.cfgs)])
        self.n = len(self.cfgs)
        if autotune:
            _lib.check(_lib.lib().bgp_plan_autotune(self.plan.handle, 1), "bgp_plan_autotune")

    def schedule(self):
        """Relaunch schedule in use: {'yield_div', 'tuned', 'candidate_ms'}."""
        yd, tuned = ctypes.c_int(), ctypes.c_int()
        ms = (ctypes.c_float * 3)()
        _lib.check(_lib.lib().bgp_plan_schedule(self.plan.handle, ctypes.byref(yd), ctypes.byref(tuned), ms),
                   "bgp_plan_schedule")
        return {"yield_div": yd.value, "tuned": bool(tuned.value), "candidate_ms": [round(x, 3) for x in ms]}

    def solve_raw(self, psi0s, out=None, trace=False):
        """Run the device solver. psi0s: device complex128 tensors (normalised
        inside). Returns (psi list, SolveResult array, trace array or None)."""
        psi0s = [_c128(p) for p in psi0s]
        outs = out if out is not None else [torch.empty_like(p) for p in psi0s]
        P = ctypes.c_void_p * self.n
        a_in = P(*[p.data_ptr() for p in psi0s])
        a_out = P(*[p.data_ptr() for p in outs])
        res = (SolveResult * self.n)()
        tr = None
        params = self.params
        if trace and params.record_trace:
            tr = (ctypes.c_double * (3 * params.trace_cap * self.n))()
        _lib.check(_lib.lib().bgp_solve(self.plan.handle, a_in, a_out, ctypes.byref(params), res, tr,
                                        _lib.stream_ptr()), "bgp_solve")
        return outs, res, tr

    def solve(self, psi0s):
        """Solve and assemble the reference's obs dict per instance."""
        t0 = time.time()
        outs, res, tr = self.solve_raw(psi0s, trace=True)
        wall = time.time() - t0
        results = []
        for i in range(self.n):
            results.append(_finish(outs[i], self.grids[i], self.cfgs[i], res[i], wall, tr, i,
                                   self.params))
        return results

    def close(self):
        self.plan.close()


def _finish(psi, G, cfg, r, wall, tr, i, params):
    if r.status != 0:
        raise RuntimeError("device solver reported an error")
    resid_abs, resid_rel = float(r.resid_abs_final), float(r.resid_rel_final)
    converged = bool(r.converged or resid_rel < float(cfg["res_tol"]))
    obs = observables(psi, G, cfg)
    obs.update(iters=int(r.iters), walltime=wall, resid_abs=resid_abs, resid_rel=resid_rel,
               min_resid=float(r.min_resid), converged=converged,
               stop_reason=STOP_NAMES[int(r.stop_reason)], preconditioner_shift=float(r.sigma),
               trials=int(r.ntrials), accepted=int(r.naccepted), fp64_from=int(r.fp64_from))
    if cfg.get("record_trace", False) and tr is not None:
        base = 3 * params.trace_cap * i
        n = int(r.ntrace)
        iters = max(int(r.iters), 1)
        # per-entry wall time is not recorded on the device; it is apportioned by iteration
        obs["trace"] = [(wall * tr[base + 3 * k] / iters, int(tr[base + 3 * k]), tr[base + 3 * k + 1],
                         tr[base + 3 * k + 2]) for k in range(n)]
    return psi.detach(), G, obs


def ground_state(cfg, G=None, psi0=None, verbose=True):
    """Riemannian preconditioned CG minimisation of the GP energy on the unit
    sphere. Returns (psi, G, obs) as becgpp/solvers.py:48-235."""
    if G is None:
        G = make_grid(cfg)
    psi = _c128(psi0) if psi0 is not None else make_seed(G, cfg)
    params = solver_params(cfg)
    plan = plan_for(G, cfg)
    out = torch.empty_like(psi)
    res = (SolveResult * 1)()
    tr = (ctypes.c_double * (3 * params.trace_cap))() if params.record_trace else None
    P = ctypes.c_void_p * 1
    t0 = time.time()
    _lib.check(_lib.lib().bgp_solve(plan.handle, P(psi.data_ptr()), P(out.data_ptr()),
                                    ctypes.byref(params), res, tr, _lib.stream_ptr()), "bgp_solve")
    wall = time.time() - t0
    psi, G, obs = _finish(out, G, cfg, res[0], wall, tr, 0, params)
    if verbose:
        print(f"[gs] {obs['stop_reason']} it={obs['iters']}: E={obs['E']:.10g} "
              f"res={obs['resid_rel']:.3e}")
    return psi, G, obs


def seed_configs(cfg):
    """Per-seed configs of multi-seed selection: kinds cycled (triangular first
    when |Omega| >= 0.3), rng + j (becgpp/solvers.py:238-251)."""
    n = int(cfg.get("nseeds", 1))
    rotating = abs(float(cfg.get("Omega", 0.0))) >= 0.3
    cycle = ("triangular", "tf", "gaussian") if rotating else ("tf", "gaussian")
    out = []
    for j in range(max(1, n)):
        c = dict(cfg)
        c["rng"] = int(cfg.get("rng", 0)) + j
        c["seed"] = cycle[j % len(cycle)]
        out.append(c)
    return out


def select_lowest(cs, results):
    """The lowest-energy result of a set of seeds, with the seed bookkeeping of
    becgpp/solvers.py:252-263 (seed_used, seed_energy_spread, seed_energies)."""
    Es = [r[2]["E"] for r in results]
    j = min(range(len(Es)), key=lambda k: (Es[k],))
    psi, G, obs = results[j]
    obs["seed_energy_spread"] = (max(Es) - min(Es)) if len(Es) > 1 else 0.0
    obs["seed_used"] = cs[j]["seed"]
    obs["seed_energies"] = ";".join(f"{e:.10g}" for e in Es)
    return psi, G, obs


def ground_state_multiseed(cfg, G=None, verbose=False):
    """Solve nseeds seeds in one batch and keep the lowest energy
    (variational selection, becgpp/solvers.py:238-263)."""
    if G is None:
        G = make_grid(cfg)
    cs = seed_configs(cfg)
    psi0s = [make_seed(G, c) for c in cs]
    bs = BatchSolver(cs, [G] * len(cs))
    try:
        results = bs.solve(psi0s)
    finally:
        bs.close()
    psi, G, obs = select_lowest(cs, results)
    if verbose:
        print(f"[gs-multiseed] {len(cs)} seeds, best {obs['seed_used']} E={obs['E']:.10g} "
              f"(seed energies {obs['seed_energies']})")
    return psi, G, obs
