"""`run(cfg)`: the reference's mode dispatch (becgpp/modes.py:469-493) over the
device solver.

Modes:
  single       one ground state (nseeds > 1: the seeds as one batch, lowest E),
               its diagnostics                         (becgpp/modes.py:207-258)
  sweep        one numeric key over sweep_values; per point the continuation
               from the previous point's state and/or fresh seeds, lowest E
               kept. Every fresh-seed solve of the sweep runs as ONE batch
               before the continuation chain, which is sequential by nature
                                                        (becgpp/modes.py:295-387)
  convergence  refine N, box and padding at fixed physics (becgpp/modes.py:393-434)
  tf_only      the Thomas-Fermi reference alone         (becgpp/modes.py:264-289)
  smoke        a small single run and tf_only           (becgpp/modes.py:440-456)

Results are returned as the reference returns them. Output files (one CSV per
mode, a JSON record and a checkpoint per single run) are written only when
cfg["output_dir"] is set; figures are not drawn. The reference's analytic
validation gate (mode "validate") is not part of this package.
"""
import hashlib
import json
import math
import os
import csv

import torch

from .config import CFG_DEFAULTS, canonical_key
from .diagnostics import diagnostics
from .grid import DEV, auto_grid, geometry, make_grid, resample_state, resolve_kernel
from .seeds import make_seed
from .solvers import (SOLVER_KEYS, BatchSolver, ground_state, ground_state_multiseed, seed_configs,
                      select_lowest)
from .thomasfermi import extract_tf

CODE_VERSION = "becgpp_b200_0.1"

# keys that do not change the physics or the solve, left out of the run id
# (becgpp/io.py:13-19)
_RID_EXCLUDE = frozenset({
    "mode", "tag", "maxit", "check", "record_trace", "mem_warn_gb", "want_vortices", "want_lll",
    "tf_cache", "validate_N", "sweep_param", "sweep_values", "sweep_autobox", "sweep_continuation",
    "conv_Ngrids", "conv_box_factors", "conv_pads", "show_inline", "save_figs", "save_ckpt",
    "zip_output", "output_dir", "precision", "mixed_switch_res",
})


def run_id(cfg):
    """tag + a hash of every config key that shapes the result."""
    keys = sorted(k for k in CFG_DEFAULTS if k not in _RID_EXCLUDE)
    raw = json.dumps(dict(code=CODE_VERSION, **{k: cfg.get(k, CFG_DEFAULTS[k]) for k in keys}),
                     sort_keys=True, default=str)
    return f"{cfg.get('tag', 'becgpp')}_{hashlib.md5(raw.encode()).hexdigest()[:10]}"


def write_csv(path, rows):
    if not rows:
        return
    fields = sorted({k for r in rows for k in r})
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=fields, extrasaction="ignore")
        w.writeheader()
        w.writerows(rows)


def _out_dir(cfg):
    d = cfg.get("output_dir")
    if d:
        os.makedirs(d, exist_ok=True)
    return d


def _solve_point(cfg, G, psi0=None):
    if int(cfg.get("nseeds", 1)) > 1 and psi0 is None:
        return ground_state_multiseed(cfg, G=G, verbose=False)
    return ground_state(cfg, G=G, psi0=psi0, verbose=False)


# --------------------------------------------------------------------- single
def mode_single(cfg):
    rid = run_id(cfg)
    G = make_grid(cfg)
    out = _out_dir(cfg)
    psi0 = None
    ck = os.path.join(out, f"{rid}.pt") if out else None
    if ck and os.path.isfile(ck):
        try:
            psi0 = torch.load(ck, map_location=DEV, weights_only=False)["psi"].to(DEV)
            print(f"[resume] {ck}")
        except Exception as exc:                       # a damaged checkpoint: start afresh
            print(f"[resume-warn] {exc}")
    psi, G, obs = _solve_point(cfg, G, psi0)
    diag = diagnostics(psi, G, cfg)
    diag.update(rid=rid, iters=obs["iters"], walltime=obs["walltime"], resid_rel=obs["resid_rel"],
                min_resid=obs.get("min_resid", float("nan")), converged=obs["converged"],
                stop_reason=obs.get("stop_reason", ""), seed_used=obs.get("seed_used", cfg.get("seed")),
                seed_energy_spread=obs.get("seed_energy_spread", 0.0), dimension=cfg["dimension"],
                kernel=G["kernel"], L=cfg["L"], N=cfg["Ngrid"], s=cfg["s"], Omega=cfg["Omega"],
                beta2=cfg["beta2"], beta3=cfg["beta3"], G_C=cfg["G_C"], l_z=cfg.get("l_z", 0.0),
                device=str(DEV))
    if out:
        if cfg.get("save_ckpt", True):
            torch.save(dict(psi=psi.cpu(), cfg=cfg, obs=diag), ck)
        write_csv(os.path.join(out, "single_summary.csv"), [diag])
        with open(os.path.join(out, f"{rid}.json"), "w") as f:
            json.dump(dict(code_version=CODE_VERSION, device=DEV, cfg=cfg, diagnostics=diag), f,
                      indent=2, default=str)
    print(f"[single] {cfg['dimension']} s={cfg['s']} Omega={cfg['Omega']} beta2={cfg['beta2']} "
          f"beta3={cfg['beta3']} G_C={cfg['G_C']} kernel={G['kernel']}")
    print(f"         E={diag['E']:.8f} mu={diag['mu']:.6f} Lz={diag['Lz']:.5f} Nv={diag['Nv']} "
          f"R90={diag['R90']:.4f} virial_rel={diag['virial_rel']:.2e}")
    print(f"         resid={diag['resid_rel']:.2e} converged={diag['converged']} it={diag['iters']}")
    return diag


# ---------------------------------------------------------------------- sweep
def _sweep_param(cfg):
    param = canonical_key(cfg.get("sweep_param", "G_C"))
    tmpl = CFG_DEFAULTS.get(param)
    if param not in CFG_DEFAULTS or isinstance(tmpl, bool) or not isinstance(tmpl, (int, float)):
        numeric = sorted(k for k, v in CFG_DEFAULTS.items()
                         if isinstance(v, (int, float)) and not isinstance(v, bool))
        raise ValueError(f"sweep_param={cfg.get('sweep_param')!r} is not a numeric CFG key; "
                         f"choose one of {numeric}")
    values = list(cfg.get("sweep_values", []))
    bad = [v for v in values if isinstance(v, bool) or not isinstance(v, (int, float))]
    if bad:
        raise ValueError(f"sweep_values must be numbers, got {bad}")
    return param, values


def _point_cfg(cfg, param, val):
    c = dict(cfg)
    c[param] = val
    if cfg.get("sweep_autobox", False):
        L, N, _ = auto_grid(c)
        c["L"], c["Ngrid"] = L, N
    c["tag"] = f"{cfg.get('tag', 'becgpp')}_{param}{val:g}"
    return c


def _fresh_candidates(points, grids, nseeds):
    """Fresh-seed solves of every point that needs them, as one batch per set of
    solver settings; per point the lowest-energy seed (multiseed selection)."""
    jobs = []                                           # (point index, seed cfg)
    for i, c in points:
        for cs in (seed_configs(c) if nseeds > 1 else [c]):
            jobs.append((i, cs))
    if not jobs:
        return {}
    # one batch per set of solver settings (a sweep over a solver key splits it)
    res = [None] * len(jobs)
    groups = {}
    for q, (_, cs) in enumerate(jobs):
        groups.setdefault(tuple(repr(cs.get(k)) for k in SOLVER_KEYS), []).append(q)
    for qs in groups.values():
        bs = BatchSolver([jobs[q][1] for q in qs], [grids[jobs[q][0]] for q in qs])
        try:
            for q, r in zip(qs, bs.solve([make_seed(grids[jobs[q][0]], jobs[q][1]) for q in qs])):
                res[q] = r
        finally:
            bs.close()
    out = {}
    for i, _ in points:
        mine = [(cs, r) for (j, cs), r in zip(jobs, res) if j == i]
        if nseeds > 1:
            psi, G, obs = select_lowest([cs for cs, _ in mine], [r for _, r in mine])
            out[i] = (f"seed:{obs.get('seed_used')}", psi, obs)
        else:
            cs, (psi, G, obs) = mine[0]
            out[i] = (f"seed:{cs.get('seed')}", psi, obs)
    return out


def mode_sweep(cfg):
    param, values = _sweep_param(cfg)
    use_cont = bool(cfg.get("sweep_continuation", True))
    nseeds = int(cfg.get("nseeds", 1))
    tag0 = cfg.get("tag", "becgpp")
    stem = param if tag0 == "becgpp" else f"{tag0}_{param}"
    print(f"SWEEP over {param!r} = {values}  (continuation={use_cont}, nseeds={nseeds})")
    if not values:
        print("[sweep] sweep_values is empty: nothing to do")
        return []
    cfgs = [_point_cfg(cfg, param, v) for v in values]
    grids = [make_grid(c) for c in cfgs]
    # points with a fresh-seed candidate: all of them with several seeds or no
    # continuation, else only the first (the others continue from their predecessor)
    fresh_at = [i for i in range(len(values)) if nseeds > 1 or not use_cont or i == 0]
    fresh = _fresh_candidates([(i, cfgs[i]) for i in fresh_at], grids, nseeds)
    out = _out_dir(cfg)
    rows, prev, G_prev = [], None, None
    for i, (val, c, G) in enumerate(zip(values, cfgs, grids)):
        cands = []
        if use_cont and prev is not None:
            same = tuple(prev.shape) == tuple(G["R2"].shape)
            psi0 = prev if same else resample_state(prev, G_prev, G)
            if psi0 is not None:
                psi_c, _, obs_c = ground_state(c, G=G, psi0=psi0, verbose=False)
                cands.append(("continuation", psi_c, obs_c))
        if i in fresh:
            cands.append(fresh[i])
        elif not cands:                                 # continuation impossible: fresh seed
            psi_s, _, obs_s = _solve_point(c, G)
            cands.append((f"seed:{obs_s.get('seed_used', c.get('seed'))}", psi_s, obs_s))
        cands.sort(key=lambda t: t[2]["E"])             # variational: lowest energy wins
        branch, psi, obs = cands[0]
        diag = diagnostics(psi, G, c)
        diag.update({param: val})
        diag.update(rid=run_id(c), resid_rel=obs["resid_rel"], iters=obs["iters"],
                    converged=obs["converged"], stop_reason=obs.get("stop_reason", ""),
                    walltime=sum(t[2]["walltime"] for t in cands), branch=branch,
                    candidate_E=";".join(f"{t[0]}={t[2]['E']:.10g}" for t in cands),
                    L=c["L"], N=c["Ngrid"], dimension=c["dimension"], kernel=G["kernel"])
        rows.append(diag)
        prev, G_prev = psi.detach(), G
        if out:
            if cfg.get("save_ckpt", True):
                torch.save(dict(psi=psi.cpu(), cfg=c, obs=diag), os.path.join(out, f"{diag['rid']}.pt"))
            write_csv(os.path.join(out, f"sweep_{stem}.csv"), rows)
        print(f"    {param}={val} [{branch}] E={diag['E']:.8f} mu={diag['mu']:.5f} "
              f"Nv={diag['Nv']} R90={diag['R90']:.4f} res={diag['resid_rel']:.2e} "
              f"conv={diag['converged']}")
    return rows


# ---------------------------------------------------------------- convergence
def mode_convergence(cfg):
    L0, N0 = float(cfg["L"]), int(cfg["Ngrid"])
    dx0 = 2.0 * L0 / N0
    pad0 = int(cfg.get("pad", 2))
    variants = [("grid", L0, int(N), pad0) for N in cfg.get("conv_Ngrids", [192, 256, 384])]
    for f in cfg.get("conv_box_factors", [1.0, 1.2]):
        L = L0 * f
        variants.append(("box", L, max(96, 32 * math.ceil((2 * L / dx0) / 32)), pad0))
    for pp in cfg.get("conv_pads", [2, 3]):
        variants.append(("pad", L0, N0, int(pp)))
    finest = max(cfg.get("conv_Ngrids", [256]))
    rows, seen, prev = [], set(), None
    out = _out_dir(cfg)
    for axis, L, N, pad in variants:
        key = (round(L, 10), N, pad)
        if key in seen:
            continue
        seen.add(key)
        c = dict(cfg, L=float(L), Ngrid=int(N), pad=int(pad),
                 tag=f"{cfg.get('tag', 'becgpp')}_{axis}_N{N}_p{pad}")
        G = make_grid(c)
        psi0 = prev if (prev is not None and tuple(prev.shape) == tuple(G["R2"].shape)) else None
        psi, G, obs = ground_state(c, G=G, psi0=psi0, verbose=False)
        d = diagnostics(psi, G, c)
        d.update(axis=axis, L=L, N=N, pad=pad, dx=G["dx"], resid_rel=obs["resid_rel"],
                 iters=obs["iters"], converged=obs["converged"], points_per_R90=d["R90"] / G["dx"])
        rows.append(d)
        if axis == "grid" and N == finest:
            prev = psi.detach()
        if out:
            write_csv(os.path.join(out, "convergence.csv"), rows)
        print(f"    {axis} L={L:.4g} N={N} p={pad}: E={d['E']:.9g} R90={d['R90']:.6g} "
              f"vir={d['virial_rel']:.2e} res={d['resid_rel']:.2e}")
    return rows


# -------------------------------------------------------------------- tf_only
def mode_tf_only(cfg):
    G = make_grid(cfg)
    tf = extract_tf(cfg, G)
    if tf is None:
        print("[tf_only] no TF reference for these parameters")
        return None
    out = _out_dir(cfg)
    if out:
        write_csv(os.path.join(out, "tf_only.csv"),
                  [dict(rid=run_id(cfg) + "_tf", kind=tf.get("kind"), R90=tf.get("R90"),
                        R99=tf.get("R99"), mu=tf.get("mu"), rho0=tf.get("rho0", float("nan")))])
    print(f"[tf_only] kind={tf.get('kind')} R90={tf.get('R90'):.4f} mu={tf.get('mu'):.5f} "
          f"converged={tf.get('converged')}")
    return tf


# ---------------------------------------------------------------------- smoke
def mode_smoke(cfg):
    """A small single run and the TF reference in the configured geometry (the
    reference's smoke mode minus its analytic validation gate)."""
    small = dict(cfg, L=10.0, Ngrid=(128 if geometry(cfg)[0] == 2 else 72), maxit=1500, res_tol=3e-3,
                 nseeds=1, want_lll=True, tag="smoke")
    d = mode_single(small)
    mode_tf_only(small)
    ok = bool(d) and bool(d.get("converged", False))
    print(f"[smoke] run_converged={ok}")
    return dict(gate=None, run=d, ok=ok)


DISPATCH = dict(smoke=mode_smoke, single=mode_single, tf_only=mode_tf_only, sweep=mode_sweep,
                convergence=mode_convergence)


def run(cfg):
    """Dispatch a configuration to its mode and return the result."""
    mode = cfg.get("mode", "smoke")
    if mode == "validate":
        raise ValueError("mode 'validate' (the reference's analytic validation gate) is not part "
                         f"of this package; choose {sorted(DISPATCH)}")
    fn = DISPATCH.get(mode)
    if fn is None:
        raise ValueError(f"unknown mode {mode!r}; choose {sorted(DISPATCH)}")
    kkind = resolve_kernel(cfg)[0]
    requested = str(cfg.get("kernel", "auto")).lower()
    if requested in ("newton", "log") and kkind == "none" and abs(float(cfg.get("G_C", 0.0))) <= 1e-15:
        print(f"[warn] kernel={requested!r} is set but G_C=0, so the long-range term is OFF "
              f"(reported kernel='none'). Set G_C>0 to activate it.")
    print(f"becgpp_b200 {CODE_VERSION} | device={DEV} | mode={mode} | "
          f"dim={cfg.get('dimension')} kernel={kkind}")
    return fn(cfg)
