"""Parity of the device-resident solver with the reference's ground states on
the same seeds.

E, mu, L_z and virial_rel are held to 1e-10 relative (max(1, |q|)) and the stop
reason must be equal, with exceptions named below. Near res_tol the reference
algorithm's outcome is decided by round-off: the energy decrease of a step is
below one ulp of E, so each Armijo decision is a coin flip. Two consequences,
measured on the reference itself:
  * the stop reason: over 40 seeded variants of the 2D harmonic configuration
    the reference ends 'converged' 21 times and 'line_search_stalled' 19 times
    (tests/golden/stop_stats.json); the test below compares that distribution;
  * first-order quantities (mu, virial_rel) of two runs that stop at different
    iterates of residual r differ by O(r). E is second order and stays within
    1e-10 everywhere. The named floor cases hold mu / virial_rel to
    1e-10 + 5 (r_ours + r_ref) (measured worst: 2.9 (r_ours + r_ref)); the CPU
    restatement of the algorithm (the oracle)
    shows the same gaps against the reference on the same cases."""
import json
import os

import numpy as np
import pytest
import torch

from becgpp_b200 import BatchSolver, default_cfg, ground_state, ground_state_multiseed, make_grid, make_seed

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

ALL = ("free2d", "free_soft", "free_rot", "maxit5", "harm48", "cq_rot48", "log2d48", "q2d48", "none48",
       "quartic32", "newton3d24", "free3d", "newton2d48", "pr48", "stall")
# cases whose stop reason is decided at the floor (one of the two runs ends within
# 10x of res_tol on the other side of it)
STOP_FLOOR = ("none48", "pr48", "q2d48", "quartic32")
# cases whose mu / virial_rel differ from the reference by more than 1e-10 (first-order
# quantities, as accurate as the residual: newton3d24 stops at res_tol = 1e-7)
MU_FLOOR = ("none48", "pr48", "q2d48", "quartic32", "newton3d24")
VIR_FLOOR = ("free2d", "free3d", "none48", "pr48", "q2d48", "quartic32", "stall", "newton3d24")


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def _solve(golden, name):
    arr, meta = golden("solves")
    m = meta[name]
    c = default_cfg(mode="single", **m["cfg"])
    psi, G, obs = ground_state(c, psi0=torch.as_tensor(arr[f"{name}/psi0"]).cuda(), verbose=False)
    return m, obs, psi, arr


@pytest.mark.parametrize("name", ALL)
def test_solve_matches_reference(golden, name):
    m, obs, psi, arr = _solve(golden, name)
    ref = m["obs"]
    assert _rel(obs["E"], ref["E"]) <= 1e-10, (obs["E"], ref["E"])
    assert _rel(obs["Lz"], ref["Lz"]) <= 1e-10, (obs["Lz"], ref["Lz"])
    floor = 1e-10 + 5.0 * (obs["resid_rel"] + ref["resid_rel"])
    assert _rel(obs["mu"], ref["mu"]) <= (floor if name in MU_FLOOR else 1e-10), (obs["mu"], ref["mu"])
    assert _rel(obs["virial_rel"], ref["virial_rel"]) <= (floor if name in VIR_FLOOR else 1e-10), (
        obs["virial_rel"], ref["virial_rel"])
    if name in STOP_FLOOR:
        tol = float(m["cfg"].get("res_tol", 1e-8))
        assert obs["stop_reason"] in ("converged", "line_search_stalled")
        assert obs["resid_rel"] < 10 * tol and ref["resid_rel"] < 10 * tol
    else:
        assert obs["stop_reason"] == m["stop_reason"], (obs["stop_reason"], m["stop_reason"])
    if name == "maxit5":
        assert obs["iters"] == 5


def test_stop_reason_distribution_matches_reference():
    """40 seeded variants of c1 (2D harmonic trap, beta2=100, N=128, L=16): every
    energy within 1e-10 of the reference's for the same seed, and the fraction of
    'converged' stops within 0.3 of the reference's (21 of 40; a 3-sigma band for
    two binomial samples of 40)."""
    from becgpp_b200.workloads import c1
    st = json.load(open(os.path.join(GOLD, "stop_stats.json")))
    conv = 0
    for row in st["rows"]:
        c = default_cfg(**dict(c1()[0]["cfg"], rng=row["rng"]))
        G = make_grid(c)
        _, _, obs = ground_state(c, G=G, psi0=make_seed(G, c), verbose=False)
        assert _rel(obs["E"], row["E"]) <= 1e-10, (row["rng"], obs["E"], row["E"])
        assert obs["stop_reason"] in ("converged", "line_search_stalled"), obs["stop_reason"]
        conv += obs["stop_reason"] == "converged"
    ref_conv = sum(r["stop_reason"] == "converged" for r in st["rows"])
    n = len(st["rows"])
    assert abs(conv - ref_conv) / n <= 0.3, (conv, ref_conv, n)


@pytest.mark.parametrize("name", ("c1", "c5"))
def test_benchmark_configuration_matches_reference(name):
    """The single-instance benchmark configurations at full size against the
    reference's own CPU run (tests/golden/baseline_runs.json): c1 2D harmonic
    128^2, c5 quasi-2D rotating pancake 256^2 (q2d kernel, l_z=0.5, Omega=0.3)."""
    from becgpp_b200.workloads import WORKLOADS
    p = WORKLOADS[name]()[0]
    ref = json.load(open(os.path.join(GOLD, "baseline_runs.json")))[p["name"]]
    r = ref["obs"]
    c = default_cfg(**p["cfg"])
    G = make_grid(c)
    _, _, obs = ground_state(c, G=G, psi0=make_seed(G, c), verbose=False)
    assert _rel(obs["E"], r["E"]) <= 1e-10, (obs["E"], r["E"])
    assert _rel(obs["Lz"], r["Lz"]) <= 1e-10 + 5.0 * (obs["resid_rel"] + r["resid_rel"]), (obs["Lz"], r["Lz"])
    floor = 1e-10 + 5.0 * (obs["resid_rel"] + r["resid_rel"])
    assert _rel(obs["mu"], r["mu"]) <= floor, (obs["mu"], r["mu"])
    assert _rel(obs["virial_rel"], r["virial_rel"]) <= floor, (obs["virial_rel"], r["virial_rel"])
    # both end at the floor (residual within 10x of res_tol): converged or stalled there
    assert obs["stop_reason"] in ("converged", "line_search_stalled")
    assert obs["resid_rel"] < 10 * float(c["res_tol"]) and r["resid_rel"] < 10 * float(c["res_tol"])


def test_droplet_stall_like_the_reference(golden):
    """The 64^2 cubic-quintic droplet (beta2=-200, beta3=1e3, Gaussian seed): the
    reference's line search stalls at residual 1.5e-3, so its energy is not a
    converged ground state and no 1e-10 comparison applies. The solve must stall
    the same way, at the same plateau (energy within 1e-5, residual of the same
    order), never report convergence."""
    m, obs, psi, arr = _solve(golden, "droplet64")
    ref = m["obs"]
    assert obs["stop_reason"] == m["stop_reason"] == "line_search_stalled"
    assert _rel(obs["E"], ref["E"]) <= 1e-5, (obs["E"], ref["E"])
    assert 0.1 * ref["resid_rel"] < obs["resid_rel"] < 10 * ref["resid_rel"]
    assert not obs["converged"]


@pytest.mark.parametrize("name,exact", [("free2d", 1.0), ("free3d", 1.5), ("free_soft", 0.5),
                                        ("free_rot", 1.0)])
def test_noninteracting_known_answers(golden, name, exact):
    _, obs, _, _ = _solve(golden, name)
    assert abs(obs["E"] - exact) < 1e-7


def test_stall_exit(golden):
    # becgpp tests/test_audit.py:165-172
    _, obs, _, _ = _solve(golden, "stall")
    assert abs(obs["E"] - 1.0) < 1e-10
    assert obs["stop_reason"] in ("line_search_stalled", "energy_converged")
    assert obs["iters"] < 400


def test_batch_equals_single(golden):
    arr, meta = golden("solves")
    names = ("harm48", "q2d48", "quartic32", "log2d48")
    cfgs = [default_cfg(mode="single", **meta[n]["cfg"]) for n in names]
    bs = BatchSolver(cfgs)
    res = bs.solve([torch.as_tensor(arr[f"{n}/psi0"]).cuda() for n in names])
    bs.close()
    for n, (psi, G, obs) in zip(names, res):
        ref = meta[n]["obs"]["E"]
        assert _rel(obs["E"], ref) <= 1e-10, n


def test_multiseed_picks_lowest_energy():
    c = default_cfg(mode="single", dimension="2D", beta2=50, L=6, Ngrid=48, nseeds=2, res_tol=1e-8,
                    maxit=3000)
    psi, G, obs = ground_state_multiseed(c)
    Es = [float(e) for e in obs["seed_energies"].split(";")]
    assert abs(obs["E"] - min(Es)) <= 1e-9 * abs(min(Es))
    assert obs["seed_used"] in ("tf", "gaussian")


def test_multiseed_verbose_prints_summary(capsys):
    # becgpp modes.py:224 calls ground_state_multiseed with verbose=True
    c = default_cfg(mode="single", dimension="2D", beta2=50, L=6, Ngrid=48, nseeds=2, res_tol=1e-8,
                    maxit=3000)
    _, _, obs = ground_state_multiseed(c, verbose=True)
    out = capsys.readouterr().out
    assert "2 seeds" in out and obs["seed_used"] in out


def test_trace_is_monotone(golden):
    arr, meta = golden("solves")
    c = default_cfg(mode="single", record_trace=True, **meta["harm48"]["cfg"])
    _, _, obs = ground_state(c, psi0=torch.as_tensor(arr["harm48/psi0"]).cuda(), verbose=False)
    E = np.array([t[2] for t in obs["trace"]])
    assert len(E) >= 2 and np.all(np.diff(E) <= 1e-12)


def test_schedule_autotuner_picks_a_candidate_and_keeps_results(golden):
    # three batched solves try the relaunch schedules; the fourth uses the fastest and
    # returns the same energies (the schedule changes team sizes, not the arithmetic
    # of any instance's solve)
    arr, meta = golden("solves")
    names = ("harm48", "q2d48", "quartic32", "log2d48")
    cfgs = [default_cfg(mode="single", **meta[n]["cfg"]) for n in names]
    bs = BatchSolver(cfgs, autotune=True)
    psi0 = [torch.as_tensor(arr[f"{n}/psi0"]).cuda() for n in names]
    for k in range(4):
        res = bs.solve(psi0)
        assert bs.schedule()["tuned"] == (k >= 2)
    sched = bs.schedule()
    bs.close()
    assert sched["yield_div"] in (2, 4, 8) and all(ms > 0 for ms in sched["candidate_ms"])
    for n, (psi, G, obs) in zip(names, res):
        ref = meta[n]["obs"]["E"]
        assert _rel(obs["E"], ref) <= 1e-10, n


@pytest.mark.parametrize("maxit", [7, 20, 45])
def test_quartic_line_search_energy_equals_direct_energy(golden, maxit):
    # 3D with a long-range kernel: the solver's energy of its last accepted state is
    # assembled from the quartic in the step (two convolutions per iteration, the
    # accepted potential from its parts, refreshed every 32 accepted steps); the
    # final pass recomputes the energy of the returned state with its own convolution
    arr, meta = golden("solves")
    m = meta["newton3d24"]
    c = default_cfg(mode="single", **dict(m["cfg"], maxit=maxit))
    bs = BatchSolver([c])
    _, res, _ = bs.solve_raw([torch.as_tensor(arr["newton3d24/psi0"]).cuda()])
    bs.close()
    r = res[0]
    assert r.status == 0
    if r.best_is_final:
        pytest.skip("the lowest-residual iterate is not the last accepted one")
    assert abs(r.E - r.E_final) <= 1e-13 * abs(r.E_final), (r.E, r.E_final)


def test_batch_with_3d_long_range_instances_matches_reference(golden):
    # 3D long-range instances (quartic line search) from the reference's seed and from
    # perturbed copies of it: they finish at different iterations, so the launch
    # yields and relaunches the unfinished ones with their control state and
    # potentials kept on the device; each reaches the reference's ground state
    arr, meta = golden("solves")
    m = meta["newton3d24"]
    c = default_cfg(mode="single", **m["cfg"])
    psi0 = torch.as_tensor(arr["newton3d24/psi0"])
    g = torch.Generator().manual_seed(11)
    seeds = [psi0] + [psi0 * (1.0 + a * torch.rand(psi0.shape, generator=g, dtype=torch.float64))
                      for a in (0.05, 0.2, 0.5)]
    bs = BatchSolver([c] * len(seeds))
    res = bs.solve([s.cuda() for s in seeds])
    bs.close()
    iters = [obs["iters"] for _, _, obs in res]
    assert len(set(iters)) > 1, iters
    for psi, G, obs in res:
        assert _rel(obs["E"], m["obs"]["E"]) <= 1e-10, (obs["E"], m["obs"]["E"], iters)


@pytest.mark.parametrize("name,precision", [("harm48", "fp64"), ("cq_rot48", "mixed"), ("newton3d24", "fp64")])
def test_single_solve_is_bitwise_reproducible(golden, name, precision):
    # one instance per launch (no relaunch vote): every reduction adds its partials in
    # a fixed order, so two solves of the same input give the same bits
    arr, meta = golden("solves")
    c = default_cfg(mode="single", precision=precision, **meta[name]["cfg"])
    psi0 = torch.as_tensor(arr[f"{name}/psi0"]).cuda()
    runs = [ground_state(c, psi0=psi0, verbose=False) for _ in range(2)]
    (p1, _, o1), (p2, _, o2) = runs
    assert o1["iters"] == o2["iters"] and o1["E"] == o2["E"] and o1["resid_rel"] == o2["resid_rel"]
    assert torch.equal(p1, p2)
