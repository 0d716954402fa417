"""Benchmark: converged ground states per second on one B200 (or N GPUs).

Workload (default ``c4``): the batched cubic-quintic droplet sweep, 64
instances (beta2 in linspace(-400,-50,16) x 4 seeds, beta3 = 1e3, L = 20, grids
128^2 and 256^2) solved together in one persistent launch sequence. A ground
state counts when the reference's own run of that instance converged
(resid_rel <= 1e-6) and our returned state's energy agrees with it to
|dE/E| <= 1e-10; the reference energies are the committed fixture
tests/golden/baseline_runs.json. The line's `accuracy` object lists every
instance (|dE/E|, residual, stop reason, iterations) and why each miss missed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed.run: the instances are partitioned over the
ranks (strong scaling: the total work is the fixed workload), each rank solves
its share alone with no collective on the data path; value = all ranks' counted
ground states / the slowest rank's time.

--impl reference times the CPU restatement of the reference's algorithm (the
oracle) on the host cores over the whole workload: its K steps partition the
instances, so together they solve every instance once.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

E_TOL = 1e-10
# DRAM bytes per algorithmic byte of the solver, per precision, from one ncu capture
# of `bench.py --case small-solve --instances 8 --maxit 200 [--precision fp64]`
# (dram__bytes_read.sum + dram__bytes_write.sum of all its solver launches / its
# algorithmic bytes): the working set lives in L2, so only a fifth to a quarter of
# the algorithmic bytes reach DRAM.
TRAFFIC_PER_ALGO_BYTE = {"fp64": 0.239, "mixed": 0.178}
ORACLE_RESID_MAX = 1e-6
METRIC = "ground states/s at |dE/E|<=1e-10 (batched solve)"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="c4")
    ap.add_argument("--cpu-sample", type=int, default=6, help="instances in the CPU baseline sample")
    ap.add_argument("--case", default="bench", choices=("bench", "hpsi", "hpsi-once", "small-solve", "phases",
                                                        "configs"),
                    help="bench: the full measurement; hpsi: H psi rates only; small-solve: one "
                         "short batched solve (for profiler captures); phases: per-phase time "
                         "breakdown with the profiling build (python -m becgpp_b200.build --profile); "
                         "hpsi-once: the 64-instance batched apply and the 3D 128^3 newton apply, a few "
                         "plain calls each (for profiler captures); "
                         "configs: each single-instance configuration against the reference's CPU run")
    ap.add_argument("--instances", type=int, default=8, help="small-solve: instances of the workload")
    ap.add_argument("--maxit", type=int, default=200, help="small-solve: iteration cap")
    ap.add_argument("--grid", type=int, default=0, help="small-solve: only instances of this N")
    ap.add_argument("--precision", default="mixed", choices=("mixed", "fp64"),
                    help="precision of the batched solve; the other precision is measured beside "
                         "it, and the plain arm (one instance at a time) is always FP64")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (c1, c5, c3, c2 in FP64 and mixed)")
    ap.add_argument("--hpsi-workloads", default="c3,c2,c4,c1,c5",
                    help="hpsi: comma-separated workloads whose grids are timed")
    ap.add_argument("--reps", type=int, default=3, help="hpsi: graph replays per grid")
    ap.add_argument("--hpsi-batch", type=int, default=1, help="hpsi: also time the 64-instance batched apply")
    ap.add_argument("--hpsi-sched", default="", help="hpsi-once: fixed schedule 'lines,order,conv_lines,conv_order[,strided_conv_lines]'")
    return ap.parse_args()


def workload_desc(name):
    return f"{name}: batched droplet sweep, 64 instances 128^2/256^2" if name == "c4" else name


def job_rate(total_s, counted, dist=None, device="cpu"):
    """Whole-job rate over the ranks: (max over ranks of the timed seconds, sum
    over ranks of the counted ground states, their ratio). Every rank must call
    it at the same point (two all-reduces)."""
    import torch
    if dist is None:
        return total_s, float(counted), (counted / total_s if total_s > 0 else 0.0)
    t = torch.tensor([total_s, float(counted)], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    tm, c = float(tmax[0]), float(t[1])
    return tm, c, (c / tm if tm > 0 else 0.0)


def _reference_runs():
    return json.load(open(os.path.join(ROOT, "tests", "golden", "baseline_runs.json")))


def _instances(workload):
    from becgpp_b200.workloads import WORKLOADS
    return WORKLOADS[workload]()


def _counts(names, energies, ref):
    """(counted, eligible): instances matching a converged reference energy."""
    counted = eligible = 0
    for n, e in zip(names, energies):
        r = ref.get(n)
        if r is None or r["obs"]["resid_rel"] > ORACLE_RESID_MAX:
            continue
        eligible += 1
        if abs(e - r["obs"]["E"]) <= E_TOL * abs(r["obs"]["E"]):
            counted += 1
    return counted, eligible


def instance_rows(names, res, grids, ref):
    """Per-instance accuracy of one solve of the workload against the
    reference's own CPU run: [name, N, |dE/E|, our resid_rel, our stop, our
    iterations, reference resid_rel, counted]. |dE/E| and the residual are those
    of the returned state (evaluated afresh on the device)."""
    from becgpp_b200._lib import STOP_NAMES
    rows = []
    for n, r, G in zip(names, res, grids):
        rr = ref.get(n)
        e_ref = rr["obs"]["E"] if rr else float("nan")
        d = abs(r.E_final - e_ref) / abs(e_ref) if rr else float("nan")
        elig = bool(rr) and rr["obs"]["resid_rel"] <= ORACLE_RESID_MAX
        rows.append([n, G["N"], float(f"{d:.3g}"), float(f"{r.resid_rel_final:.3g}"),
                     STOP_NAMES[int(r.stop_reason)], int(r.iters),
                     float(f"{rr['obs']['resid_rel']:.3g}") if rr else None, int(elig and d <= E_TOL)])
    return rows


def miss_reasons(rows, oracle_runs=None):
    """Why each instance the reference converged was not counted: 'stalled' when
    our solve stopped with its residual above the eligibility bar (a premature
    line-search stall, the reference algorithm's own failure mode), else
    'other state' (a stationary state with a different energy). `oracle` says
    whether the CPU restatement of the same algorithm missed it as well."""
    out = {}
    for n, _, d, res, stop, it, rres, ok in rows:
        if ok or rres is None or rres > ORACLE_RESID_MAX:
            continue
        why = "stalled" if res > ORACLE_RESID_MAX else "other state"
        m = {"reason": why, "dE_rel": d, "resid": res, "stop": stop, "iters": it, "ref_resid": rres}
        if oracle_runs and n in oracle_runs:
            o = oracle_runs[n]
            m["oracle_missed"] = not _matches(n, o["E"])
        out[n] = m
    return out


_REF_CACHE = {}


def _matches(name, E):
    ref = _REF_CACHE.setdefault("r", _reference_runs())
    r = ref[name]["obs"]
    return abs(E - r["E"]) <= E_TOL * abs(r["E"])


def _oracle_runs():
    """The oracle's own solves of the workloads (tests/golden/oracle_runs.json),
    or None when the fixture is absent."""
    try:
        return json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_runs.json")))
    except OSError:
        return None


def partition(insts, ref, world, rank):
    """Instances of this rank: the list dealt over the ranks by descending cost
    (greedy, to the least loaded rank), so the long instances land on different
    GPUs. No exchange between ranks: each solves its share alone."""
    load = [0.0] * world
    mine = []
    for i, p in sorted(enumerate(insts), key=lambda q: -_cost(q[1], ref)):
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += _cost(p, ref)
        if r == rank:
            mine.append(i)
    return sorted(mine)


class Clocks:
    """Sample SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        import statistics
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------------- CPU baseline
def _oracle_solve(p):
    """One instance solved by the oracle (the reference's algorithm restated in
    numpy/scipy FP64) in a worker process with one host thread. Runs in a
    `spawn` pool: it never touches the GPU."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import gpp as O
    from becgpp_b200.config import default_cfg
    from becgpp_b200.seeds import make_seed, phase_noise
    O.WORKERS = 1
    c = default_cfg(**p["cfg"])
    if p.get("maxit") is not None:
        c = dict(c, maxit=p["maxit"])
    G = O.make_grid(c)
    Gd = dict(ndim=G["ndim"], N=G["N"], L=G["L"], s=G["s"], trap_coeff=G["trap_coeff"],
              kernel=G["kernel"], pad=G["pad"], l_z=G["l_z"], dx=G["dx"])
    s = make_seed(Gd, c, device="cpu")
    if p.get("phase_noise"):
        s = phase_noise(s, p["phase_noise"], p["phase_seed"])
    t0, c0 = time.perf_counter(), time.process_time()
    _, obs = O.ground_state(c, s.numpy())
    return dict(name=p["name"], E=obs["E"], resid=obs["resid_rel"], stop=obs["stop_reason"],
                iters=obs["iters"], wall_s=time.perf_counter() - t0, cpu_s=time.process_time() - c0)


def _cost(p, ref):
    """Expected cost of an instance: the reference's iterations x grid points."""
    r = ref.get(p["name"])
    it = r["obs"]["iters"] if r else int(p["cfg"].get("maxit", 1000))
    return it * int(p["cfg"]["Ngrid"]) ** (3 if p["cfg"].get("dimension") == "3D" else 2)


def rotation_groups(insts, ref, steps, procs):
    """Partition the workload into `steps` groups that together cover every
    instance once: the `procs` costliest instances (the long tail) form the first
    group, so they run side by side; the rest are dealt out by descending cost."""
    order = sorted(insts, key=lambda p: -_cost(p, ref))
    k = max(1, min(steps, len(order)))
    groups = [order[:procs]] + [[] for _ in range(k - 1)]
    for j, p in enumerate(order[procs:]):
        groups[1 + j % (k - 1) if k > 1 else 0].append(p)
    return [g for g in groups if g]


def cpu_baseline(insts, ref, sample, procs=None):
    """The oracle on a bounded sample of the workload: `sample` of the instances
    the reference converged, at evenly spaced ranks of their cost, one worker
    process per instance. It leaves out the time of the instances that can
    never count, so it reads high; the reference arm times the whole workload."""
    import multiprocessing as mp
    elig = sorted([p for p in insts if ref.get(p["name"]) and ref[p["name"]]["obs"]["resid_rel"] <= ORACLE_RESID_MAX],
                  key=lambda p: _cost(p, ref))
    sample = max(1, min(sample, len(elig)))
    picked = [elig[(j * len(elig)) // sample] for j in range(sample)]
    procs = procs or min(len(picked), os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(procs) as pool:
        t0 = time.perf_counter()
        rows = pool.map(_oracle_solve, picked)
        wall = time.perf_counter() - t0
    counted, _ = _counts([r["name"] for r in rows], [r["E"] for r in rows], ref)
    return dict(value=counted / wall, wall_s=wall, counted=counted, solves=len(rows), cores=procs,
                names=[p["name"] for p in picked])


def run_reference(a):
    """The reference arm: the reference's algorithm (the oracle port; becGPP is
    Python and cannot travel) on the host cores, over the WHOLE workload: the K
    timed steps partition the instances (rotation_groups), so together they
    solve every instance once, and each step runs its group in a process pool
    over all host cores. rate = counted / sum of the step times."""
    import multiprocessing as mp
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    insts = _instances(a.workload)
    ref = _reference_runs()
    procs = os.cpu_count() or 1
    groups = rotation_groups(insts, ref, a.steps, procs)
    with mp.get_context("spawn").Pool(procs) as pool:
        # warm-up: start every worker and import its modules on a tiny solve
        tiny = dict(insts[0], maxit=2)
        for _ in range(a.warmup):
            pool.map(_oracle_solve, [tiny] * procs)
        walls, rows = [], []
        for g in groups:
            t0 = time.perf_counter()
            rows.extend(pool.map(_oracle_solve, g))
            walls.append(time.perf_counter() - t0)
    counted, eligible = _counts([r["name"] for r in rows], [r["E"] for r in rows], ref)
    tot = sum(walls)
    value = counted / tot if tot > 0 else 0.0
    cpu = sum(r["cpu_s"] for r in rows)
    sample = (f"rotation over the whole workload: {len(rows)} instances in {len(groups)} steps "
              f"(step 1: the {len(groups[0])} costliest side by side, the rest dealt by cost), "
              f"oracle port, {procs} worker processes x 1 thread; "
              f"rate = counted / sum of step times")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "ground states/s",
            "n_gpus": a.gpus, "steps": len(groups), "warmup": a.warmup,
            "ms_per_step": 1e3 * tot / len(groups), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded workload instances)",
            "config": {"workload": workload_desc(a.workload), "precision": "fp64",
                       "instances": len(insts), "instances_solved": len(rows),
                       "eligible": eligible, "counted": counted,
                       "parallelism": f"{procs} host processes"},
            "cpu_baseline": {"value": value, "unit": "ground states/s", "cores": procs,
                             "kind": "port", "sample": sample,
                             "cpu_seconds": cpu, "rate_per_cpu_second_x_cores": counted / cpu * procs if cpu else None},
            "e2e": {"value": value, "unit": "ground states/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def algorithmic_bytes(ndim, n, iters, naccept, ntrials, fp32_iters=0):
    """Compulsory bytes of one instance's solve in the fused design: per
    accepted iteration the H psi passes (read psi twice, A once, write A and H),
    the gradient pass (read H, psi; write g, the transformed g and the median
    keys), three median key scans, the preconditioner passes (2D: 2, 3D: 4, each
    reading and writing one field, the last also reading psi), the direction
    pass (7 fields read, z written) and per trial the state pass (first trial
    reads z, dir, g, psi and writes dirc, w; later ones read dirc, psi and write
    w) plus one read of w per remaining axis. Solver fields are complex128 (16
    bytes a point), complex64 (8) in the first `fp32_iters` iterations of the
    mixed form; accepted steps and trials are apportioned by iterations."""
    def total(S):
        d = ndim
        resid = S * n * (2 + (d - 1) * 3 + 1) + S * n * 4 + 8.0 * n
        median = 3 * 8.0 * n
        precond = S * n * (2 * (1 if d == 2 else 3) + 3)
        direction = S * n * 8
        first_trial = S * n * (4 + 2) + S * n * (d - 1)
        later_trial = S * n * 3 + S * n * (d - 1)
        per_iter = median + precond + direction
        return (iters * per_iter + naccept * resid + iters * first_trial
                + max(ntrials - iters, 0) * later_trial)
    f32 = min(max(fp32_iters, 0), iters) / iters if iters > 0 else 0.0
    return f32 * total(8.0) + (1.0 - f32) * total(16.0)


def fp32_iterations(r):
    """Iterations a solve ran with complex64 fields (fp64_from: -1 never handed
    over, 0 FP64 throughout)."""
    return int(r.iters) if int(r.fp64_from) < 0 else int(r.fp64_from)


def hpsi_bytes(G):
    """Compulsory bytes of one H psi: read psi, write H psi (complex128), and with a
    long-range kernel read the real FP64 half-spectrum of the kernel once."""
    n = G["N"] ** G["ndim"]
    b = 2 * 16 * n
    if G["kernel"] != "none":
        M = G["pad"] * G["N"]
        b += 8 * M ** (G["ndim"] - 1) * (M // 2 + 1)
    return b


def _graph_time(fn, reps=3):
    """Device seconds of one call of fn (enqueues GPU work only): fn captured once in
    a CUDA graph, the graph replayed `reps` times between CUDA events."""
    import torch
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def hpsi_rates(workloads=("c3", "c2", "c4", "c1", "c5"), reps=3, peak=None, batched=True):
    """H psi device time per apply through the batched entry point (stream
    passes, autotuned schedule), potential computed from |psi|^2 when the kernel
    is on: one apply per distinct grid of each workload, and the whole droplet
    sweep (64 instances, 128^2 and 256^2) in one batched apply. Each timed apply
    works on its own buffers, rotated through a set larger than L2 (256 MB), so
    inputs come from HBM; the applies of a set are one CUDA graph (no host time).
    Compulsory bytes: read psi, write H psi (complex128), read the kernel's real
    half-spectrum once."""
    import torch
    from becgpp_b200 import HamiltonianBatch, default_cfg, make_grid, make_seed
    out = {}

    def measure(name, cfgs, grids, psi0):
        hb = HamiltonianBatch(cfgs, grids)
        hb.apply(psi0)                                 # tunes the schedules of these grid sizes
        torch.cuda.synchronize()
        b = sum(hpsi_bytes(G) for G in grids)
        per = sum(2 * 16 * G["N"] ** G["ndim"] for G in grids)
        nbuf = max(1, min(512, -(-256 * 2 ** 20 // per)))
        ins = [[p.clone() for p in psi0] for _ in range(nbuf)]
        outs = [[torch.empty_like(p) for p in psi0] for _ in range(nbuf)]

        def run():
            for k in range(nbuf):
                hb.apply(ins[k], out=outs[k])
        t = _graph_time(run, reps) / nbuf
        sched = {f"{G['N']}": {k: v for k, v in hb.schedule(G["N"]).items() if k != "candidates_ms"}
                 for G in grids[:1] + [g for g in grids if g["N"] != grids[0]["N"]][:1]}
        hb.close()
        out[name] = {"us_per_apply": 1e6 * t, "compulsory_MB": b / 1e6, "GB_s": b / t / 1e9,
                     "frac_of_peak": (b / t / 1e9 / peak) if peak else None, "instances": len(grids),
                     "schedule": sched, "buffers_rotated": nbuf}
        print(name, out[name], file=sys.stderr, flush=True)

    for w in workloads:
        seen = set()
        for p in _instances(w):
            c = default_cfg(**p["cfg"])
            key = (c["dimension"], c["Ngrid"])
            if key in seen:
                continue
            seen.add(key)
            G = make_grid(c)
            name = f"{w}_{G['N']}^{G['ndim']}" + ("" if G["kernel"] == "none" else f"_{G['kernel']}")
            measure(name, [c], [G], [make_seed(G, c).contiguous()])
    if batched:
        cfgs = [default_cfg(**p["cfg"]) for p in _instances("c4")]
        grids = [make_grid(c) for c in cfgs]
        measure("c4_batch_64_instances", cfgs, grids, [make_seed(G, c).contiguous() for G, c in zip(grids, cfgs)])
    return out


PHASE_KINDS = {0: "max-reduction", 1: "H psi last axis", 2: "preconditioner last axis",
               5: "gradient + key and window counts", 13: "energy/trial axis or convolution end",
               15: "direction", 16: "barrier only", 17: "median selection"}


def phase_breakdown(plan, i, per):
    """Per phase kind: count per unit and mean microseconds of work, reduction
    commit, barrier wait and gather (profiling build only)."""
    import ctypes
    from becgpp_b200 import _lib
    buf = (ctypes.c_ulonglong * 100)()
    _lib.check(_lib.lib().bgp_prof_read(plan, i, buf, 1), "bgp_prof_read")
    out, tot = {}, 0
    c, t = buf[90], buf[91]
    if c:
        out["inside tile loops (part of work)"] = {"per_unit": c / per, "us_each": t / c / 1e3,
                                                   "us_per_unit": t / per / 1e3}
    for k in range(18):
        c, w, cm, sy, ga = buf[5 * k:5 * k + 5]
        if c == 0:
            continue
        tot += w + cm + sy + ga
        out[PHASE_KINDS.get(k, str(k))] = {
            "per_unit": c / per, "work_us": w / c / 1e3, "commit_us": cm / c / 1e3,
            "wait_us": sy / c / 1e3, "gather_us": ga / c / 1e3, "us_per_unit": (w + cm + sy + ga) / per / 1e3}
    return out, tot / per / 1e3


def run_configs(names=("c1", "c2", "c5", "c3")):
    """Each single-instance configuration solved alone, as the reference ran it
    (one ground_state call per instance): the device time of the first call (plan
    and kernel tables included, as the reference's time includes its table) and
    of a repeat, against the reference's CPU time and result on the same seed."""
    import time
    import torch
    from becgpp_b200 import default_cfg, ground_state, make_grid, make_seed
    from becgpp_b200.grid import clear_plans
    from becgpp_b200.interactions import clear_kernel_cache
    from becgpp_b200.seeds import phase_noise
    ref = _reference_runs()
    out = {}
    for w in names:
        for p in _instances(w):
            clear_plans()
            clear_kernel_cache()
            c = default_cfg(**p["cfg"])
            times = []
            for _ in range(2):
                torch.cuda.synchronize()
                t0 = time.time()
                G = make_grid(c)
                s0 = make_seed(G, c)
                if p.get("phase_noise"):
                    s0 = phase_noise(s0, p["phase_noise"], p["phase_seed"])
                psi, G, obs = ground_state(c, G=G, psi0=s0, verbose=False)
                torch.cuda.synchronize()
                times.append(time.time() - t0)
            r = ref.get(p["name"])
            out[p["name"]] = {
                "grid": f"{G['N']}^{G['ndim']} {G['kernel']}", "first_s": round(times[0], 4),
                "repeat_s": round(times[1], 4), "iters": obs["iters"], "stop": obs["stop_reason"],
                "E": obs["E"], "ref_s": r and round(r["wall_s"], 3), "ref_threads": r and r["threads"],
                "ref_iters": r and r["obs"]["iters"], "ref_stop": r and r["stop_reason"],
                "dE_rel": r and abs(obs["E"] - r["obs"]["E"]) / abs(r["obs"]["E"])}
            print(p["name"], out[p["name"]], flush=True, file=sys.stderr)
    return out


def config_results(names=("c1", "c5", "c3", "c2")):
    """The other benchmark configurations, each solved in FP64 and in the mixed
    form, the way `ground_state`/`ground_state_multiseed` run them: c1, c5 and c3
    alone, c2's three seeds (triangular, tf, gaussian, phase noise 1e-3) as one
    batch. Per result: device seconds, |dE/E| against the reference's own CPU run
    of the same seed, the returned state's residual, the stop reason, iterations
    and, for the mixed form, the iteration of the hand-over to FP64."""
    import torch
    from becgpp_b200 import BatchSolver, default_cfg, make_grid, make_seed
    from becgpp_b200._lib import STOP_NAMES
    from becgpp_b200.seeds import phase_noise
    ref = _reference_runs()
    out = {}
    for w in names:
        insts = _instances(w)
        for prec in ("fp64", "mixed"):
            cfgs = [default_cfg(**dict(p["cfg"], precision=prec)) for p in insts]
            grids = [make_grid(c) for c in cfgs]
            psi0 = []
            for p, c, G in zip(insts, cfgs, grids):
                s0 = make_seed(G, c)
                if p.get("phase_noise"):
                    s0 = phase_noise(s0, p["phase_noise"], p["phase_seed"])
                psi0.append(s0.contiguous())
            bs = BatchSolver(cfgs, grids)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            _, res, _ = bs.solve_raw(psi0)
            e1.record()
            torch.cuda.synchronize()
            secs = e0.elapsed_time(e1) / 1e3
            bs.close()
            rows = []
            for p, r in zip(insts, res):
                rr = ref.get(p["name"])
                rows.append({"instance": p["name"],
                             "dE_rel": float(f"{abs(r.E_final - rr['obs']['E']) / abs(rr['obs']['E']):.3g}"),
                             "resid_rel": float(f"{r.resid_rel_final:.3g}"), "stop": STOP_NAMES[int(r.stop_reason)],
                             "iters": int(r.iters), "fp64_from": int(r.fp64_from),
                             "ref_resid_rel": float(f"{rr['obs']['resid_rel']:.3g}"), "ref_stop": rr["stop_reason"],
                             "ref_cpu_s": round(rr["wall_s"], 2)})
            out[f"{w}_{prec}"] = {"seconds": round(secs, 4), "results": rows}
            print(w, prec, out[f"{w}_{prec}"], file=sys.stderr, flush=True)
    return out


def run_phases(a):
    import torch
    from becgpp_b200 import BatchSolver, default_cfg, make_grid, make_seed
    rep = {}
    insts = _instances("c4")
    for name in ("c4_b03_s0", "c4_b00_s1"):
        p = [q for q in insts if q["name"] == name][0]
        c = dict(default_cfg(**p["cfg"]), maxit=a.maxit)
        G = make_grid(c)
        psi0 = make_seed(G, c).contiguous()
        bs = BatchSolver([c], [G])
        bs.solve_raw([psi0])
        torch.cuda.synchronize()
        phase_breakdown(bs.plan.handle, 0, 1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, r, _ = bs.solve_raw([psi0])
        e1.record()
        torch.cuda.synchronize()
        it = r[0].iters
        br, tot = phase_breakdown(bs.plan.handle, 0, it)
        rep[f"solve {name} {G['N']}^2, per iteration"] = {
            "us_per_iter": 1e3 * e0.elapsed_time(e1) / it, "iters": it, "trials": r[0].ntrials,
            "accepted": r[0].naccepted, "phases_us_per_iter": tot, "phases": br}
        bs.close()
    # the tail of the sweep: the four 256^2 instances that run longest, together (the
    # profile is the first instance's; us_per_iter is the batch's time per iteration)
    tail = [q for q in insts if q["name"] in ("c4_b03_s0", "c4_b03_s1", "c4_b03_s2", "c4_b03_s3")]
    cs = [dict(default_cfg(**q["cfg"]), maxit=a.maxit) for q in tail]
    Gs = [make_grid(c) for c in cs]
    ps = [make_seed(G, c).contiguous() for G, c in zip(Gs, cs)]
    bs = BatchSolver(cs, Gs)
    bs.solve_raw(ps)
    torch.cuda.synchronize()
    phase_breakdown(bs.plan.handle, 0, 1)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    _, r, _ = bs.solve_raw(ps)
    e1.record()
    torch.cuda.synchronize()
    it = max(r[q].iters for q in range(len(tail)))
    br, tot = phase_breakdown(bs.plan.handle, 0, r[0].iters)
    rep["solve of the four c4_b03 instances together (256^2), per iteration"] = {
        "us_per_iter": 1e3 * e0.elapsed_time(e1) / it, "iters": it, "trials": r[0].ntrials,
        "accepted": r[0].naccepted, "phases_us_per_iter": tot, "phases": br}
    bs.close()
    # the 3D self-gravitating case: a few iterations in each precision
    for prec in ("fp64", "mixed"):
        c = dict(default_cfg(**_instances("c3")[0]["cfg"]), maxit=min(a.maxit, 40), precision=prec)
        G = make_grid(c)
        psi0 = make_seed(G, c).contiguous()
        bs = BatchSolver([c], [G])
        bs.solve_raw([psi0])
        torch.cuda.synchronize()
        phase_breakdown(bs.plan.handle, 0, 1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, r, _ = bs.solve_raw([psi0])
        e1.record()
        torch.cuda.synchronize()
        it = r[0].iters
        br, tot = phase_breakdown(bs.plan.handle, 0, it)
        rep[f"solve c3 128^3 newton ({prec}), per iteration"] = {
            "us_per_iter": 1e3 * e0.elapsed_time(e1) / it, "iters": it, "trials": r[0].ntrials,
            "accepted": r[0].naccepted, "phases_us_per_iter": tot, "phases": br}
        bs.close()
    print(json.dumps({"case": "phases", "report": rep}, indent=1), flush=True)


def run_case(a):
    """Single-purpose runs for profiler captures and the H psi table."""
    if a.case == "phases":
        prof_lib = os.path.join(ROOT, "becgpp_b200", "libbgp_prof.so")
        if not os.path.isfile(prof_lib):
            raise SystemExit("the phase profiler needs `python -m becgpp_b200.build --profile` first")
        os.environ["BECGPP_B200_LIB"] = prof_lib
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if a.case == "hpsi":
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except OSError:
            pass
        print(json.dumps({"case": "hpsi", "rates": hpsi_rates(tuple(a.hpsi_workloads.split(",")), a.reps,
                                                                   peak=peaks.get("hbm_gbs"),
                                                                   batched=bool(a.hpsi_batch))}), flush=True)
        return
    if a.case == "phases":
        run_phases(a)
        return
    if a.case == "hpsi-once":
        from becgpp_b200 import HamiltonianBatch, default_cfg, make_grid, make_seed
        for w in ("c4", "c3"):
            cfgs = [default_cfg(**p["cfg"]) for p in _instances(w)]
            grids = [make_grid(c) for c in cfgs]
            psi = [make_seed(G, c).contiguous() for G, c in zip(grids, cfgs)]
            hb = HamiltonianBatch(cfgs, grids)
            if a.hpsi_sched:
                # a fixed schedule (lines, radix order, conv lines, conv order[, strided
                # conv lines]): no tuning launches
                f = [int(x) for x in a.hpsi_sched.split(",")]
                csl = f[4] if len(f) > 4 else f[2]
                for N in sorted({G["N"] for G in grids}):
                    hb.set_schedule(N, f[0], f[1], f[2], f[3], conv_strided_lines=csl)
            for _ in range(a.reps):
                hb.apply(psi)
            torch.cuda.synchronize()
            hb.close()
        print(json.dumps({"case": "hpsi-once", "reps": a.reps}), flush=True)
        return
    if a.case == "configs":
        print(json.dumps({"case": "configs", "results": run_configs()}), flush=True)
        return
    from becgpp_b200 import BatchSolver, default_cfg, make_grid, make_seed
    insts = [p for p in _instances(a.workload) if not a.grid or int(p["cfg"]["Ngrid"]) == a.grid]
    insts = insts[: a.instances]
    cfgs = [dict(default_cfg(**p["cfg"]), maxit=a.maxit, precision=a.precision) for p in insts]
    grids = [make_grid(c) for c in cfgs]
    psi0s = [make_seed(G, c).contiguous() for G, c in zip(grids, cfgs)]
    bs = BatchSolver(cfgs, grids)
    _, res, _ = bs.solve_raw(psi0s)
    torch.cuda.synchronize()
    algo = sum(algorithmic_bytes(G["ndim"], G["N"] ** G["ndim"], r.iters, r.naccepted, r.ntrials,
                                 fp32_iterations(r)) for r, G in zip(res, grids))
    print(json.dumps({"case": "small-solve", "workload": a.workload, "precision": a.precision, "instances": len(insts),
                      "maxit": a.maxit, "iters": [r.iters for r in res],
                      "launches": bs.plan.launches, "algorithmic_bytes": algo}), flush=True)
    bs.close()


def fp64_comparison(insts, cfgs, grids, psi0s, names, ref, precision, value):
    """The same workload (1) batched in the other precision and (2) solved one
    instance at a time in FP64, the plain path: ground states/s of each, and the
    main arm's ratio to the plain path."""
    import torch
    from becgpp_b200 import BatchSolver

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1) / 1e3

    out = {}
    c64 = [dict(c, precision="fp64") for c in cfgs]
    other = "mixed" if precision == "fp64" else "fp64"
    co = [dict(c, precision=other) for c in cfgs]
    bs = BatchSolver(co, grids)
    bs.solve_raw(psi0s)
    (_, res, _), t = timed(lambda: bs.solve_raw(psi0s))
    bs.close()
    c, el = _counts(names, [r.E_final for r in res], ref)
    orc = _oracle_runs()
    out[f"batched_{other}"] = {"value": c / t, "seconds": t, "counted": c, "eligible": el,
                               "fp64_from_median": sorted(r.fp64_from for r in res)[len(res) // 2],
                               "misses": miss_reasons(instance_rows(names, res, grids, ref), orc)}
    total, counted = 0.0, 0
    plain_res = []
    for c, G, p0, n in zip(c64, grids, psi0s, names):
        bs = BatchSolver([c], [G])
        (_, res, _), t = timed(lambda: bs.solve_raw([p0]))
        bs.close()
        total += t
        counted += _counts([n], [res[0].E_final], ref)[0]
        plain_res.append(res[0])
    plain = counted / total
    out["plain_fp64"] = {"value": plain, "seconds": total, "counted": counted,
                         "how": "one instance per solve, sequentially, FP64",
                         "misses": miss_reasons(instance_rows(names, plain_res, grids, ref), orc)}
    out["value_over_plain_fp64"] = value / plain if plain > 0 else None
    return out


def run_ours(a):
    import torch
    from becgpp_b200 import BatchSolver, default_cfg, make_grid, make_seed
    from becgpp_b200.seeds import phase_noise

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    ref = _reference_runs()
    all_insts = _instances(a.workload)
    insts = [all_insts[i] for i in partition(all_insts, ref, world, rank)]
    cfgs = [default_cfg(**dict(p["cfg"], precision=a.precision)) for p in insts]
    grids = [make_grid(c) for c in cfgs]
    psi0s = []
    for p, c, G in zip(insts, cfgs, grids):
        s = make_seed(G, c)
        if p.get("phase_noise"):
            s = phase_noise(s, p["phase_noise"], p["phase_seed"])
        psi0s.append(s.contiguous())
    names = [p["name"] for p in insts]
    # the warm-up solves run the relaunch-schedule autotuner (three candidates)
    bs = BatchSolver(cfgs, grids, autotune=a.warmup >= 3)
    outs = [torch.empty_like(s) for s in psi0s]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2

    def step():
        _, res, _ = bs.solve_raw(psi0s, out=outs)
        return res

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    times, counted = [], 0
    eligible = 0
    step_counts = []
    last = None
    launches0 = bs.plan.launches
    with Clocks(local) as clk:
        for _ in range(a.steps):
            flush.fill_(1.0)
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            res = step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            c, el = _counts(names, [r.E_final for r in res], ref)
            counted += c
            eligible = el
            last = res
            step_counts.append(c)
    total = sum(times)
    launches = bs.plan.launches - launches0
    total_max, counted_all, value = job_rate(total, counted, dist, "cuda")

    # end to end through the public API with host buffers: pinned psi0 -> device,
    # solve, final states and energies back to the host, every step
    host_in = [s.cpu().pin_memory() for s in psi0s]
    host_out = [torch.empty(s.shape, dtype=s.dtype).pin_memory() for s in psi0s]
    h2d = sum(s.numel() * 16 for s in psi0s)
    d2h = h2d + 8 * len(psi0s)
    e2e_t, e2e_c = [], 0
    for _ in range(max(1, a.steps)):
        flush.fill_(1.0)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        dev_in = [h.to("cuda", non_blocking=True) for h in host_in]
        _, res, _ = bs.solve_raw(dev_in, out=outs)
        for o, h in zip(outs, host_out):
            h.copy_(o, non_blocking=True)
        energies = torch.tensor([r.E_final for r in res], dtype=torch.float64)
        e1.record()
        torch.cuda.synchronize()
        e2e_t.append(e0.elapsed_time(e1) / 1e3)
        e2e_c += _counts(names, energies.tolist(), ref)[0]
    e2e_value = job_rate(sum(e2e_t), e2e_c, dist, "cuda")[2]

    # roofline of the solver kernel (one persistent launch per step)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    algo = 0.0
    for r, G in zip(last, grids):
        n = G["N"] ** G["ndim"]
        algo += algorithmic_bytes(G["ndim"], n, r.iters, r.naccepted, r.ntrials, fp32_iterations(r))
    achieved = algo / (total / len(times)) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "ground states/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * total_max / len(times),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64" if a.precision == "fp64" else "f32 bulk (complex64 fields, FP32 transforms) with f64 reductions, potential and finish",
            "data": "synthetic (seeded workload instances, reference energies from a CPU run of becGPP)",
            "config": {"workload": workload_desc(a.workload),
                       "precision": a.precision,
                       "instances": len(insts), "eligible_per_step": eligible,
                       "schedule": bs.schedule(),
                       "counted_per_step": counted / len(times), "l2": "flushed between steps (256 MB)",
                       "parallelism": f"instances partitioned over {world} GPU(s), no collective"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": TRAFFIC_PER_ALGO_BYTE[a.precision] * algo,
                         "note": "algorithmic bytes of the fused passes per step / step time; "
                                 "peak = measured copy bandwidth" + ("" if peaks else " (fallback)")
                                 + "; traffic = DRAM bytes per step, scaled from an ncu capture of "
                                   "a smaller batch (DRAM bytes / algorithmic bytes = "
                                   f"{TRAFFIC_PER_ALGO_BYTE[a.precision]})"},
            "clocks": clk.summary(),
            "e2e": {"value": e2e_value, "unit": "ground states/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "iterations_max": max(r.iters for r in last)}
    rows = instance_rows(names, last, grids, ref)
    orc = _oracle_runs()
    line["accuracy"] = {
        "counted_each_step": step_counts,
        "fields": ["name", "N", "dE_rel", "resid_rel", "stop", "iters", "ref_resid_rel", "counted"],
        "rows": rows, "misses": miss_reasons(rows, orc),
        "oracle_counted": (sum(_matches(n, orc[n]["E"]) for n in names
                               if n in orc and ref[n]["obs"]["resid_rel"] <= ORACLE_RESID_MAX)
                           if orc else None),
        "note": "last timed step; dE_rel and resid_rel of the returned state against the reference's "
                "own CPU run; oracle_counted = the same count for the CPU restatement of the "
                "reference algorithm (tests/golden/oracle_runs.json), whose premature stalls "
                "show the algorithm's own sensitivity to round-off"}
    if rank == 0 and world == 1 and not a.no_plain:
        line["comparison"] = fp64_comparison(insts, cfgs, grids, psi0s, names, ref, a.precision,
                                             value)
    if rank == 0:
        line["hpsi"] = hpsi_rates(peak=peak)
    if rank == 0 and world == 1 and not a.no_configs:
        line["configs"] = config_results()
    if rank == 0 and world == 1 and a.cpu_sample > 0:
        cb = cpu_baseline(insts, ref, a.cpu_sample)
        line["cpu_baseline"] = {"value": cb["value"], "unit": "ground states/s", "cores": cb["cores"],
                                "kind": "port",
                                "sample": f"{cb['solves']} reference-converged instances at evenly spaced cost "
                                          f"ranks ({', '.join(cb['names'])}), {cb['cores']} worker processes, "
                                          f"{cb['wall_s']:.1f}s wall; the instances that never count are not "
                                          f"in it (the reference arm times the whole workload)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    bs.close()
    if dist:
        dist.destroy_process_group()


def main():
    a = _args()
    if a.case != "bench":
        run_case(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
