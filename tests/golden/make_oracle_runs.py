"""Solve the benchmark workloads with the oracle and commit the outcomes
(tests/golden/oracle_runs.json). TEST INFRASTRUCTURE: the oracle is the CPU
restatement of the reference's algorithm, not the product.

The reference's own CPU runs of the same instances are tests/golden/
baseline_runs.json. Comparing the two shows how far two faithful FP64
implementations of the same algorithm agree: on the droplet sweep both stop
some instances early (line search stalled at a large residual) on different
instances, because that stop depends on round-off.

    python tests/golden/make_oracle_runs.py [WORKLOADS]   # default c4,c1,c5,c3

One worker process per host core, one thread each (`spawn` pool).
"""
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def solve(p):
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    from oracle import gpp as O
    from becgpp_b200.config import default_cfg
    from becgpp_b200.seeds import make_seed, phase_noise
    O.WORKERS = 1
    c = default_cfg(**p["cfg"])
    G = O.make_grid(c)
    Gd = dict(ndim=G["ndim"], N=G["N"], L=G["L"], s=G["s"], trap_coeff=G["trap_coeff"],
              kernel=G["kernel"], pad=G["pad"], l_z=G["l_z"], dx=G["dx"])
    s = make_seed(Gd, c, device="cpu")
    if p.get("phase_noise"):
        s = phase_noise(s, p["phase_noise"], p["phase_seed"])
    t0 = time.time()
    _, obs = O.ground_state(c, s.numpy())
    return p["name"], dict(E=float(obs["E"]), resid_rel=float(obs["resid_rel"]),
                           stop_reason=obs["stop_reason"], iters=int(obs["iters"]),
                           wall_s=round(time.time() - t0, 2))


def main():
    sys.path.insert(0, ROOT)
    from becgpp_b200.workloads import WORKLOADS
    names = (sys.argv[1] if len(sys.argv) > 1 else "c4,c1,c5,c3").split(",")
    insts = [p for w in names for p in WORKLOADS[w]()]
    path = os.path.join(HERE, "oracle_runs.json")
    done = json.load(open(path)) if os.path.isfile(path) else {}
    todo = [p for p in insts if p["name"] not in done]
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        for name, r in pool.imap_unordered(solve, todo):
            done[name] = r
            print(name, r, flush=True)
            with open(path, "w") as f:
                json.dump(done, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
