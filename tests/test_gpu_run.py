"""run(cfg) and diagnostics() on the device against the reference's own results
(tests/golden/diag.*): the diagnostic bundle of solved states, a single run with
two seeds (one batch), a sweep with continuation (sequential) and a sweep of
fresh seeds (one batch). Tolerances: energies and observables 1e-10 relative,
radii and vortex counts exact, the TF reference 1e-8."""
import math

import pytest
import torch

from becgpp_b200 import default_cfg, diagnostics, make_grid, run

pytestmark = pytest.mark.gpu


def _close(a, b, tol):
    if isinstance(b, float) and math.isnan(b):
        return math.isnan(a)
    return abs(a - b) <= tol * max(1.0, abs(b))


def test_diagnostics_of_solved_states(golden):
    arr, meta = golden("diag")
    sol, _ = golden("solves")
    for key, m in meta.items():
        if not key.startswith("diag/"):
            continue
        name = key.split("/", 1)[1]
        c = default_cfg(mode="single", **m["cfg"])
        G = make_grid(c)
        d = diagnostics(torch.as_tensor(sol[f"{name}/psi"]).cuda(), G, c)
        ref = m["diag"]
        for k in ("Nv", "Nplus", "Nminus", "Nnet", "R50", "R90", "R99", "R_1pct", "points_per_R90"):
            assert _close(float(d[k]), ref[k], 0.0), (name, k, d[k], ref[k])
        for k in ("E", "mu", "Lz", "virial", "peak", "w_LLL", "lll_param"):
            assert _close(float(d[k]), ref[k], 1e-10), (name, k, d[k], ref[k])
        for k in ("tf_R90", "tf_R99", "tf_mu"):
            assert _close(float(d[k]), ref[k], 1e-8), (name, k, d[k], ref[k])
        assert d["tf_kind"] == ref["tf_kind"]


@pytest.mark.parametrize("name", ["single_rot", "sweep_b2", "sweep_fresh"])
def test_run_matches_reference(golden, name):
    _, meta = golden("diag")
    m = meta[f"run/{name}"]
    out = run(default_cfg(show_inline=False, save_figs=False, save_ckpt=False, **m["cfg"]))
    rows = out if isinstance(out, list) else [out]
    assert len(rows) == len(m["rows"])
    for got, ref in zip(rows, m["rows"]):
        assert _close(got["E"], ref["E"], 1e-10), (name, got["E"], ref["E"])
        assert got["stop_reason"] == ref["stop_reason"]
        assert got["Nv"] == ref["Nv"]
        if "branch" in ref:
            assert got["branch"] == ref["branch"]
        if "seed_used" in ref:
            assert got["seed_used"] == ref["seed_used"]
