"""Post-solve diagnostics on the host (no GPU): the oracle's vortex count and LLL
weight of synthetic states against the reference's own values (tests/golden/diag.*;
the device kernels are checked against the same fixtures in
test_gpu_diag_tf.py), and the run() dispatch errors."""
import math

import pytest

from becgpp_b200 import default_cfg, run
from oracle import gpp


@pytest.mark.parametrize("name", ["mixed2d", "lll2d", "mixed3d"])
def test_oracle_vortex_count_and_lll_weight(golden, name):
    arr, meta = golden("diag")
    m = meta[name]
    c = m["cfg"]
    N, L = int(c["Ngrid"]), float(c["L"])
    psi = arr[f"{name}/psi"]
    if c["dimension"] == "3D":
        psi = psi[:, :, N // 2]
    assert gpp.vortex_count_2d(psi, N, L, c["Omega"]) == m["vortex"]
    w = gpp.lll_weight_2d(psi, N, L, 60, c["Omega"]) if c["dimension"] == "2D" else float("nan")
    if math.isnan(m["w_LLL"]):
        assert math.isnan(w)
    else:
        assert abs(w - m["w_LLL"]) <= 1e-12


def test_run_rejects_unknown_modes_and_sweeps():
    with pytest.raises(ValueError, match="unknown mode"):
        run(default_cfg(mode="nope"))
    with pytest.raises(ValueError, match="validate"):
        run(default_cfg(mode="validate"))
    with pytest.raises(ValueError, match="not a numeric CFG key"):
        run(default_cfg(mode="sweep", sweep_param="seed"))
    with pytest.raises(ValueError, match="must be numbers"):
        run(default_cfg(mode="sweep", sweep_param="beta2", sweep_values=[1.0, "x"]))
    assert run(default_cfg(mode="sweep", sweep_param="beta2", sweep_values=[])) == []


def test_auto_grid_matches_reference(golden):
    from becgpp_b200 import auto_grid
    _, meta = golden("diag")
    for key, m in meta.items():
        if key.startswith("autogrid/"):
            L, N, R = auto_grid(default_cfg(mode="single", **m["cfg"]))
            assert (L, N) == (m["L"], m["N"]) and abs(R - m["R"]) <= 1e-15 * max(1.0, abs(m["R"])), key


@pytest.mark.parametrize("name", ["2d", "3d"])
def test_oracle_resample_matches_reference(golden, name):
    # the interpolation rule the device kernel implements, pinned on the CPU
    from oracle import gpp as O
    arr, meta = golden("diag")
    m = meta[f"resample/{name}"]
    Ga = O.make_grid(default_cfg(mode="single", **m["a"]))
    Gb = O.make_grid(default_cfg(mode="single", **m["b"]))
    out = O.resample_state(arr[f"resample/{name}/psi"], Ga, Gb)
    ref = arr[f"resample/{name}/out"]
    assert abs(out - ref).max() <= 1e-13 * abs(ref).max()
