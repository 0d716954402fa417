"""The batched H psi (bgp_apply_H_batch: per-axis stream launches, no host
synchronisation) against the reference's H psi (tests/golden/ops.*, bigops.*),
under every pass schedule its autotuner can choose: each compiled (lines per
tile, radix order) of the H psi passes and each lines-per-tile of the
convolution passes. Tolerance 1e-12 relative (max-norm), the single-apply bar.
Also: a batch that mixes grid sizes equals the single applies, mu equals
Re<psi, H psi> dV, the persistent single-instance entry point bgp_apply_H
still matches the reference, and argument errors are reported."""
import ctypes

import numpy as np
import pytest
import torch

from becgpp_b200 import HamiltonianBatch, _lib, default_cfg, make_grid
from becgpp_b200.grid import plan_for

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _cases(golden):
    arr, meta = golden("ops")
    for name, m in meta.items():
        c = default_cfg(mode="single", **m["cfg"])
        yield name, c, make_grid(c), torch.as_tensor(arr[f"{name}/psi"]).cuda(), arr


def test_every_schedule_matches_reference(golden):
    for name, c, G, psi, arr in _cases(golden):
        hb = HamiltonianBatch([c], [G])
        out = hb.apply([psi])[0]                       # first call: the autotuner's choice
        assert _rel(out, arr[f"{name}/H"]) < TOL, (name, hb.schedule(G["N"]))
        sched = hb.schedule(G["N"])
        assert sched["tuned"] == 1
        cands = [(ln, v) for ln, v, _, _ in sched["candidates_ms"] if ln > 0]
        assert len(cands) >= 6, (name, cands)          # >= 2 tile widths x 3 radix orders
        conv = G["kernel"] != "none"
        cconv = [(-ln, v, sl) for ln, v, sl, _ in sched["candidates_ms"] if ln < 0] if conv else [(8, 0, 8)]
        # contiguous widths 4 and 8, strided widths 4, 8 and 16, each with the Stockham transform
        assert not conv or len(cconv) >= 6, (name, cconv)
        for ln, v in cands:
            for cl, cv, csl in cconv:
                hb.set_schedule(G["N"], ln, v, cl, cv, conv_strided_lines=csl)
                out = hb.apply([psi])[0]
                assert _rel(out, arr[f"{name}/H"]) < TOL, (name, ln, v, cl, cv, csl)
        hb.close()


def test_mixed_size_batch_equals_single_applies_and_mu(golden):
    arr, meta = golden("ops")
    names = list(meta)
    cfgs = [default_cfg(mode="single", **meta[n]["cfg"]) for n in names]
    grids = [make_grid(c) for c in cfgs]
    psis = [torch.as_tensor(arr[f"{n}/psi"]).cuda() for n in names]
    hb = HamiltonianBatch(cfgs, grids)
    mu = torch.zeros(len(names), dtype=torch.float64, device="cuda")
    outs = hb.apply(psis, mu=mu)
    torch.cuda.synchronize()
    for k, n in enumerate(names):
        assert _rel(outs[k], arr[f"{n}/H"]) < TOL, n
        dv = grids[k]["dx"] ** grids[k]["ndim"]
        want = float((psis[k].conj() * outs[k]).real.sum()) * dv
        assert abs(float(mu[k]) - want) <= 1e-12 * max(1.0, abs(want)), (n, float(mu[k]), want)
    hb.close()


def test_big_batch_of_droplets_matches_single_applies():
    # the droplet sweep's shape: 128^2 and 256^2 instances interleaved
    cfgs, psis = [], []
    g = torch.Generator().manual_seed(3)
    for b in range(12):
        c = default_cfg(dimension="2D", beta2=-400.0 + 25.0 * b, beta3=1e3, L=20.0, Ngrid=128 if b % 2 == 0 else 256)
        cfgs.append(c)
        N = c["Ngrid"]
        psis.append((torch.randn(N, N, generator=g, dtype=torch.float64)
                     + 1j * torch.randn(N, N, generator=g, dtype=torch.float64)).cuda())
    grids = [make_grid(c) for c in cfgs]
    hb = HamiltonianBatch(cfgs, grids)
    outs = hb.apply(psis)
    for c, G, p, o in zip(cfgs, grids, psis, outs):
        one = HamiltonianBatch([c], [G])
        ref = one.apply([p])[0]
        one.close()
        assert _rel(o, ref.cpu().numpy()) < 1e-14
    hb.close()


def test_persistent_single_apply_matches_reference(golden):
    for name, c, G, psi, arr in _cases(golden):
        plan = plan_for(G, c)
        out = torch.empty_like(psi)
        mu = ctypes.c_double()
        _lib.check(_lib.lib().bgp_apply_H(plan.handle, 0, _lib.ptr(psi), _lib.ptr(out), None,
                                          2 if G["kernel"] != "none" else 0, ctypes.byref(mu), _lib.stream_ptr()),
                   "bgp_apply_H")
        assert _rel(out, arr[f"{name}/H"]) < TOL, name


def test_batch_rejects_bad_arguments():
    c = default_cfg(mode="single", Ngrid=32, L=6)
    G = make_grid(c)
    hb = HamiltonianBatch([c], [G])
    psi = torch.zeros((32, 32), dtype=torch.complex128, device="cuda")
    o1, o2 = torch.empty_like(psi), torch.empty_like(psi)
    P = ctypes.c_void_p * 2
    lib = _lib.lib()
    # the same instance twice
    rc = lib.bgp_apply_H_batch(hb.plan.handle, 2, (ctypes.c_int * 2)(0, 0), P(psi.data_ptr(), psi.data_ptr()),
                               P(o1.data_ptr(), o2.data_ptr()), None, 0, None, _lib.stream_ptr())
    assert rc == -1 and b"twice" in lib.bgp_last_error()
    # aliasing input and output
    rc = lib.bgp_apply_H_batch(hb.plan.handle, 1, (ctypes.c_int * 1)(0), (ctypes.c_void_p * 1)(psi.data_ptr()),
                               (ctypes.c_void_p * 1)(psi.data_ptr()), None, 0, None, _lib.stream_ptr())
    assert rc == -1 and b"alias" in lib.bgp_last_error()
    with pytest.raises(ValueError):
        hb.set_schedule(32, 3, 0, 8)                   # 3 lines per tile is not compiled
    with pytest.raises(ValueError):
        hb.set_schedule(32, 4, 0, 16)                  # contiguous convolution tiles: 4 or 8 lines
    hb.close()


def test_one_line_tiles_of_a_large_3d_grid():
    # 192^3 in one-line tiles: 36864 tiles in the last pass, each leaving its part of
    # Re<psi, H psi>; equal to the 4-line schedule, mu equal to the direct sum
    c = default_cfg(mode="single", dimension="3D", Ngrid=192, L=8.0, beta2=10.0, Omega=0.3)
    G = make_grid(c)
    g = torch.Generator().manual_seed(5)
    psi = (torch.randn(192, 192, 192, generator=g, dtype=torch.float64)
           + 1j * torch.randn(192, 192, 192, generator=g, dtype=torch.float64)).cuda()
    hb = HamiltonianBatch([c], [G])
    outs = {}
    for ln in (1, 4):
        hb.set_schedule(192, ln, 0)
        mu = torch.zeros(1, dtype=torch.float64, device="cuda")
        outs[ln] = hb.apply([psi], mu=mu)[0].clone()
        torch.cuda.synchronize()
        want = float((psi.conj() * outs[ln]).real.sum()) * G["dx"] ** 3
        assert abs(float(mu[0]) - want) <= 1e-12 * abs(want), (ln, float(mu[0]), want)
    assert _rel(outs[1], outs[4].cpu().numpy()) < 1e-13
    hb.close()
