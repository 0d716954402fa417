"""The allocation-free Hamiltonian apply (bgp_apply_H_noalloc).

It serves callers that cannot call cudaMalloc (a host framework that owns the
device-memory budget, or a loop that cannot afford cudaMalloc's device-wide
synchronisation); its scratch is a fixed static device array. Its output must
equal the planned entry point's (bgp_apply_H) within the parity tolerance, on
two calls in a row, since every call reuses the same static scratch.
This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from becgpp_b200 import _lib, apply_H, default_cfg, make_grid
from becgpp_b200.grid import instance_desc

pytestmark = pytest.mark.gpu
TOL = 1e-12
BGP_ERR_ARG = -1


def _noalloc(desc, psi, phi):
    out = torch.empty_like(psi)
    rc = _lib.lib().bgp_apply_H_noalloc(ctypes.byref(desc), _lib.ptr(psi), _lib.ptr(out), _lib.ptr(phi),
                                        _lib.stream_ptr())
    _lib.check(rc, "bgp_apply_H_noalloc")
    torch.cuda.synchronize()
    return out


def test_noalloc_matches_planned_apply_twice(golden):
    arr, meta = golden("ops")
    for name, m in meta.items():
        c = default_cfg(mode="single", **m["cfg"])
        G = make_grid(c)
        psi = torch.as_tensor(arr[f"{name}/psi"]).cuda().contiguous()
        phi = torch.as_tensor(arr[f"{name}/phi"]).cuda().contiguous() if G["kernel"] != "none" else None
        ref = apply_H(psi, G, c, phi=phi)
        want = torch.as_tensor(arr[f"{name}/H"]).cuda()
        desc = instance_desc(G, c)
        for call in range(2):
            out = _noalloc(desc, psi, phi)
            err = float((out - ref).abs().max() / ref.abs().max())
            assert err < TOL, (name, call, err)
            # and directly against the reference's own H psi of the fixture
            err_ref = float((out - want).abs().max() / want.abs().max())
            assert err_ref < TOL, (name, call, err_ref)


def test_noalloc_rejects_grids_beyond_its_scratch():
    c = default_cfg(mode="single", dimension="3D", Ngrid=96, L=6)
    G = make_grid(c)
    desc = instance_desc(G, c)
    psi = torch.zeros((96, 96, 96), dtype=torch.complex128, device="cuda")
    out = torch.empty_like(psi)
    rc = _lib.lib().bgp_apply_H_noalloc(ctypes.byref(desc), _lib.ptr(psi), _lib.ptr(out), None,
                                        _lib.stream_ptr())
    assert rc == BGP_ERR_ARG
    assert b"262144" in _lib.lib().bgp_last_error()
