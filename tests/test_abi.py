"""The C ABI library: it loads on a machine without a GPU, exports every entry
point include/bgp.h declares, and its host-only helpers are exact."""
import ctypes
import os
import re

import numpy as np
import pytest

from becgpp_b200 import _lib
from becgpp_b200.config import default_cfg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "bgp.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bgp_[A-Za-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert "bgp_solve" in names and "bgp_apply_H" in names
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.exported_symbols())


def test_version_and_error_string():
    assert _lib.lib().bgp_version() >= 100
    assert isinstance(_lib.lib().bgp_last_error(), bytes)


def test_bessel_helpers_match_scipy():
    from scipy import special
    xs = np.concatenate([np.logspace(-12, 5, 300), [0.5, 1.0, 2.0, 10.0]])
    k0 = np.array([_lib.lib().bgp_k0e(x) for x in xs])
    k1 = np.array([_lib.lib().bgp_k1e(x) for x in xs])
    assert np.max(np.abs(k0 - special.k0e(xs)) / special.k0e(xs)) < 3e-15
    assert np.max(np.abs(k1 - special.k1e(xs)) / special.k1e(xs)) < 3e-15


def test_size_table():
    f = _lib.lib().bgp_size_supported
    for n in (16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512):
        assert f(2, n, 2, 0) == 1 and f(3, n, 2, 0) == 1
    for n in (16, 128, 256, 384):
        assert f(2, n, 2, 1) == 1
    assert f(2, 512, 2, 1) == 0      # M = 1024 lines are not compiled in
    assert f(2, 100, 2, 0) == 0
    assert f(2, 128, 3, 1) == 0      # pad 3 not compiled in
    assert f(4, 128, 2, 0) == 0


def test_default_cfg_aliases_and_unknown_keys():
    assert default_cfg(res=1e-7)["res_tol"] == 1e-7
    assert default_cfg(N=64)["Ngrid"] == 64
    with pytest.raises(ValueError):
        default_cfg(omega=0.9)
    with pytest.raises(ValueError):
        default_cfg(res=1e-7, res_tol=1e-6)


def test_device_calls_fail_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from becgpp_b200 import apply_H, make_grid
    c = default_cfg(Ngrid=32, L=6)
    G = make_grid(c)
    with pytest.raises(RuntimeError):
        apply_H(torch.zeros(32, 32, dtype=torch.complex128), G, c)
