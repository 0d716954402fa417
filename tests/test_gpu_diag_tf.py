"""Device density diagnostics and the Thomas-Fermi reference.

* Mass-quantile radii, centre of mass and radial profiles of libbgp's kernels
  against the oracle's restatement of becgpp/fields.py:9-57 (numpy sort and
  cumulative sum) on seeded fields: 2D and 3D, given and computed centres,
  negative values (clamped), symmetric fields (ties in distance), a massless
  field, fractions 0, 1 and beyond 1. The quantile radius is the distance of a
  grid point, so it must be the same point: equal to the last bit.
* The Thomas-Fermi densities of the device fixed point and the local inverted
  profile against the reference's own extract_tf (tests/golden/tf.*): chemical
  potential and density within 1e-8, radii and kind equal.
"""
import os
import sys

import numpy as np
import pytest
import torch

from becgpp_b200 import default_cfg, make_grid
from becgpp_b200.fields import center_of_mass, droplet_radius, mass_quantiles, radial_average
from becgpp_b200.thomasfermi import clear_tf_cache, extract_tf
from oracle import gpp as O

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from make_golden import big_weights  # noqa: E402

pytestmark = pytest.mark.gpu
FRACS = (0.0, 0.25, 0.5, 0.9, 0.99)


def _fields():
    g = np.random.default_rng(7)
    for ndim, N, L in ((2, 64, 6.0), (2, 128, 10.0), (3, 32, 5.0)):
        G = O.make_grid(default_cfg(dimension=f"{ndim}D", Ngrid=N, L=L))
        R2 = sum(c ** 2 for c in O._coords(G))
        env = np.exp(-0.5 * R2)
        yield f"{ndim}D{N}-noisy", G, env * (1.0 + 0.3 * g.standard_normal(R2.shape))
        yield f"{ndim}D{N}-signed", G, env * g.standard_normal(R2.shape)          # clamped negatives
        yield f"{ndim}D{N}-symmetric", G, env                                        # distance ties
        shifted = np.exp(-0.5 * ((O._coords(G)[0] - 0.7) ** 2 + (O._coords(G)[1] + 0.3) ** 2))
        yield f"{ndim}D{N}-offcentre", G, shifted
    G = O.make_grid(default_cfg(dimension="2D", Ngrid=48, L=4.0))
    yield "massless", G, np.zeros((48, 48))


def test_mass_quantiles_match_oracle():
    # the selection must pick the oracle's point given the same centre: with the
    # centre of mass (the device's; the centres agree to 1e-13 in the next test,
    # and a last-bit difference of a centre near 0 moves every distance) and with
    # a given centre
    for name, G, rho in _fields():
        t = torch.as_tensor(rho).cuda()
        cm = center_of_mass(t, G)
        assert mass_quantiles(t, G, FRACS) == O.mass_quantiles(rho, G, FRACS, center=cm), name
        c = (0.3, -0.2, 0.1)[:G["ndim"]]
        got = mass_quantiles(t, G, FRACS, center=c)
        want = O.mass_quantiles(rho, G, FRACS, center=c)
        assert got == want, (name, got, want)


def test_mass_quantiles_at_and_beyond_the_total():
    # f = 1: the last point in distance order whose mass counts (at least half a unit
    # of the 2^-58 fixed point of the total); f > 1: the farthest point (the
    # reference's clamp of the index). The reference's own f = 1 point is where its
    # floating running sum stops changing, which its rounding decides.
    for name, G, rho in _fields():
        if name == "massless":
            continue
        t = torch.as_tensor(rho).cuda()
        cm = center_of_mass(t, G)
        r = np.sqrt(sum((c - cm[i]) ** 2 for i, c in enumerate(O._coords(G))))
        w = np.clip(rho, 0.0, None) * G["dx"] ** G["ndim"]
        q = np.rint(w * (2.0 ** 58 / w.sum()))
        r1, r15 = mass_quantiles(t, G, (1.0, 1.5))
        assert r1 == float(r[q > 0].max()), name
        assert r15 == float(r.max()), name


def test_center_of_mass_matches_oracle():
    for name, G, rho in _fields():
        got = center_of_mass(torch.as_tensor(rho).cuda(), G)
        want = O.center_of_mass(rho, G)
        assert np.allclose(got, want, rtol=1e-13, atol=1e-15), (name, got, want)


def test_radial_profile_matches_oracle():
    for name, G, rho in _fields():
        for center in ((0.0,) * G["ndim"], (0.3, -0.2, 0.1)[:G["ndim"]]):
            ctr, prof = radial_average(torch.as_tensor(rho).cuda(), G, center=center)
            c2, p2 = O.radial_average(rho, G, center=center)
            assert np.array_equal(ctr, c2)
            assert np.array_equal(np.isnan(prof), np.isnan(p2)), name
            ok = ~np.isnan(p2)
            scale = max(np.abs(p2[ok]).max(), 1e-300) if ok.any() else 1.0
            assert np.abs(prof[ok] - p2[ok]).max() <= 1e-13 * scale, name


def test_droplet_radius_matches_oracle():
    for name, G, rho in _fields():
        if name == "massless":
            continue
        c = center_of_mass(torch.as_tensor(rho).cuda(), G)
        ctr, prof = O.radial_average(rho, G, center=c)
        pk = np.nanmax(prof)
        want = ctr[prof > 1e-2 * pk][-1]
        assert droplet_radius(torch.as_tensor(rho).cuda(), G) == want, name


def test_thomas_fermi_matches_reference(golden):
    arr, meta = golden("tf")
    for name, m in meta.items():
        clear_tf_cache()
        c = default_cfg(mode="single", **m["cfg"])
        G = make_grid(c)
        tf = extract_tf(c, G)
        assert tf is not None and tf["kind"] == m["kind"], (name, tf and tf["kind"])
        assert abs(tf["mu"] - m["mu"]) <= 1e-8 * max(1.0, abs(m["mu"])), (name, tf["mu"], m["mu"])
        assert bool(tf["converged"]) == m["converged"], name
        for k in ("R90", "R99"):
            assert abs(tf[k] - m[k]) <= 1e-8 * max(1.0, abs(m[k])), (name, k, tf[k], m[k])
        n = tf["n"].reshape(-1).cpu().numpy()
        idx, w = big_weights(m["n"], m["case_index"])
        assert np.array_equal(idx, arr[f"{name}/idx"])
        scale = m["field"]["maxabs"]
        err = np.abs(n[idx] - arr[f"{name}/n/samples"]).max() / scale
        assert err <= 1e-8, (name, err)
        proj = w @ n.astype(np.complex128)
        perr = np.abs(proj - arr[f"{name}/n/proj"]) / (np.sqrt((np.abs(w) ** 2).sum(axis=1)) * m["field"]["norm2"])
        assert perr.max() <= 1e-8, (name, perr.max())


@pytest.mark.parametrize("name", ["2d", "3d"])
def test_resample_state_matches_reference(golden, name):
    # device bi/trilinear resampling (bgp_resample) against the reference's grid_sample
    from becgpp_b200 import resample_state
    arr, meta = golden("diag")
    m = meta[f"resample/{name}"]
    Ga = make_grid(default_cfg(mode="single", **m["a"]))
    Gb = make_grid(default_cfg(mode="single", **m["b"]))
    psi = torch.as_tensor(arr[f"resample/{name}/psi"]).cuda()
    out = resample_state(psi, Ga, Gb).cpu().numpy()
    ref = arr[f"resample/{name}/out"]
    assert abs(out - ref).max() <= 1e-13 * abs(ref).max()


@pytest.mark.parametrize("name", ["mixed2d", "lll2d", "mixed3d"])
def test_vortex_count_and_lll_weight_match_reference(golden, name):
    # bgp_vortex_count / bgp_lll_weight against the reference's own values
    from becgpp_b200.vortex import lll_weight, vortex_diagnostic
    arr, meta = golden("diag")
    m = meta[name]
    c = default_cfg(mode="single", **m["cfg"])
    G = make_grid(c)
    psi = torch.as_tensor(arr[f"{name}/psi"]).cuda()
    assert vortex_diagnostic(psi, G, c["Omega"]) == m["vortex"]
    w = lll_weight(psi, G, 60, c["Omega"])
    if np.isnan(m["w_LLL"]):
        assert np.isnan(w)
    else:
        assert abs(w - m["w_LLL"]) <= 1e-12


@pytest.mark.parametrize("N,L,Omega,cores", [(128, 8.0, 0.7, ((1.0, 0.5, 1), (-1.5, -1.0, 1), (0.5, -2.0, -1))),
                                             (96, 6.0, -0.5, ((0.0, 0.0, 2), (2.0, 1.0, -1))),
                                             (64, 5.0, 0.9, ())])
def test_vortex_count_and_lll_weight_match_oracle(N, L, Omega, cores):
    # a Gaussian droplet with vortex cores (z - z_k)^(+-1) placed inside it
    from becgpp_b200.vortex import lll_weight, vortex_diagnostic
    x = (np.arange(N) - N // 2) * (2.0 * L / N)
    X, Y = np.meshgrid(x, x, indexing="ij")
    z = X + 1j * Y
    psi = np.exp(-0.5 * (X ** 2 + Y ** 2) / 4.0).astype(np.complex128)
    for cx, cy, q in cores:
        d = z - (cx + 1j * cy) + 1e-3 * (1 + 1j) * (2.0 * L / N)   # off the grid nodes
        for _ in range(abs(q)):
            psi = psi * (d if q > 0 else np.conj(d))
    G = dict(ndim=2, N=N, L=L)
    want_v = O.vortex_count_2d(psi, N, L, Omega)
    got_v = vortex_diagnostic(torch.as_tensor(psi).cuda(), G, Omega)
    assert got_v == want_v
    assert got_v["Nnet"] == sum(q for _, _, q in cores)
    want_w = O.lll_weight_2d(psi, N, L, 60, Omega)
    got_w = lll_weight(torch.as_tensor(psi).cuda(), G, 60, Omega)
    assert abs(got_w - want_w) <= 1e-12, (got_w, want_w)
