"""Derivatives of the energy functional on the device (bgp_energy_grad behind
torch.autograd): against torch autograd through the reference's FP64 energy
(fixtures), central differences of our own energy, the identity
dE/dpsi* = H psi dV, and Hellmann-Feynman sensitivities of a ground state
against central differences of the reference's ground-state energies."""
import numpy as np
import pytest
import torch

from becgpp_b200 import apply_H, default_cfg, ground_state, make_grid
from becgpp_b200.autodiff import PARAMS, energy, energy_and_grad, ground_state_sensitivities

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _cases(golden):
    arr, meta = golden("grads")
    for name, m in meta.items():
        if name == "hf":
            continue
        c = default_cfg(mode="single", **m["cfg"])
        G = make_grid(c)
        yield name, m, c, G, torch.as_tensor(arr[f"{name}/psi"]).cuda(), arr


def test_autograd_matches_reference_autograd(golden):
    # tolerance: 1e-10 relative for the autograd values, 1e-6 for the l_z central difference
    for name, m, c, G, psi, arr in _cases(golden):
        p = psi.clone().requires_grad_(True)
        pars = {k: torch.tensor(float(c[k]) if k != "l_z" else float(G["l_z"]), dtype=torch.float64,
                                requires_grad=True) for k in PARAMS}
        lz = pars["l_z"] if G["kernel"] == "q2d" else None
        E = energy(p, G, pars["beta2"], pars["beta3"], pars["G_C"], pars["Omega"], lz)
        E.backward()
        assert abs(float(E.detach()) - m["E"]) <= 1e-12 * max(1.0, abs(m["E"])), name
        assert _rel(p.grad, arr[f"{name}/dpsi"]) < 1e-11, name
        for k, v in m["dparams"].items():
            got = float(pars[k].grad)
            tol = 1e-6 if k == "l_z" else 1e-10
            assert abs(got - v) <= tol * max(1.0, abs(v)), (name, k, got, v)


def test_psi_gradient_is_hamiltonian(golden):
    for name, m, c, G, psi, arr in _cases(golden):
        _, dpsi, _ = energy_and_grad(psi, G, c["beta2"], c["beta3"], c["G_C"], c["Omega"],
                                     G["l_z"] if G["kernel"] == "q2d" else None)
        ref = apply_H(psi, G, c) * G["dx"] ** G["ndim"]
        assert float((dpsi - ref).abs().max() / ref.abs().max()) < 1e-12, name


def test_parameter_gradients_match_central_differences(golden):
    # central differences of our own energy, h = 1e-6 (relative to max(1, |p|)); tolerance 1e-6
    for name, m, c, G, psi, arr in _cases(golden):
        base = dict(beta2=c["beta2"], beta3=c["beta3"], G_C=c["G_C"], Omega=c["Omega"],
                    l_z=G["l_z"] if G["kernel"] == "q2d" else None)
        _, _, d = energy_and_grad(psi, G, want_psi_grad=False, **base)
        for k in PARAMS:
            if base[k] is None or (k == "G_C" and G["kernel"] == "none"):
                continue
            h = 1e-6 * max(1.0, abs(base[k]))
            Es = []
            for sgn in (1, -1):
                pk = dict(base, **{k: base[k] + sgn * h})
                t, _, _ = energy_and_grad(psi, G, want_psi_grad=False, **pk)
                Es.append(t["E"])
            fd = (Es[0] - Es[1]) / (2 * h)
            assert abs(fd - d[k]) <= 1e-6 * max(1.0, abs(d[k])), (name, k, fd, d[k])


def test_psi_gradient_matches_directional_difference(golden):
    # d/de E(psi + e v) = 2 Re <dE/dpsi*, v>  (real directional derivative)
    for name, m, c, G, psi, arr in _cases(golden):
        g = torch.Generator().manual_seed(5)
        v = torch.complex(torch.randn(psi.shape, generator=g, dtype=torch.float64),
                          torch.randn(psi.shape, generator=g, dtype=torch.float64)).cuda() * psi.abs()
        lz = G["l_z"] if G["kernel"] == "q2d" else None
        args = (c["beta2"], c["beta3"], c["G_C"], c["Omega"], lz)
        _, dpsi, _ = energy_and_grad(psi, G, *args)
        an = 2.0 * float((dpsi.conj() * v).real.sum())
        eps = 1e-6
        Ep = energy_and_grad(psi + eps * v, G, *args, want_psi_grad=False)[0]["E"]
        Em = energy_and_grad(psi - eps * v, G, *args, want_psi_grad=False)[0]["E"]
        assert abs((Ep - Em) / (2 * eps) - an) <= 1e-6 * abs(an), name


def test_hellmann_feynman_sensitivities(golden):
    # ground state of a quasi-2D rotating pancake, then dE_gs/dp from the explicit
    # parameter derivatives at the converged state, against central differences of the
    # reference's own ground-state energies (fixture); tolerance 1e-5 relative
    arr, meta = golden("grads")
    hf = meta["hf"]
    c = default_cfg(mode="single", **hf["cfg"])
    psi, G, obs = ground_state(c, psi0=torch.as_tensor(arr["hf/psi0"]).cuda(), verbose=False)
    assert abs(obs["E"] - hf["E"]) <= 1e-10 * abs(hf["E"])
    sens = ground_state_sensitivities(psi, G, c)
    for k, fd in hf["fd"].items():
        assert abs(sens[k] - fd["dE"]) <= 1e-5 * max(1.0, abs(fd["dE"])), (k, sens[k], fd["dE"])
