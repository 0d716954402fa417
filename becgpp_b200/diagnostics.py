"""Diagnostic bundle of a solved state, the record `run` returns per result
(becgpp/diagnostics.py:18-47): the observables (energy terms, mu, L_z, virial),
mass radii, vortex count, lowest-Landau-level weight where it applies, and the
Thomas-Fermi reference of the same configuration."""
import math

from .fields import droplet_radius, mass_quantiles
from .operators import observables
from .thomasfermi import extract_tf
from .vortex import lll_weight, vortex_diagnostic


def lll_applicable(G, cfg):
    """The LLL basis z^m exp(-r^2/2) belongs to the isotropic harmonic trap
    V = r^2/2 in 2D; the weight is reported for rotating runs there only."""
    return (G["ndim"] == 2 and abs(float(G["s"]) - 2.0) < 1e-12
            and abs(float(G.get("trap_coeff", 0.5)) - 0.5) < 1e-12
            and abs(float(cfg.get("Omega", 0.0))) > 0.0)


def diagnostics(psi, G, cfg):
    d = observables(psi, G, cfg)
    rho = psi.abs() ** 2
    R50, R90, R99 = mass_quantiles(rho, G, (0.50, 0.90, 0.99))
    d.update(R50=R50, R90=R90, R99=R99, R_1pct=droplet_radius(rho, G))
    Omega = float(cfg.get("Omega", 0.0))
    if cfg.get("want_vortices", True):
        d.update(vortex_diagnostic(psi, G, Omega))
    else:
        d.update(Nv=0, Nplus=0, Nminus=0, Nnet=0)
    lll = bool(cfg.get("want_lll", True)) and lll_applicable(G, cfg)
    d["w_LLL"] = lll_weight(psi, G, 60, Omega) if lll else float("nan")
    # mean-field LLL criterion: interaction energy at the peak against the gap
    # (1 + |Omega|) to the next Landau level in the rotating frame
    d["lll_param"] = (abs(float(cfg["beta2"])) * d["peak"] / (1.0 + abs(Omega))) if lll else float("nan")
    tf = extract_tf(cfg, G)
    nan = float("nan")
    if tf is not None:
        d.update(tf_kind=tf.get("kind", ""), tf_R90=tf.get("R90", nan), tf_R99=tf.get("R99", nan),
                 tf_mu=tf.get("mu", nan), tf_rho0=tf.get("rho0", nan),
                 tf_converged=bool(tf.get("converged", False)))
    else:
        d.update(tf_kind="", tf_R90=nan, tf_R99=nan, tf_mu=nan, tf_rho0=nan, tf_converged=False)
    d["mem_estimate_gb"] = G.get("mem_estimate_gb", nan)
    d["points_per_R90"] = d["R90"] / G["dx"] if math.isfinite(d["R90"]) else nan
    return d
