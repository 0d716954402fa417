"""Run configuration: the flat key/default table of becGPP and its validation.

The key set, defaults and aliases are the reference's interface
(becgpp/config.py:15-119) and are kept identical so a config dict written for
becGPP runs here unchanged. Two keys are added for this implementation:

* ``precision``  -- ``"fp64"`` (every kernel in double precision, the reference's
  arithmetic) or ``"mixed"`` (FP32 transforms and bulk with FP64 reductions,
  switching to FP64 iterations once the residual reaches the FP32 floor).
* ``mixed_switch_res`` -- relative residual below which the mixed form hands
  over to FP64 transforms (it also hands over at its first failed line search).
* ``batch_team`` -- CTAs per instance in a batched solve; 0 lets the scheduler
  choose.
"""

CFG_DEFAULTS = dict(
    mode="smoke",
    # geometry
    dimension="2D",
    s=2,
    trap_coeff=0.5,
    Omega=0.0,
    # interactions
    beta2=100.0,
    beta3=0.0,
    G_C=0.0,
    kernel="auto",
    l_z=0.0,
    # grid
    L=10.0,
    Ngrid=128,
    pad=2,
    mem_warn_gb=12.0,
    # solver
    maxit=60000,
    res_tol=1e-4,
    energy_tol=1e-9,
    conv_window=2000,
    step=1.0,
    step_max=3.0,
    linesearch_max=8,
    linesearch_stall=10,
    precond_shift_min=0.5,
    cg_beta="pr_precond",
    cg_restart=30,
    record_trace=False,
    check=200,
    # seeding
    seed="tf",
    seed_winding=0,
    seed_noise=1e-2,
    seed_phase_noise=5e-2,
    rng=0,
    nseeds=1,
    # diagnostics
    want_vortices=True,
    want_lll=True,
    tf_cache=True,
    # validate mode
    validate_N=256,
    # sweep mode
    sweep_param="G_C",
    sweep_values=[1.0, 2.0, 4.0, 8.0, 16.0],
    sweep_autobox=False,
    sweep_continuation=True,
    # convergence mode
    conv_Ngrids=[96, 128, 192],
    conv_box_factors=[1.0, 1.2],
    conv_pads=[2, 3],
    # output
    tag="becgpp",
    show_inline=True,
    save_figs=True,
    save_ckpt=True,
    zip_output=False,
    # this implementation
    precision="fp64",
    mixed_switch_res=1e-5,
    batch_team=0,
)

_ALIASES = dict(res="res_tol", etol="energy_tol", N="Ngrid", dim="dimension",
                precond_shift="precond_shift_min")


def canonical_key(key):
    """Map a short alias (``res``, ``etol``, ``N``, ``dim``, ``precond_shift``) to its key."""
    return _ALIASES.get(key, key)


def default_cfg(**overrides):
    """A fresh copy of the defaults with ``overrides`` applied.

    Aliases map to their canonical keys; giving both an alias and its key, or
    any unknown key, raises ``ValueError`` (becgpp/config.py:100-119)."""
    cfg = dict(CFG_DEFAULTS)
    for alias, canonical in _ALIASES.items():
        if alias in overrides:
            if canonical in overrides:
                raise ValueError(f"pass only one of {alias!r} or {canonical!r}")
            overrides[canonical] = overrides.pop(alias)
    unknown = set(overrides) - set(CFG_DEFAULTS)
    if unknown:
        raise ValueError(f"unknown config key(s): {sorted(unknown)}; "
                         f"see becgpp_b200.config.CFG_DEFAULTS for valid keys")
    cfg.update(overrides)
    return cfg
