"""becgpp_b200 -- B200-native ground states of the Gross-Pitaevskii(-Poisson)
energy functional, a drop-in for the solve path of becGPP.

The Hamiltonian apply, energy, residual, zero-padded long-range convolution,
preconditioner and the whole normalised preconditioned CG iteration run as
hand-written sm_100a CUDA kernels in ``libbgp.so`` (C ABI in include/bgp.h);
this package mirrors becGPP's Python surface over it:

    from becgpp_b200 import default_cfg, run
    cfg = default_cfg(mode="single", dimension="2D", Omega=0.9, beta2=200,
                      seed="triangular", nseeds=3, L=12, Ngrid=384)
    diag = run(cfg)

As in becGPP, importing the package sets torch's default dtype to float64.
"""
import torch

torch.set_default_dtype(torch.float64)

from .config import CFG_DEFAULTS, default_cfg, canonical_key  # noqa: E402
from .grid import (DEV, make_grid, geometry, resolve_kernel, dV, norm_of, Plan,  # noqa: E402
                   plan_for, clear_plans)
from .interactions import long_range_phi, kernel_convolution, q2d_kernel, clear_kernel_cache  # noqa: E402
from .operators import energy_components, apply_H, compute_residual, observables, HamiltonianBatch  # noqa: E402
from .fields import mass_quantiles, mass_radius, radial_average, droplet_radius  # noqa: E402
from .thomasfermi import extract_tf  # noqa: E402
from .seeds import make_seed  # noqa: E402
from .solvers import ground_state, ground_state_multiseed, BatchSolver  # noqa: E402
from .autodiff import EnergyFunction, energy_and_grad, ground_state_sensitivities  # noqa: E402
from .vortex import vortex_diagnostic, lll_weight  # noqa: E402
from .diagnostics import diagnostics  # noqa: E402
from .modes import run, DISPATCH, run_id, write_csv  # noqa: E402
from .grid import auto_grid, resample_state  # noqa: E402

CODE_VERSION = "becgpp_b200_0.1"
__version__ = "0.1.0"

__all__ = [
    "CODE_VERSION", "DEV", "CFG_DEFAULTS", "default_cfg", "canonical_key",
    "make_grid", "geometry", "resolve_kernel", "dV", "norm_of", "Plan", "plan_for", "clear_plans",
    "long_range_phi", "kernel_convolution", "q2d_kernel", "clear_kernel_cache",
    "energy_components", "apply_H", "compute_residual", "observables", "HamiltonianBatch",
    "mass_quantiles", "mass_radius", "radial_average", "droplet_radius",
    "extract_tf", "make_seed", "ground_state", "ground_state_multiseed", "BatchSolver",
    "EnergyFunction", "energy_and_grad", "ground_state_sensitivities",
    "vortex_diagnostic", "lll_weight", "diagnostics", "run", "DISPATCH", "run_id", "write_csv",
    "auto_grid", "resample_state",
]
