"""ctypes binding of libbgp.so (the C ABI in include/bgp.h).

The library is loaded from this package directory (or from the path in the
environment variable BECGPP_B200_LIB, e.g. the phase-profiling build
libbgp_prof.so). There is no fallback: if the shared object is missing, or no
CUDA device is visible when a device entry point is called, a RuntimeError says
so.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbgp.so")

KERNEL_CODES = {"none": 0, "newton": 1, "log": 2, "q2d": 3}
CG_BETA_CODES = {"pr_precond": 0, "pr": 1, "none": 2}
STOP_NAMES = {0: "maxit", 1: "converged", 2: "energy_converged", 3: "line_search_stalled",
              4: "device_error"}


class InstanceDesc(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("N", ctypes.c_int), ("pad", ctypes.c_int),
                ("kernel", ctypes.c_int), ("L", ctypes.c_double), ("s", ctypes.c_double),
                ("trap_coeff", ctypes.c_double), ("beta2", ctypes.c_double),
                ("beta3", ctypes.c_double), ("Omega", ctypes.c_double), ("G_C", ctypes.c_double),
                ("l_z", ctypes.c_double)]


class SolverParams(ctypes.Structure):
    _fields_ = [("maxit", ctypes.c_int), ("linesearch_max", ctypes.c_int),
                ("linesearch_stall", ctypes.c_int), ("cg_restart", ctypes.c_int),
                ("cg_beta", ctypes.c_int), ("conv_window", ctypes.c_int),
                ("record_trace", ctypes.c_int), ("trace_cap", ctypes.c_int),
                ("mixed", ctypes.c_int),
                ("res_tol", ctypes.c_double), ("energy_tol", ctypes.c_double),
                ("step", ctypes.c_double), ("step_max", ctypes.c_double),
                ("precond_shift_min", ctypes.c_double), ("mixed_switch_res", ctypes.c_double)]


class SolveResult(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int), ("stop_reason", ctypes.c_int), ("converged", ctypes.c_int),
                ("ntrials", ctypes.c_int), ("ntrace", ctypes.c_int), ("best_is_final", ctypes.c_int),
                ("status", ctypes.c_int), ("naccepted", ctypes.c_int),
                ("E", ctypes.c_double), ("resid_rel", ctypes.c_double),
                ("resid_abs", ctypes.c_double), ("min_resid", ctypes.c_double),
                ("sigma", ctypes.c_double), ("mu", ctypes.c_double), ("alpha", ctypes.c_double),
                ("maxrho", ctypes.c_double), ("E_final", ctypes.c_double), ("mu_final", ctypes.c_double),
                ("resid_abs_final", ctypes.c_double), ("resid_rel_final", ctypes.c_double),
                ("mass_final", ctypes.c_double), ("fp64_from", ctypes.c_int), ("reserved", ctypes.c_int)]


class EnergyTerms(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("E", "Ekin", "Etrap", "Econtact", "Ethree", "Erot",
                                                "Egrav", "Lz", "mass", "r2mean", "peak", "rperp2",
                                                "z2")]


_P = ctypes.c_void_p
_SIGS = {
    "bgp_version": ([], ctypes.c_int),
    "bgp_last_error": ([], ctypes.c_char_p),
    "bgp_plan_create": ([ctypes.POINTER(InstanceDesc), ctypes.c_int, ctypes.POINTER(_P)], ctypes.c_int),
    "bgp_plan_destroy": ([_P], ctypes.c_int),
    "bgp_plan_bytes": ([_P], ctypes.c_longlong),
    "bgp_plan_launches": ([_P], ctypes.c_longlong),
    "bgp_plan_autotune": ([_P, ctypes.c_int], ctypes.c_int),
    "bgp_plan_schedule": ([_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "bgp_apply_H": ([_P, ctypes.c_int, _P, _P, _P, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _P],
                    ctypes.c_int),
    "bgp_energy": ([_P, ctypes.c_int, _P, _P, ctypes.POINTER(EnergyTerms), _P], ctypes.c_int),
    "bgp_residual": ([_P, ctypes.c_int, _P, ctypes.POINTER(ctypes.c_double), _P], ctypes.c_int),
    "bgp_energy_grad": ([_P, ctypes.c_int, _P, ctypes.POINTER(EnergyTerms), _P,
                         ctypes.POINTER(ctypes.c_double), _P], ctypes.c_int),
    "bgp_convolve": ([_P, ctypes.c_int, _P, _P, ctypes.c_int, _P], ctypes.c_int),
    "bgp_precondition": ([_P, ctypes.c_int, _P, _P, _P, ctypes.c_double, _P,
                          ctypes.POINTER(ctypes.c_double), _P], ctypes.c_int),
    "bgp_solve": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(SolverParams),
                   ctypes.POINTER(SolveResult), ctypes.POINTER(ctypes.c_double), _P], ctypes.c_int),
    "bgp_apply_H_noalloc": ([ctypes.POINTER(InstanceDesc), _P, _P, _P, _P], ctypes.c_int),
    "bgp_apply_H_batch": ([_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_P), ctypes.POINTER(_P),
                           ctypes.POINTER(_P), ctypes.c_int, _P, _P], ctypes.c_int),
    "bgp_plan_stream_schedule": ([_P, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "bgp_plan_stream_set": ([_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                             ctypes.c_int], ctypes.c_int),
    "bgp_tf_density": ([_P, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, _P,
                        ctypes.POINTER(ctypes.c_double), _P], ctypes.c_int),
    "bgp_density_center": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, _P, ctypes.POINTER(ctypes.c_double),
                            ctypes.POINTER(ctypes.c_double), _P], ctypes.c_int),
    "bgp_mass_quantiles": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, _P, ctypes.POINTER(ctypes.c_double),
                            ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(ctypes.c_double), _P],
                           ctypes.c_int),
    "bgp_radial_profile": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, _P, ctypes.POINTER(ctypes.c_double),
                            ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(ctypes.c_double), _P],
                           ctypes.c_int),
    "bgp_vortex_count": ([ctypes.c_int, ctypes.c_double, _P, ctypes.c_double, ctypes.c_double,
                          ctypes.POINTER(ctypes.c_int), _P], ctypes.c_int),
    "bgp_lll_weight": ([ctypes.c_int, ctypes.c_double, _P, ctypes.c_double, ctypes.c_int,
                        ctypes.POINTER(ctypes.c_double), _P], ctypes.c_int),
    "bgp_resample": ([ctypes.c_int, ctypes.c_int, ctypes.c_double, _P, ctypes.c_int, ctypes.c_double, _P, _P],
                     ctypes.c_int),
    "bgp_k0e": ([ctypes.c_double], ctypes.c_double),
    "bgp_k1e": ([ctypes.c_double], ctypes.c_double),
    "bgp_size_supported": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
}

_lib = None


def lib():
    """The loaded library (loaded on first use)."""
    global _lib
    if _lib is None:
        path = os.environ.get("BECGPP_B200_LIB") or LIB_PATH
        if not os.path.isfile(path):
            raise RuntimeError(f"libbgp.so not built at {path}: run `python -m becgpp_b200.build` "
                               "(there is no CPU fallback)")
        h = ctypes.CDLL(path)
        for name, (args, res) in _SIGS.items():
            f = getattr(h, name)
            f.argtypes = args
            f.restype = res
        if hasattr(h, "bgp_prof_read"):   # profiling builds only
            h.bgp_prof_read.argtypes = [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]
            h.bgp_prof_read.restype = ctypes.c_int
        _lib = h
    return _lib


def exported_symbols():
    return tuple(_SIGS)


def check(rc, what):
    if rc != 0:
        msg = lib().bgp_last_error().decode(errors="replace")
        exc = ValueError if rc in (-1, -5) else RuntimeError
        raise exc(f"{what} failed ({rc}): {msg}")


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("becgpp_b200 needs a CUDA device (B200); none is visible and there is "
                           "no CPU fallback")


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None
