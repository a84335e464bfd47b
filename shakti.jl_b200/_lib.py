"""ctypes binding of libshakti_b200.so (include/shakti_b200.h).

There is no fallback: if the shared library is missing or CUDA is unavailable, every entry point
raises.  Build the library with `python shakti.jl_b200/build.py` (or __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libshakti_b200.so"
DP = C.POINTER(C.c_double)

# shk_status
OK, NOT_CONVERGED, BREAKDOWN, BAD_ARG, CUDA_ERROR, NOT_BOUND = range(6)
STATUS_NAMES = {0: "ok", 1: "not converged", 2: "breakdown", 3: "bad argument", 4: "cuda error", 5: "not bound"}

PARAM_NAMES = ["rho_w", "rho_sw", "rho_i", "g", "nu", "n", "omega", "L", "br", "lr", "ct", "cw", "p_atm",
               "b_min", "b_max", "e_v"]
CENTER_FIELDS = ["h", "pw", "po", "b", "beta", "abs_ub", "mdot", "shear", "potential", "sensible", "Re", "K",
                 "G", "zb", "zs", "H", "ieb", "lambda_", "A_visc", "N", "mask"]
XFACE_FIELDS = ["dhdx", "q_x", "Re_x", "b_x", "ub_x", "taub_x", "dpwdx", "valid_x"]
YFACE_FIELDS = ["dhdy", "q_y", "Re_y", "b_y", "ub_y", "taub_y", "dpwdy", "valid_y"]
STATE_FIELDS = CENTER_FIELDS + XFACE_FIELDS + YFACE_FIELDS


class shk_params(C.Structure):
    _fields_ = [(n, C.c_double) for n in PARAM_NAMES]


class shk_state(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in STATE_FIELDS]


class shk_sliding_law(C.Structure):
    _fields_ = [("kind", C.c_int), ("C", C.c_double), ("v0", C.c_double), ("Cx", C.c_void_p), ("Cy", C.c_void_p)]


class shk_melt_input(C.Structure):
    _fields_ = [("kind", C.c_int)] + [(n, C.c_double) for n in (
        "t_start", "period", "omega", "amplitude", "offset", "i_min", "seconds_per_year")] + [("base", C.c_void_p)]


class shk_cg_opts(C.Structure):
    _fields_ = [("precond", C.c_int), ("cheb_degree", C.c_int), ("cheb_nsteps", C.c_int), ("stop_rule", C.c_int),
                ("precision", C.c_int), ("max_refine", C.c_int), ("atol", C.c_double), ("rtol", C.c_double),
                ("inner_rtol", C.c_double), ("itmax", C.c_long), ("inner_itmax", C.c_long)]


class shk_cg_stats(C.Structure):
    _fields_ = [("niter", C.c_long), ("status", C.c_int), ("refinements", C.c_int), ("rnorm0", C.c_double),
                ("rnorm", C.c_double), ("lambda_min", C.c_double), ("lambda_max", C.c_double),
                ("bounds_valid", C.c_int)]


class shk_picard_opts(C.Structure):
    _fields_ = [("iters", C.c_int), ("check_every", C.c_int), ("tol", C.c_double), ("alpha", C.c_double)]


class shk_picard_stats(C.Structure):
    _fields_ = [("converged", C.c_int), ("last_iter", C.c_int), ("cg_iters_total", C.c_long),
                ("cg_solves", C.c_int), ("cg_breakdowns", C.c_int), ("max_dh", C.c_double), ("max_h", C.c_double)]


class shk_ensemble_stats(C.Structure):
    _fields_ = [("steps", C.c_longlong), ("steps_converged", C.c_longlong), ("picard_iters", C.c_longlong),
                ("cg_iters", C.c_longlong), ("last_picard_iters", C.c_int), ("last_converged", C.c_int),
                ("march_th", C.c_int), ("pad", C.c_int), ("max_dh", C.c_double), ("max_h", C.c_double)]


# Every symbol include/shakti_b200.h declares, with (restype, argtypes).
VP = C.c_void_p
FP = C.POINTER(C.c_float)
SIGNATURES = {
    "shk_version": (C.c_int, []),
    "shk_status_string": (C.c_char_p, [C.c_int]),
    "shk_create": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, VP, C.POINTER(VP)]),
    "shk_destroy": (C.c_int, [VP]),
    "shk_last_error": (C.c_char_p, [VP]),
    "shk_set_stream": (C.c_int, [VP, VP]),
    "shk_set_params": (C.c_int, [VP, C.POINTER(shk_params)]),
    "shk_set_sliding_law": (C.c_int, [VP, C.POINTER(shk_sliding_law)]),
    "shk_set_schemes": (C.c_int, [VP, C.c_int, C.c_int]),
    "shk_bind_state": (C.c_int, [VP, C.POINTER(shk_state)]),
    "shk_set_initial_conditions": (C.c_int, [VP]),
    "shk_assemble": (C.c_int, [VP, C.c_int, C.c_double]),
    "shk_export_mfls": (C.c_int, [VP, VP, VP, VP, VP, VP, VP]),
    "shk_matvec": (C.c_int, [VP, VP, VP]),
    "shk_update_chebyshev_bounds": (C.c_int, [VP, C.c_int, VP, DP, C.POINTER(C.c_int)]),
    "shk_get_chebyshev_bounds": (C.c_int, [VP, DP, DP]),
    "shk_set_chebyshev_bounds": (C.c_int, [VP, C.c_double, C.c_double]),
    "shk_chebyshev_apply": (C.c_int, [VP, C.c_int, VP, VP]),
    "shk_cg_solve": (C.c_int, [VP, C.POINTER(shk_cg_opts), C.POINTER(shk_cg_stats)]),
    "shk_solve_elliptic": (C.c_int, [VP, C.POINTER(shk_cg_opts), C.POINTER(shk_cg_stats)]),
    "shk_solve_parabolic": (C.c_int, [VP, C.c_double, C.POINTER(shk_cg_opts), C.POINTER(shk_cg_stats)]),
    "shk_picard_tail": (C.c_int, [VP]),
    "shk_relax_h": (C.c_int, [VP, C.c_double, VP]),
    "shk_picard_solve": (C.c_int, [VP, C.POINTER(shk_picard_opts), C.POINTER(shk_cg_opts),
                                   C.POINTER(shk_picard_stats)]),
    "shk_parabolic_step": (C.c_int, [VP, C.c_double, C.POINTER(shk_cg_opts), C.POINTER(shk_cg_stats)]),
    "shk_step_b": (C.c_int, [VP, C.c_double]),
    "shk_update_ieb": (C.c_int, [VP, C.POINTER(shk_melt_input), C.c_double]),
    "shk_step": (C.c_int, [VP, C.c_int, C.c_double, C.c_double, C.POINTER(shk_melt_input),
                           C.POINTER(shk_picard_opts), C.POINTER(shk_cg_opts), C.POINTER(shk_picard_stats)]),
    "shk_run": (C.c_int, [VP, C.c_int, C.c_double, C.c_int, DP, C.POINTER(shk_melt_input),
                          C.POINTER(shk_picard_opts), C.POINTER(shk_cg_opts), C.POINTER(shk_picard_stats)]),
    "shk_kernel_launches": (C.c_long, [VP]),
    "shk_cg_solve_static": (C.c_int, [C.c_int, C.c_int, VP, VP, VP, VP, VP, C.POINTER(shk_cg_opts),
                                      C.POINTER(shk_cg_stats), VP]),
    "shk_nn_conv3x3": (C.c_int, [VP, VP, FP, VP, FP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, VP]),
    "shk_nn_conv3x3_wgrad": (C.c_int, [VP, VP, FP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, VP]),
    "shk_nn_conv_fault": (C.c_int, [C.POINTER(C.c_int)]),
    "shk_nn_relu_grad": (C.c_int, [FP, VP, VP, FP, C.c_longlong, C.c_int, C.c_int, VP]),
    "shk_nn_pool2": (C.c_int, [VP, VP, C.c_int, C.c_int, C.c_int, C.c_int, VP]),
    "shk_nn_pool2_grad": (C.c_int, [FP, FP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, VP]),
    "shk_nn_up2_add": (C.c_int, [VP, VP, VP, C.c_int, C.c_int, C.c_int, C.c_int, VP]),
    "shk_nn_up2_grad": (C.c_int, [FP, FP, C.c_int, C.c_int, C.c_int, C.c_int, VP]),
    "shk_nn_axpy": (C.c_int, [FP, FP, C.c_longlong, C.c_int, VP]),
    "shk_nn_mse": (C.c_int, [FP, FP, FP, FP, FP, C.c_longlong, C.c_int, C.c_float, VP]),
    "shk_nn_adam": (C.c_int, [FP, FP, FP, FP, VP, VP, C.c_longlong, C.c_int, C.c_int, C.c_float, C.c_float,
                              C.c_float, C.c_float, C.c_int, VP]),
    "shk_nn_wcast": (C.c_int, [FP, VP, VP, C.c_longlong, C.c_int, C.c_int, VP]),
    "shk_nn_zero": (C.c_int, [FP, C.c_longlong, VP]),
    "shk_nn_pack_state": (C.c_int, [C.POINTER(shk_state), C.c_int, C.c_int, C.c_int, C.c_int, FP, VP, VP]),
    "shk_nn_apply_increment": (C.c_int, [FP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, VP, VP, VP, VP]),
    "shk_initial_residual": (C.c_int, [VP, DP, DP]),
    "shk_residual_of": (C.c_int, [VP, VP, DP, DP]),
    "shk_smooth_guess": (C.c_int, [VP, VP, VP, C.c_int, C.c_double]),
    "shk_set_cg_warm_start": (C.c_int, [VP, VP]),
    "shk_ensemble_create": (C.c_int, [C.c_int, C.POINTER(VP), VP, C.POINTER(VP)]),
    "shk_ensemble_destroy": (C.c_int, [VP]),
    "shk_ensemble_set_snapshots": (C.c_int, [VP, C.POINTER(VP)]),
    "shk_ensemble_last_error": (C.c_char_p, [VP]),
    "shk_ensemble_autotune": (C.c_int, [VP, C.c_int, C.POINTER(C.c_int)]),
    "shk_ensemble_run": (C.c_int, [VP, C.c_double, C.c_int, C.POINTER(shk_picard_opts), C.POINTER(shk_cg_opts),
                                   C.POINTER(shk_ensemble_stats)]),
    "shk_ensemble_launch_counts": (C.c_int, [VP, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                             C.POINTER(C.c_int)]),
}

_LIB = None


class ShaktiError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def load(path: Path | None = None):
    """Load the CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: the CUDA library has not been built "
                          "(run `python shakti.jl_b200/build.py`); there is no CPU fallback")
    L = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = L
    return L


def check(ctx, rc: int, allow=(OK,)) -> int:
    if rc in allow:
        return rc
    msg = load().shk_last_error(ctx)
    raise ShaktiError(rc, msg.decode() if msg else "")


def cuda_stream_handle():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def default_cg_opts(**kw) -> shk_cg_opts:
    sq = math.sqrt(2.220446049250313e-16)
    o = shk_cg_opts(precond=0, cheb_degree=4, cheb_nsteps=15, stop_rule=0, precision=0, max_refine=0,
                    atol=sq, rtol=sq, inner_rtol=0.0, itmax=0, inner_itmax=0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o
