"""ctypes binding of ``libifos_b200.so`` (declared in ``include/ifos_gpu.h``).

The library is the product: this module only loads it and declares the
entry points.  There is no CPU fallback -- if the shared library cannot be
built or loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libifos_b200.so")
MAX_L = 8
NS, NG, NF = 6, 10, 12

IFOS_OK, IFOS_ERR_ARG, IFOS_ERR_CUDA, IFOS_ERR_NOMEM, IFOS_ERR_UNSTABLE, IFOS_ERR_STATE = range(6)
SNAP_FORMATS = {"fp32": 0, "bf16": 1, "fp16": 2, "fp16s": 3, "i16s": 4}

# every symbol include/ifos_gpu.h declares
EXPORTS = [
    "ifos_params_default", "ifos_ctx_create", "ifos_ctx_destroy", "ifos_last_error", "ifos_ctx_bytes",
    "ifos_model_upload", "ifos_shot_setup", "ifos_forward", "ifos_adjoint", "ifos_stage_adjoint",
    "ifos_fetch_sections", "ifos_fetch_grads", "ifos_grad_sum", "ifos_forward_steps", "ifos_fetch_fields",
    "ifos_dot_f64", "ifos_calc_res", "ifos_fd_coeffs", "ifos_cpml_profiles", "ifos_kernel_timing",
    "ifos_kernel_times", "ifos_grad_sum_device", "ifos_set_stream", "ifos_dot_f64_noalloc", "ifos_last_ms", "ifos_launch_count",
    "ifos_sync", "ifos_trkill_table", "ifos_time_window", "ifos_set_option", "ifos_get_option",
    "ifos_residual_adjoint", "ifos_fetch_snapshot", "ifos_opt_step", "ifos_timedomain_filt",
    "ifos_taper_grad_shot", "ifos_taper_grad_coeff", "ifos_lbfgs_core", "ifos_median_smooth", "ifos_mat_change_test", "ifos_fetch_sections_async",
    "ifos_fetch_grads_async", "ifos_fetch_wait", "ifos_host_alloc", "ifos_host_free", "ifos_status",
]
OPTIONS = {"graphs": 0, "pdl": 1, "blocks_per_sm": 2, "tile_order": 3, "wait_limit": 4}


class IfosParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nt", C.c_int),
        ("dh", C.c_float), ("dt", C.c_float),
        ("fdorder", C.c_int), ("maxrelerror", C.c_int),
        ("fw", C.c_int), ("free_surf", C.c_int), ("boundary", C.c_int),
        ("vppml", C.c_float), ("fpml", C.c_float), ("npower", C.c_float), ("k_max_pml", C.c_float),
        ("L", C.c_int), ("f_ref", C.c_float), ("tau", C.c_float), ("fl", C.c_float * MAX_L),
        ("wavetype", C.c_int), ("acoustic", C.c_int), ("parameterization", C.c_int), ("velocity", C.c_int),
        ("seismo", C.c_int), ("source_type", C.c_int), ("adjoint_type", C.c_int), ("dtinv", C.c_int),
        ("hi_order_corrected", C.c_int), ("precision", C.c_int), ("snap_format", C.c_int),
        ("max_shots", C.c_int), ("max_models", C.c_int), ("max_src", C.c_int), ("max_rec", C.c_int),
        ("grad_acc64", C.c_int), ("mu_corrected", C.c_int),
    ]


class IfosWindow(C.Structure):
    _fields_ = [("tw_ind", C.c_int), ("picks", C.POINTER(C.c_float)), ("gamma", C.c_float),
                ("twl_plus", C.c_float), ("twl_minus", C.c_float)]


class IfosMatChange(C.Structure):
    """ifos_mat_change of include/ifos_gpu.h (field order as declared)."""
    _fields_ = [("eps_scale", C.c_float), ("iter", C.c_int), ("itest", C.c_int), ("inv_vp_iter", C.c_int),
                ("inv_vs_iter", C.c_int), ("inv_rho_iter", C.c_int), ("lbfgs_unnormalised", C.c_int),
                ("vp_lower", C.c_float), ("vp_upper", C.c_float), ("vs_lower", C.c_float), ("vs_upper", C.c_float),
                ("rho_lower", C.c_float), ("rho_upper", C.c_float), ("vp_vs_ratio", C.c_float),
                ("limit_update", C.c_int), ("s_vp", C.c_float), ("s_vs", C.c_float), ("s_rho", C.c_float),
                ("lbfgs_npar", C.c_int), ("vs_avg", C.c_float), ("rho_avg", C.c_float), ("vp_avg", C.c_float)]


class IfosError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ifos error {code}: {msg}")
        self.code = code


_lib = None


def ensure_built() -> str:
    from . import build as _build
    return _build.build()


def load():
    """Load the shared library, building it first when it is missing or stale."""
    global _lib
    if _lib is not None:
        return _lib
    path = ensure_built()
    lib = C.CDLL(path)
    vp = C.c_void_p
    FP = C.POINTER(C.c_float)
    IP = C.POINTER(C.c_int)
    DP = C.POINTER(C.c_double)
    P = C.POINTER(IfosParams)
    sig = {
        "ifos_params_default": (None, [P]),
        "ifos_ctx_create": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(vp)]),
        "ifos_ctx_destroy": (C.c_int, [vp]),
        "ifos_last_error": (C.c_char_p, [vp]),
        "ifos_ctx_bytes": (C.c_size_t, [P, C.c_int]),
        "ifos_model_upload": (C.c_int, [vp, C.c_int, FP, FP, FP, FP, FP]),
        "ifos_shot_setup": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, FP, FP, C.c_int, IP]),
        "ifos_forward": (C.c_int, [vp, C.c_int, C.c_int, FP]),
        "ifos_adjoint": (C.c_int, [vp, C.c_int, FP, FP]),
        "ifos_stage_adjoint": (C.c_int, [vp, C.c_int, FP]),
        "ifos_fetch_sections": (C.c_int, [vp, C.c_int, FP]),
        "ifos_fetch_grads": (C.c_int, [vp, C.c_int, FP]),
        "ifos_grad_sum": (C.c_int, [vp, C.c_int, FP]),
        "ifos_forward_steps": (C.c_int, [vp, C.c_int, FP]),
        "ifos_fetch_fields": (C.c_int, [vp, C.c_int, FP]),
        "ifos_dot_f64": (C.c_int, [vp, vp, vp, C.c_size_t, C.c_int, DP]),
        "ifos_calc_res": (C.c_int, [vp, C.c_int, FP, FP, FP, DP, DP]),
        "ifos_fd_coeffs": (C.c_int, [P, FP]),
        "ifos_cpml_profiles": (C.c_int, [P, FP]),
        "ifos_kernel_timing": (C.c_int, [vp, C.c_int]),
        "ifos_kernel_times": (C.c_int, [vp, DP, C.POINTER(C.c_longlong), C.c_int]),
        "ifos_grad_sum_device": (C.c_int, [vp, C.c_int, vp]),
        "ifos_set_stream": (C.c_int, [vp, vp]),
        "ifos_dot_f64_noalloc": (C.c_int, [C.c_int, vp, vp, C.c_size_t, vp, DP]),
        "ifos_last_ms": (C.c_double, [vp]),
        "ifos_launch_count": (C.c_longlong, [vp]),
        "ifos_sync": (C.c_int, [vp]),
        "ifos_trkill_table": (C.c_int, [vp, C.c_int, IP, IP, C.c_int, FP, FP, C.c_float, C.c_float, IP]),
        "ifos_time_window": (C.c_int, [vp, C.c_int, C.c_int, FP, C.c_int, FP, C.c_float, C.c_float, C.c_float,
                                       C.POINTER(C.c_ubyte)]),
        "ifos_set_option": (C.c_int, [vp, C.c_int, C.c_int]),
        "ifos_get_option": (C.c_int, [vp, C.c_int, IP]),
        "ifos_residual_adjoint": (C.c_int, [vp, C.c_int, FP, IP, C.POINTER(IfosWindow), DP, DP]),
        "ifos_fetch_snapshot": (C.c_int, [vp, C.c_int, C.c_int, FP]),
        "ifos_opt_step": (C.c_int, [FP, FP, C.c_int, FP]),
        "ifos_timedomain_filt": (C.c_int, [vp, FP, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_float]),
        "ifos_taper_grad_shot": (C.c_int, [vp, C.c_int, FP, C.c_float, C.c_int, C.c_int, C.c_uint]),
        "ifos_taper_grad_coeff": (C.c_int, [vp, C.c_int, C.c_uint, FP]),
        "ifos_lbfgs_core": (C.c_int, [vp, C.c_int, C.c_int, C.c_size_t, FP, FP, FP, FP, FP, FP, C.c_int]),
        "ifos_median_smooth": (C.c_int, [vp, FP, C.c_int]),
        "ifos_fetch_sections_async": (C.c_int, [vp, C.c_int, FP]),
        "ifos_fetch_grads_async": (C.c_int, [vp, C.c_int, FP]),
        "ifos_fetch_wait": (C.c_int, [vp]),
        "ifos_status": (C.c_int, [vp]),
        "ifos_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
        "ifos_host_free": (C.c_int, [C.c_void_p]),
        "ifos_mat_change_test": (C.c_int, [vp, C.POINTER(IfosMatChange), FP, FP, FP, FP, FP, FP, FP, FP, FP, FP, FP,
                                           FP, FP, FP, IP]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
