"""ctypes binding of libmf3d.so (the C-ABI declared in include/mf3d.h).

The shared library is built in-tree by macroflow3d_b200/build.py.  Loading it does not need
a GPU; every compute entry point does, and fails with an error status when none is present.
There is no CPU fallback: a missing library raises at load time.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmf3d.so")

MF3D_OK, MF3D_E_INVALID, MF3D_E_CUDA, MF3D_E_NOMEM, MF3D_E_STATE = 0, -1, -2, -3, -4


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double)]


class BC(C.Structure):
    _fields_ = [("type", C.c_int * 6), ("value", C.c_double * 6)]


class SolverConfig(C.Structure):
    _fields_ = [("solver", C.c_int), ("mg_levels", C.c_int), ("mg_pre_smooth", C.c_int),
                ("mg_post_smooth", C.c_int), ("mg_max_cycles", C.c_int), ("mg_coarse_iters", C.c_int),
                ("cg_max_iter", C.c_int), ("cg_check_every", C.c_int), ("cg_rtol", C.c_double),
                ("rtol", C.c_double), ("pin_mode", C.c_int), ("precision", C.c_int),
                ("flexible", C.c_int), ("conv_norm", C.c_int), ("use_graph", C.c_int)]


class SolveResult(C.Structure):
    _fields_ = [("num_iterations", C.c_int), ("converged", C.c_int), ("status", C.c_int),
                ("num_levels", C.c_int), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("true_rel_residual", C.c_double),
                ("b_norm", C.c_double), ("device_ms", C.c_float), ("kernel_launches", C.c_int)]


class KernelTiming(C.Structure):
    _fields_ = [("name", C.c_char * 40), ("ms", C.c_float), ("bytes", C.c_double),
                ("launches_per_iter", C.c_int)]


class BatchTuning(C.Structure):
    _fields_ = [("phase", C.c_int), ("level", C.c_int), ("sweep", C.c_int), ("mode", C.c_int),
                ("path", C.c_int), ("chunks", C.c_int), ("ms_default", C.c_double),
                ("ms_best", C.c_double)]


# every symbol include/mf3d.h declares, with its ctypes signature
_P = C.c_void_p
_G = C.POINTER(Grid)
_B = C.POINTER(BC)
SIGNATURES = {
    "mf3d_last_error": ([], C.c_char_p),
    "mf3d_version": ([], C.c_char_p),
    "mf3d_default_config": ([C.POINTER(SolverConfig)], C.c_int),
    "mf3d_head_solver_create": ([_G, _B, C.POINTER(SolverConfig), _P, C.POINTER(_P)], C.c_int),
    "mf3d_head_solver_destroy": ([_P], C.c_int),
    "mf3d_head_solver_num_levels": ([_P], C.c_int),
    "mf3d_head_solver_coarse_info": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "mf3d_head_solver_device_bytes": ([_P], C.c_longlong),
    "mf3d_head_solver_set_K": ([_P, _P], C.c_int),
    "mf3d_head_solve": ([_P, _P, _P, C.POINTER(SolveResult)], C.c_int),
    "mf3d_head_solver_vcycle": ([_P, _P, _P], C.c_int),
    "mf3d_head_solver_profile": ([_P, C.c_int, C.POINTER(KernelTiming), C.c_int, C.POINTER(C.c_int)],
                                 C.c_int),
    "mf3d_head_solver_setup_launches": ([_P], C.c_int),
    "mf3d_batch_create": ([C.c_int, _G, _B, C.POINTER(SolverConfig), _P, C.POINTER(_P)], C.c_int),
    "mf3d_batch_destroy": ([_P], C.c_int),
    "mf3d_batch_count": ([_P], C.c_int),
    "mf3d_batch_device_bytes": ([_P], C.c_longlong),
    "mf3d_batch_set_K": ([_P, C.POINTER(_P)], C.c_int),
    "mf3d_batch_solve": ([_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(SolveResult)], C.c_int),
    "mf3d_batch_autotune": ([_P, C.c_int, C.POINTER(BatchTuning), C.c_int, C.POINTER(C.c_int)], C.c_int),
    "mf3d_ws_create": ([C.c_ulonglong, C.POINTER(_P)], C.c_int),
    "mf3d_ws_destroy": ([_P], C.c_int),
    "mf3d_ws_num_params": ([_P], C.c_longlong),
    "mf3d_ws_get_params": ([_P, _P], C.c_int),
    "mf3d_ws_set_params": ([_P, _P], C.c_int),
    "mf3d_ws_get_grads": ([_P, _P], C.c_int),
    "mf3d_ws_train_step": ([_P, _G, _B, C.c_int, C.POINTER(_P), C.POINTER(_P), C.c_float,
                            C.POINTER(C.c_double), _P], C.c_int),
    "mf3d_ws_eval": ([_P, _G, _B, C.c_int, C.POINTER(_P), C.POINTER(_P), C.POINTER(C.c_double), _P], C.c_int),
    "mf3d_ws_predict": ([_P, _G, _B, _P, _P, _P], C.c_int),
    "mf3d_nn_conv3d": ([_G, C.c_int, C.c_int, _P, _P, _P, C.c_int, _P, C.c_int, _P, _P], C.c_int),
    "mf3d_nn_flip_weights": ([C.c_int, C.c_int, _P, _P, _P], C.c_int),
    "mf3d_nn_conv3d_wgrad": ([_G, C.c_int, C.c_int, _P, _P, _P, _P, _P], C.c_int),
    "mf3d_velocity_from_head": ([_G, _B, _P, _P, C.c_int, _P, _P, _P, _P], C.c_int),
    "mf3d_velocity_mass_balance": ([_G, _B, _P, _P, _P, _P, _P, C.POINTER(C.c_double), _P], C.c_int),
    "mf3d_velocity_mass_balance_noalloc": ([_G, _B, _P, _P, _P, _P, _P, C.POINTER(C.c_double), _P], C.c_int),
    "mf3d_head_solver_set_time_budget": ([_P, C.c_double], C.c_int),
    "mf3d_diag_bounded_wait": ([C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "mf3d_velocity_diagnostics": ([_G, C.c_int, _P, _P, _P, _P, _P, _P, C.POINTER(C.c_double), _P], C.c_int),
    "mf3d_apply_A": ([_G, _B, C.c_int, _P, _P, _P, _P], C.c_int),
    "mf3d_gsrb": ([_G, _B, C.c_int, _P, _P, _P, C.c_int, _P], C.c_int),
    "mf3d_residual": ([_G, _B, C.c_int, _P, _P, _P, _P, _P], C.c_int),
    "mf3d_restrict": ([_G, _P, _P, _P], C.c_int),
    "mf3d_prolong_add": ([_G, _P, _P, _P], C.c_int),
    "mf3d_coarsen_K": ([_G, _P, _P, _P], C.c_int),
    "mf3d_build_rhs": ([_G, _B, _P, _P, _P], C.c_int),
    "mf3d_init_head_guess": ([_G, _B, _P, _P], C.c_int),
    "mf3d_kfield_modes": ([C.c_ulonglong, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                           C.POINTER(C.c_double)], C.c_int),
    "mf3d_kfield_eval": ([_G, C.c_int, _P, C.c_double, C.c_double, C.c_int, _P, _P], C.c_int),
}

_lib = None


class Mf3dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mf3d error {code}: {msg}")
        self.code = code


def lib():
    """Loads libmf3d.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m macroflow3d_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != MF3D_OK:
        raise Mf3dError(rc, lib().mf3d_last_error().decode())
