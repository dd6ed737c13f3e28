"""ctypes binding of the C ABI in include/tps.h (libtps.so, built in-tree).

The library is the only compute path: if it is missing or fails to load,
every entry point raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtps.so")

TPS_OK = 0
STATUS_NAMES = {
    0: "TPS_OK", 1: "TPS_ERR_INVALID", 2: "TPS_ERR_CUDA", 3: "TPS_ERR_ALLOC",
    4: "TPS_ERR_NOT_CONVERGED", 5: "TPS_ERR_BREAKDOWN", 6: "TPS_ERR_NONFINITE",
    7: "TPS_ERR_UNSUPPORTED", 8: "TPS_ERR_TIMEOUT",
}
TPS_F64, TPS_F32, TPS_TF32, TPS_TF32X3 = 0, 1, 2, 3
VCYCLE_F64, VCYCLE_F32, VCYCLE_F64_ROUNDED, VCYCLE_TF32, VCYCLE_TF32X3 = 0, 1, 2, 3, 4
DRIVER_CG, DRIVER_GMRES = 0, 1
SMOOTHER_VARIANTS = 5  # TPS_SMOOTHER_VARIANTS
SMOOTHER_FUSED, SMOOTHER_SEPARATE, SMOOTHER_GLOBAL, SMOOTHER_EXACT, SMOOTHER_ADDITIVE = 0, 1, 2, 3, 4
MAX_HISTORY = 256


class TpsProblem(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("degree", ctypes.c_int), ("n_coarse", ctypes.c_int),
                ("n_levels", ctypes.c_int), ("relaxation", ctypes.c_double),
                ("kappa", ctypes.POINTER(ctypes.c_double)), ("device", ctypes.c_int)]


class TpsSolveOpts(ctypes.Structure):
    _fields_ = [("driver", ctypes.c_int), ("precision", ctypes.c_int), ("symmetric", ctypes.c_int),
                ("max_iter", ctypes.c_int), ("rel_tol", ctypes.c_double),
                ("abs_tol", ctypes.c_double), ("use_graph", ctypes.c_int)]


class TpsReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("initial_residual", ctypes.c_double), ("final_residual", ctypes.c_double),
                ("history", ctypes.c_double * MAX_HISTORY), ("time_ms", ctypes.c_double)]


class TpsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

# (name, restype, argtypes) of every exported entry point of include/tps.h
_VP = ctypes.c_void_p
SIGNATURES = [
    ("tps_create", ctypes.c_int, [ctypes.POINTER(TpsProblem), ctypes.POINTER(_VP)]),
    ("tps_destroy", ctypes.c_int, [_VP]),
    ("tps_last_error", ctypes.c_char_p, [_VP]),
    ("tps_level_info", ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int)]),
    ("tps_laplace_vmult", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP]),
    ("tps_smoother_step", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, ctypes.c_int,
                                         ctypes.c_int, _VP]),
    ("tps_smoother_step_variant", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, _VP]),
    ("tps_prolongate_add", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP]),
    ("tps_restrict_add", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP]),
    ("tps_vcycle", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP]),
    ("tps_solve_opts_default", None, [ctypes.POINTER(TpsSolveOpts)]),
    ("tps_solve", ctypes.c_int, [_VP, ctypes.POINTER(TpsSolveOpts), _VP, _VP,
                                 ctypes.POINTER(TpsReport), _VP]),
    ("tps_solve_host", ctypes.c_int, [_VP, ctypes.POINTER(TpsSolveOpts), _VP, _VP,
                                      ctypes.POINTER(TpsReport)]),
    ("tps_solve_host_guess", ctypes.c_int, [_VP, ctypes.POINTER(TpsSolveOpts), _VP, _VP, _VP,
                                            ctypes.POINTER(TpsReport)]),
    ("tps_solve_host_many", ctypes.c_int, [_VP, ctypes.POINTER(TpsSolveOpts), ctypes.c_int,
                                           ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(TpsReport)]),
    ("tps_time_smoother", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double), _VP]),
    ("tps_set_kappa", ctypes.c_int, [_VP, _VP, ctypes.c_int]),
    ("tps_mass_vmult", ctypes.c_int, [_VP, _VP, _VP, _VP]),
    ("tps_assemble_rhs", ctypes.c_int, [_VP, ctypes.c_int, _VP, _VP, _VP]),
    ("tps_adjoint", ctypes.c_int, [_VP, ctypes.POINTER(TpsSolveOpts), _VP, _VP, _VP, _VP,
                                   ctypes.POINTER(TpsReport), _VP]),
    ("tps_cell_energy", ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    ("tps_restrict_add_noalloc", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, _VP, _VP, _VP]),
    ("tps_fmg", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_VP), ctypes.POINTER(_VP), _VP,
                               ctypes.POINTER(TpsReport), _VP]),
    ("tps_autotune", ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    ("tps_set_operator_layers", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("tps_get_operator_layers", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    ("tps_smoother_variants", ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    ("tps_set_smoother_variant", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("tps_get_smoother_variant", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    ("tps_set_smoother_kind", ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_double]),
    ("tps_device_status", ctypes.c_int, [_VP]),
    ("tps_selftest_wait_timeout", ctypes.c_int, [_VP, ctypes.c_longlong, _VP]),
    ("tps_inject_alloc_failure", None, [ctypes.c_int]),
    ("tps_check_colouring", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("tps_batch_create", ctypes.c_int, [ctypes.POINTER(TpsProblem), ctypes.c_int, ctypes.POINTER(_VP)]),
    ("tps_batch_destroy", ctypes.c_int, [_VP]),
    ("tps_batch_last_error", ctypes.c_char_p, [_VP]),
    ("tps_batch_system", ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(_VP)]),
    ("tps_batch_solve", ctypes.c_int, [_VP, ctypes.POINTER(TpsSolveOpts), ctypes.POINTER(_VP),
                                       ctypes.POINTER(_VP), ctypes.POINTER(TpsReport), _VP]),
]


def lib():
    """Load libtps.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"native library {LIB_PATH} is missing; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, handle=None):
    if status != TPS_OK:
        msg = lib().tps_last_error(handle)
        raise TpsError(status, msg.decode() if msg else "")
