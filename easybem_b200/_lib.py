"""ctypes binding of libeasybem_gpu.so (the C ABI of include/easybem_gpu.h).

The shared library is built in-tree by ``easybem_b200.build``. There is no
CPU fallback: if the library is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# EASYBEM_B200_LIB may name another build of the library (e.g. for A/B timing)
LIB_PATH = os.environ.get("EASYBEM_B200_LIB") or os.path.join(HERE, "libeasybem_gpu.so")

EB_OK = 0
EB_ERR_INVALID = 1
EB_ERR_MESH = 2
EB_ERR_CUDA = 3
EB_ERR_NOMEM = 4
EB_ERR_TIMEOUT = 5
EB_ERR_STATE = 6
EB_ERR_NOT_CONVERGED = 7

EB_PREC_FP64 = 0
EB_PREC_MIXED = 1

_STATUS_NAMES = {1: "invalid argument", 2: "invalid mesh", 3: "CUDA error", 4: "out of memory",
                 5: "timeout", 6: "bad state", 7: "not converged"}

# name -> (restype, argtypes); every entry point returns an int status except
# the two string accessors.
_dp = ctypes.c_void_p
_SIGNATURES = {
    "eb_version": (ctypes.c_char_p, []),
    "eb_last_error": (ctypes.c_char_p, []),
    "eb_mesh_create": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.POINTER(_dp)]),
    "eb_mesh_destroy": (ctypes.c_int, [_dp]),
    "eb_mesh_info": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "eb_mesh_finalize_bytes": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_longlong)]),
    "eb_far_engine_costs": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double)]),
    "eb_mesh_cell_pairs": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "eb_sym_plan": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.c_void_p, ctypes.c_void_p]),
    "eb_set_device_topology_min": (ctypes.c_int, [ctypes.c_int]),
    "eb_get_device_topology_min": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "eb_mesh_topology_on_device": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_int)]),
    "eb_mesh_set_far_engine": (ctypes.c_int, [_dp, ctypes.c_int]),
    "eb_mesh_get_far_engine": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "eb_mesh_near_field_bytes": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_longlong),
                                                ctypes.POINTER(ctypes.c_longlong)]),
    "eb_release_cached_memory": (ctypes.c_int, []),
    "eb_cached_memory_bytes": (ctypes.c_int, [ctypes.POINTER(ctypes.c_longlong)]),
    "eb_apply_sl_p0": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp]),
    "eb_apply_dl_p1": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp]),
    "eb_apply_sl_dl": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp, _dp, _dp]),
    "eb_apply_sl_dl_device": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp, _dp, _dp, _dp]),
    "eb_apply_sl_dl_noalloc": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp, _dp, _dp, _dp]),
    "eb_apply_sl_p1": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp]),
    "eb_apply_sl_p1_device": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp, _dp]),
    "eb_apply_hypersingular": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp]),
    "eb_apply_hypersingular_device": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp, _dp]),
    "eb_quadrature": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp, _dp,
                                     ctypes.POINTER(ctypes.c_int), _dp, _dp, _dp]),
    "eb_measure_fp32_peak": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "eb_measure_rsqrt_peak": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "eb_set_profiling": (ctypes.c_int, [_dp, ctypes.c_int]),
    "eb_dirichlet_rhs": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp]),
    "eb_dirichlet_rhs_prec": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int, _dp, _dp]),
    "eb_evaluate_potential": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp]),
    "eb_solve_options_default": (None, [_dp]),
    "eb_apply_near_precond": (ctypes.c_int, [_dp, _dp, _dp]),
    "eb_solve_sl": (ctypes.c_int, [ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp]),
    "eb_solver_create": (ctypes.c_int, [_dp, ctypes.POINTER(_dp)]),
    "eb_solver_destroy": (ctypes.c_int, [_dp]),
    "eb_solver_add": (ctypes.c_int, [_dp, _dp, ctypes.c_int, _dp, _dp]),
    "eb_solver_step": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_int)]),
    "eb_solver_done": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "eb_solver_result": (ctypes.c_int, [_dp, ctypes.c_int, _dp, _dp]),
    "eb_solver_remove": (ctypes.c_int, [_dp, ctypes.c_int]),
    "eb_solver_bytes_per_system": (ctypes.c_int, [_dp, _dp, ctypes.POINTER(ctypes.c_longlong)]),
    "eb_batch_create": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_dp)]),
    "eb_batch_destroy": (ctypes.c_int, [_dp]),
    "eb_batch_apply": (ctypes.c_int, [_dp, _dp, _dp, _dp]),
    "eb_read_surface_txt": (ctypes.c_int, [ctypes.c_char_p, _dp, _dp, _dp, _dp, _dp]),
    "eb_read_netgen_vol": (ctypes.c_int, [ctypes.c_char_p, _dp, _dp, _dp, _dp, _dp]),
    "eb_mesh_refine": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "eb_batch_create_sl_dl": (ctypes.c_int, [ctypes.c_int, _dp, ctypes.c_int, ctypes.POINTER(_dp)]),
    "eb_batch_apply_sl_dl": (ctypes.c_int, [_dp, _dp, _dp, _dp, _dp, _dp]),
    "eb_batch_info": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_longlong)]),
    "eb_server_create": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, _dp, ctypes.POINTER(_dp)]),
    "eb_server_destroy": (ctypes.c_int, [_dp]),
    "eb_server_submit": (ctypes.c_int, [_dp, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int, _dp,
                                        ctypes.POINTER(ctypes.c_longlong)]),
    "eb_server_step": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "eb_server_poll": (ctypes.c_int, [_dp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int)]),
    "eb_server_result": (ctypes.c_int, [_dp, ctypes.c_longlong, _dp, _dp, _dp]),
    "eb_server_release": (ctypes.c_int, [_dp, ctypes.c_longlong]),
    "eb_server_usage": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "eb_server_stats": (ctypes.c_int, [_dp, _dp, ctypes.c_int]),
    "eb_last_kernel_ms": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "eb_mesh_set_plan": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int]),
    "eb_mesh_get_plan": (ctypes.c_int, [_dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "eb_autotune": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]),
    "eb_plan_table_save": (ctypes.c_int, [ctypes.c_char_p]),
    "eb_plan_table_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "eb_plan_table_clear": (ctypes.c_int, []),
}


class SolveOptions(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("inner_tol", ctypes.c_double), ("restart", ctypes.c_int),
                ("max_cycles", ctypes.c_int), ("max_iterations", ctypes.c_int), ("inner_precision", ctypes.c_int),
                ("precond", ctypes.c_int), ("rhs_precision", ctypes.c_int)]


class SolveStats(ctypes.Structure):
    _fields_ = [("converged", ctypes.c_int), ("cycles", ctypes.c_int), ("iterations", ctypes.c_int),
                ("rel_residual", ctypes.c_double)]


class EasyBemError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"easybem error {status} ({_STATUS_NAMES.get(status, '?')}): {message}")
        self.status = status


_LIB = None


def lib():
    """Loads the CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m easybem_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            if hasattr(L, name):
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
        _LIB = L
    return _LIB


def check(status: int):
    if status != EB_OK:
        raise EasyBemError(status, lib().eb_last_error().decode(errors="replace"))


def exported_symbols():
    """Names declared in include/easybem_gpu.h that the library must export."""
    return list(_SIGNATURES)
