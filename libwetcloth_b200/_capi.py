"""ctypes binding of libwcgpu.so (include/wetcloth_gpu.h).

The CUDA library is the only implementation: if it is missing or cannot be
loaded this module raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwcgpu.so")

_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_longlong)
_I = ctypes.POINTER(ctypes.c_int)

WCG_OK = 0
WCG_ERR_ARG = 1
WCG_ERR_CUDA = 2
WCG_ERR_NOT_CONVERGED = 3
WCG_ERR_DEVICE = 4
WCG_ERR_STATE = 5
WCG_ERR_UNSUPPORTED = 6
WCG_FP64 = 0
WCG_FP32_REFINE = 1
WCG_SOLVER_MIC0 = 0
WCG_SOLVER_MG = 1


class WcgParams(ctypes.Structure):
    _fields_ = [
        ("dx", ctypes.c_double),
        ("gravity", ctypes.c_double * 3),
        ("liquid_density", ctypes.c_double),
        ("flip_coeff", ctypes.c_double),
        ("liquid_boundary_friction", ctypes.c_double),
        ("box_center", ctypes.c_double * 3),
        ("box_half", ctypes.c_double * 3),
        ("box_radius", ctypes.c_double),
        ("walls", ctypes.c_int),
        ("criterion", ctypes.c_double),
        ("maxiters", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("refine_inner_tol", ctypes.c_double),
        ("max_refinements", ctypes.c_int),
        ("solver", ctypes.c_int),
        ("viscosity", ctypes.c_double),
        ("viscosity_substeps", ctypes.c_int),
        ("elasto_flip_coeff", ctypes.c_double),
        ("elasto_flip_asym_coeff", ctypes.c_double),
        ("elasto_advect_coeff", ctypes.c_double),
        ("drag_viscosity", ctypes.c_double),
        ("correction_strength", ctypes.c_double),
        ("correction_step", ctypes.c_int),
        ("correction_multiplier", ctypes.c_double),
        ("correction_seed", ctypes.c_ulonglong),
        ("viscosity_implicit", ctypes.c_int),
        ("viscosity_criterion", ctypes.c_double),
        ("particle_merge", ctypes.c_int),
        ("merge_seed", ctypes.c_ulonglong),
        ("particle_cell_multiplier", ctypes.c_double),
        ("particle_split", ctypes.c_int),
        ("split_seed", ctypes.c_ulonglong),
        ("terminator", ctypes.c_int),
        ("terminator_center", ctypes.c_double * 3),
        ("terminator_half", ctypes.c_double * 3),
        ("terminator_radius", ctypes.c_double),
        ("terminator_inside", ctypes.c_int),
    ]


WCG_SHAPE_BOX, WCG_SHAPE_SPHERE, WCG_SHAPE_CAPSULE, WCG_SHAPE_CYLINDER = 0, 1, 2, 3


class WcgShape(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int),
        ("inside", ctypes.c_int),
        ("center", ctypes.c_double * 3),
        ("rot", ctypes.c_double * 4),
        ("param", ctypes.c_double * 4),
    ]


class WcgSchedule(ctypes.Structure):
    _fields_ = [
        ("sweep_cluster", ctypes.c_int),
        ("sweep_cluster_a", ctypes.c_int),
        ("pcg_batch", ctypes.c_int),
    ]


class WcgStats(ctypes.Structure):
    _fields_ = [
        ("substeps", ctypes.c_int),
        ("pcg_iters", ctypes.c_int),
        ("refinements", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("residual", ctypes.c_double),
        ("rhs_norm", ctypes.c_double),
        ("ndof", ctypes.c_longlong),
        ("nactive_buckets", ctypes.c_longlong),
        ("visc_iters", ctypes.c_int),
        ("visc_converged", ctypes.c_int),
        ("visc_residual", ctypes.c_double),
    ]


# every symbol include/wetcloth_gpu.h declares, with (restype, argtypes)
SIGNATURES = {
    "wcg_last_error": (ctypes.c_char_p, []),
    "wcg_default_params": (None, [ctypes.POINTER(WcgParams)]),
    "wcg_create": (ctypes.c_int, [ctypes.POINTER(WcgParams), ctypes.POINTER(ctypes.c_void_p)]),
    "wcg_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_upload_liquid": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, _D, _D, _D, _D, _D, _D]),
    "wcg_upload_liquid_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p]),
    "wcg_download_liquid": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D]),
    "wcg_download_liquid_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p]),
    "wcg_num_particles": (ctypes.c_longlong, [ctypes.c_void_p]),
    "wcg_upload_elasto": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong] + [_D] * 10 + [_I]),
    "wcg_download_elasto": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D]),
    "wcg_num_elasto": (ctypes.c_longlong, [ctypes.c_void_p]),
    "wcg_upload_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _D, ctypes.c_longlong]),
    "wcg_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "wcg_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_batch_step": (ctypes.c_int, [ctypes.c_void_p, _D, ctypes.c_int, _I]),
    "wcg_batch_set_threads": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "wcg_batch_threads": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, _D, _I, ctypes.c_int, _D]),
    "wcg_batch_autotune_schedules": (ctypes.c_int, [ctypes.c_void_p, _D,
                                                    ctypes.POINTER(WcgSchedule), ctypes.c_int,
                                                    ctypes.c_int, _D, _I]),
    "wcg_set_schedule": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WcgSchedule)]),
    "wcg_batch_set_shared_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "wcg_batch_shared_launches": (ctypes.c_longlong, [ctypes.c_void_p]),
    "wcg_batch_set_shared_solve_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "wcg_get_schedule": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WcgSchedule)]),
    "wcg_save_positions": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "wcg_load_positions": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "wcg_write_fluid_obj": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "wcg_rebucketize_and_resample": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_map_particle_nodes": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_step_velocity": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "wcg_project_fine": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "wcg_apply_pressure_drag_fluid": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "wcg_constrain_liquid_velocity": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_map_node_particles": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_merge_liquid_particles": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                                  ctypes.POINTER(ctypes.c_int),
                                                  ctypes.POINTER(ctypes.c_longlong)]),
    "wcg_set_correction_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_ulonglong]),
    "wcg_split_liquid_particles": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_ulonglong,
                                                  ctypes.POINTER(ctypes.c_longlong)]),
    "wcg_split_parents": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "wcg_split_liquid_particles_with": (ctypes.c_int, [ctypes.c_void_p,
                                                       ctypes.POINTER(ctypes.c_double),
                                                       ctypes.POINTER(ctypes.c_double),
                                                       ctypes.c_longlong,
                                                       ctypes.POINTER(ctypes.c_longlong)]),
    "wcg_terminate_liquid_particles": (ctypes.c_int, [ctypes.c_void_p,
                                                      ctypes.POINTER(ctypes.c_longlong)]),
    "wcg_set_terminators": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                           ctypes.POINTER(WcgShape)]),
    "wcg_split_key": (ctypes.c_ulonglong, [ctypes.c_ulonglong, ctypes.c_ulonglong]),
    "wcg_merge_draws": (ctypes.c_int, [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "wcg_download_liquid_async": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D]),
    "wcg_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_stage_liquid_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, _D, _D, _D, _D,
                                              _D, _D]),
    "wcg_upload_staged": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_correct_liquid_particles": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]),
    "wcg_correction_selector": (ctypes.c_int, [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int]),
    "wcg_advect": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "wcg_substep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "wcg_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _I]),
    "wcg_num_substeps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _I]),
    "wcg_substep_vjp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _D, _D, _D, _D, _D, _D,
                                       _D]),
    "wcg_set_viscosity": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]),
    "wcg_set_adjoint_positions": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "wcg_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WcgStats)]),
    "wcg_grid_info": (ctypes.c_int, [ctypes.c_void_p, _I, _D, _D]),
    "wcg_field_size": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_char_p]),
    "wcg_download_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _D, ctypes.c_longlong]),
    "wcg_download_ifield": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _L, ctypes.c_longlong]),
    "wcg_export_pressure_system": (ctypes.c_int, [ctypes.c_void_p, _L, _L, _L, _L, _D, _D]),
    "wcg_stream": (ctypes.c_void_p, [ctypes.c_void_p]),
    "wcg_launch_count": (ctypes.c_longlong, [ctypes.c_void_p]),
    "wcg_profile_begin": (ctypes.c_int, [ctypes.c_void_p]),
    "wcg_profile_end": (ctypes.c_int, [ctypes.c_void_p, _D, _L, ctypes.c_int]),
    "wcg_profile_num_phases": (ctypes.c_int, []),
    "wcg_profile_phase_name": (ctypes.c_char_p, [ctypes.c_int]),
    "wcg_pressure_solve_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_double,
                                                  ctypes.c_int, ctypes.c_void_p, _I, _D]),
    "wcg_correction_count": (ctypes.c_ulonglong, [ctypes.c_void_p]),
    "wcg_set_wait_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int]),
    "wcg_pcg_solve_csr": (ctypes.c_int, [_I, _I, _D, ctypes.c_int, _D, _D, ctypes.c_double,
                                         ctypes.c_int, _D, _I]),
}

_lib = None


def load():
    """Load libwcgpu.so (raises OSError if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libwcgpu.so not built ({LIB_PATH}); run __graft_entry__.build()")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class WcgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libwcgpu error {code}: {msg}")
        self.code = code


def check(code):
    if code != WCG_OK:
        raise WcgError(code, load().wcg_last_error().decode(errors="replace"))
    return code


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


def pcg_solve_csr(rowstart, col, val, rhs, tolerance_factor, max_iterations):
    """robertbridson::PCGSolver<double>::solve on a CSR matrix (wcg_pcg_solve_csr).
    Returns (x, residual, iterations, status); status is WCG_OK or
    WCG_ERR_NOT_CONVERGED (any other code raises)."""
    L = load()
    rs = np.ascontiguousarray(rowstart, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vl = np.ascontiguousarray(val, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    n = rs.shape[0] - 1
    x = np.zeros(n, dtype=np.float64)
    res = ctypes.c_double(0.0)
    it = ctypes.c_int(0)
    st = L.wcg_pcg_solve_csr(rs.ctypes.data_as(_I), cl.ctypes.data_as(_I), vl.ctypes.data_as(_D),
                             n, b.ctypes.data_as(_D), x.ctypes.data_as(_D),
                             float(tolerance_factor), int(max_iterations), ctypes.byref(res),
                             ctypes.byref(it))
    if st not in (WCG_OK, WCG_ERR_NOT_CONVERGED):
        check(st)
    return x, res.value, it.value, st
