"""ctypes declarations of libsdfgpu.so (the C ABI in include/sdfgpu.h)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsdfgpu.so")

c_int_p = ctypes.POINTER(ctypes.c_int32)
c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_i64_p = ctypes.POINTER(ctypes.c_int64)
vp = ctypes.c_void_p

SDFGPU_OK = 0
SDFGPU_ERR_INVALID_ARGUMENT = 1
SDFGPU_ERR_NUMERICAL = 2
SDFGPU_ERR_OUT_OF_MEMORY = 3
SDFGPU_ERR_TIMEOUT = 4
SDFGPU_ERR_CUDA = 5
SDFGPU_ERR_NOT_READY = 6


class ProblemDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("min_x", ctypes.c_double), ("min_y", ctypes.c_double),
        ("max_x", ctypes.c_double), ("max_y", ctypes.c_double),
        ("map_values", c_dbl_p),
        ("num_frames", ctypes.c_int32), ("poses", c_dbl_p),
        ("num_points", ctypes.c_int32), ("point_frame", c_int_p), ("point_xy", c_dbl_p),
        ("point_expected", c_dbl_p), ("point_sqrt_weight", c_dbl_p),
        ("num_eikonal", ctypes.c_int32), ("eikonal_wh", c_int_p), ("eikonal_normal", c_dbl_p),
        ("eikonal_sqrt_weight", c_dbl_p),
        ("num_odom", ctypes.c_int32), ("odom_ij", c_int_p), ("odom_meas", c_dbl_p),
        ("odom_sqrt_weight", c_dbl_p),
        ("node_to_active", c_int_p),
        ("huber_delta", ctypes.c_double), ("smooth_gradient", ctypes.c_int32),
        ("smooth_gradient_step", ctypes.c_double),
    ]


class ProblemOptionsC(ctypes.Structure):
    _fields_ = [
        ("weight_scan", ctypes.c_double), ("weight_hallucination", ctypes.c_double),
        ("weight_eikonal", ctypes.c_double), ("weight_odometry", ctypes.c_double),
        ("weight_relation", ctypes.c_double),
        ("hallucination_points_per_scan_point", ctypes.c_int32),
        ("hallucination_step_size", ctypes.c_double),
        ("hallucination_both_directions", ctypes.c_int32),
        ("normals_method", ctypes.c_int32), ("normals_k_neighbors", ctypes.c_int32),
        ("normals_per_scan", ctypes.c_int32), ("normals_corner_threshold", ctypes.c_double),
        ("huber_delta", ctypes.c_double), ("smooth_gradient", ctypes.c_int32),
        ("smooth_gradient_step", ctypes.c_double), ("active_region", ctypes.c_int32),
        ("active_margin", ctypes.c_int32),
    ]


class SolverOptionsC(ctypes.Structure):
    _fields_ = [
        ("max_iterations", ctypes.c_int32), ("step_tolerance", ctypes.c_double),
        ("lambda_init", ctypes.c_double), ("lambda_factor", ctypes.c_double),
        ("reject_worse_steps", ctypes.c_int32), ("marquardt_scaling", ctypes.c_int32),
        ("trust_region", ctypes.c_int32), ("num_threads", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("refine_steps", ctypes.c_int32),
        ("refine_tolerance", ctypes.c_double),
    ]


class SolveResultC(ctypes.Structure):
    _fields_ = [
        ("converged", ctypes.c_int32), ("iterations", ctypes.c_int32),
        ("initial_cost", ctypes.c_double), ("final_cost", ctypes.c_double),
        ("duration_seconds", ctypes.c_double), ("cost_history_length", ctypes.c_int32),
        ("status", ctypes.c_int32),
    ]


SnapshotFn = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int32, c_dbl_p, c_dbl_p)


class IncrementalDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("min_x", ctypes.c_double), ("min_y", ctypes.c_double),
        ("max_x", ctypes.c_double), ("max_y", ctypes.c_double),
        ("map_values", c_dbl_p),
        ("num_frames", ctypes.c_int32), ("poses", c_dbl_p),
        ("scan_offsets", c_int_p), ("scan_xy", c_dbl_p),
        ("num_relations", ctypes.c_int32), ("relation_ij", c_int_p), ("relation_meas", c_dbl_p),
        ("relation_sqrt_weight", c_dbl_p),
        ("increment_size", ctypes.c_int32), ("iterations_per_increment", ctypes.c_int32),
        ("snapshot_every", ctypes.c_int32), ("snapshot", SnapshotFn), ("snapshot_user", ctypes.c_void_p),
        ("build_on_device", ctypes.c_int32), ("warm_analysis", ctypes.c_int32),
    ]


# name -> (restype, argtypes); every exported symbol of include/sdfgpu.h
SIGNATURES = {
    "sdfgpu_last_error_message": (ctypes.c_char_p, []),
    "sdfgpu_version": (ctypes.c_char_p, []),
    "sdfgpu_device_count": (ctypes.c_int32, []),
    "sdfgpu_problem_options_default": (None, [ctypes.POINTER(ProblemOptionsC)]),
    "sdfgpu_problem_build": (ctypes.c_int, [
        ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, c_dbl_p, ctypes.c_int32, c_dbl_p, c_int_p, c_dbl_p, c_dbl_p,
        ctypes.c_int32, ctypes.c_int32, c_int_p, c_dbl_p, c_dbl_p,
        ctypes.POINTER(ProblemOptionsC), ctypes.POINTER(vp)]),
    "sdfgpu_problem_build_device": (ctypes.c_int, [
        ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, c_dbl_p, ctypes.c_int32, c_dbl_p, c_int_p, c_dbl_p, c_dbl_p,
        ctypes.c_int32, ctypes.c_int32, c_int_p, c_dbl_p, c_dbl_p,
        ctypes.POINTER(ProblemOptionsC), ctypes.POINTER(vp)]),
    "sdfgpu_problem_create": (ctypes.c_int, [ctypes.POINTER(ProblemDesc), ctypes.POINTER(vp)]),
    "sdfgpu_problem_create_batch": (ctypes.c_int, [ctypes.POINTER(ProblemDesc), ctypes.c_int32,
                                                   ctypes.POINTER(vp)]),
    "sdfgpu_problem_destroy": (ctypes.c_int, [vp]),
    "sdfgpu_release_cached_memory": (ctypes.c_int, []),
    "sdfgpu_measure_fp64_peak": (ctypes.c_int, [c_dbl_p]),
    "sdfgpu_debug_solve_fault": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_uint32]),
    "sdfgpu_debug_supernode_count": (ctypes.c_int32, [vp]),
    "sdfgpu_kernel_timing": (ctypes.c_int, [vp, ctypes.c_uint32]),
    "sdfgpu_kernel_times": (ctypes.c_int, [vp, c_dbl_p, c_i64_p, c_dbl_p, ctypes.c_int32]),
    "sdfgpu_kernel_class_name": (ctypes.c_char_p, [ctypes.c_int32]),
    "sdfgpu_kernel_class_is_memory_bound": (ctypes.c_int32, [ctypes.c_int32]),
    "sdfgpu_problem_count": (ctypes.c_int32, [vp]),
    "sdfgpu_problem_sizes": (ctypes.c_int, [vp, ctypes.c_int32, c_int_p]),
    "sdfgpu_problem_get_specs": (ctypes.c_int, [vp, ctypes.c_int32, c_int_p, c_dbl_p, c_dbl_p,
                                                c_dbl_p, c_int_p, c_dbl_p, c_dbl_p, c_int_p,
                                                c_dbl_p, c_dbl_p, c_int_p]),
    "sdfgpu_get_state": (ctypes.c_int, [vp, ctypes.c_int32, c_dbl_p, c_dbl_p]),
    "sdfgpu_set_state": (ctypes.c_int, [vp, ctypes.c_int32, c_dbl_p, c_dbl_p]),
    "sdfgpu_cost": (ctypes.c_int, [vp, ctypes.c_int32, c_dbl_p]),
    "sdfgpu_apply_step": (ctypes.c_int, [vp, ctypes.c_int32, c_dbl_p]),
    "sdfgpu_solver_options_default": (None, [ctypes.POINTER(SolverOptionsC)]),
    "sdfgpu_solve": (ctypes.c_int, [vp, ctypes.POINTER(SolverOptionsC),
                                    ctypes.POINTER(SolveResultC), c_dbl_p, ctypes.c_int32]),
    "sdfgpu_linearize": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                        ctypes.c_int32]),
    "sdfgpu_linearization_sizes": (ctypes.c_int, [vp, c_i64_p]),
    "sdfgpu_linearization_get": (ctypes.c_int, [vp, c_dbl_p, c_int_p, c_int_p, c_int_p, c_dbl_p,
                                                c_int_p, c_int_p, c_dbl_p, c_dbl_p, c_dbl_p]),
    "sdfgpu_last_profile": (ctypes.c_int, [vp, c_dbl_p]),
    "sdfgpu_set_schedule": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int32)]),
    "sdfgpu_set_tensor_core_choice": (ctypes.c_int, [vp, ctypes.c_int32]),
    "sdfgpu_tensor_core_choice": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
                                                 ctypes.POINTER(ctypes.c_double)]),
    "sdfgpu_autotune": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int32), c_dbl_p, c_dbl_p, ctypes.c_int32,
                                       ctypes.POINTER(ctypes.c_int32)]),
    "sdfgpu_run_incremental": (ctypes.c_int, [ctypes.POINTER(IncrementalDesc), ctypes.POINTER(ProblemOptionsC),
                                              ctypes.POINTER(SolverOptionsC), c_dbl_p, c_dbl_p,
                                              ctypes.POINTER(SolveResultC), c_dbl_p, ctypes.c_int32, c_dbl_p]),
    "sdfgpu_write_poses": (ctypes.c_int, [ctypes.c_char_p, c_dbl_p, ctypes.c_int32]),
    "sdfgpu_write_map": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, c_dbl_p]),
    "sdfgpu_write_scan_points": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, c_dbl_p, c_int_p, c_dbl_p]),
    "sdfgpu_write_metrics": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(SolveResultC), c_dbl_p]),
    "sdfgpu_evaluate_trajectory": (ctypes.c_int, [c_dbl_p, c_dbl_p, ctypes.c_int32, c_dbl_p]),
    "sdfgpu_points_outside_map": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_int32, c_dbl_p, c_int_p, c_dbl_p, c_i64_p, c_i64_p]),
    "sdfgpu_ldlt_create": (ctypes.c_int, [ctypes.c_int32, c_int_p, c_int_p, c_int_p,
                                          ctypes.POINTER(vp)]),
    "sdfgpu_ldlt_factorize": (ctypes.c_int, [vp, c_dbl_p]),
    "sdfgpu_ldlt_solve": (ctypes.c_int, [vp, c_dbl_p, c_dbl_p]),
    "sdfgpu_ldlt_destroy": (ctypes.c_int, [vp]),
    "sdfgpu_server_create": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(vp)]),
    "sdfgpu_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(ProblemDesc),
                                            ctypes.POINTER(SolverOptionsC), c_i64_p]),
    "sdfgpu_server_poll": (ctypes.c_int, [vp, ctypes.c_int64, ctypes.POINTER(SolveResultC),
                                          c_dbl_p, c_dbl_p]),
    "sdfgpu_server_cancel": (ctypes.c_int, [vp, ctypes.c_int64]),
    "sdfgpu_server_stats": (ctypes.c_int, [vp, c_dbl_p]),
    "sdfgpu_server_drain": (ctypes.c_int, [vp, ctypes.c_int64]),
    "sdfgpu_server_destroy": (ctypes.c_int, [vp]),
    "sdfgpu_dense_ldlt_solve_noalloc": (ctypes.c_int, [ctypes.c_int32, c_dbl_p, c_dbl_p, c_dbl_p]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Loads libsdfgpu.so; raises if it has not been built. There is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} is missing: build it with sdf-slam_b200/build.py")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
