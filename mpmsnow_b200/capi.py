"""ctypes binding of the C-ABI in ``include/mpm_gpu.h`` (``mpmsnow_b200/libmpmsnow_b200.so``).

This is the path a Python caller takes into the CUDA step.  There is no CPU fallback: if the shared library is
missing the import of the binding raises, and on a machine without a CUDA device ``mpm_create`` returns
``MPM_ERR_NO_DEVICE``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpmsnow_b200.so")

# every entry point include/mpm_gpu.h declares
EXPORTS = [
    "mpm_abi_version", "mpm_status_string", "mpm_last_error", "mpm_create", "mpm_destroy", "mpm_step", "mpm_step_ex",
    "mpm_num_particles", "mpm_variable_info", "mpm_get_variable", "mpm_set_variable", "mpm_get_variable_device",
    "mpm_set_variable_device", "mpm_get_bodies", "mpm_debug_grid_info", "mpm_debug_grid_get", "mpm_debug_apply",
    "mpm_debug_particle_cells", "mpm_get_stream", "mpm_set_collider", "mpm_set_colliders", "mpm_seed_particles",
    "mpm_profile_enable", "mpm_profile_read",
    "mpm_calculate_bodies_noalloc_max", "mpm_calculate_bodies_noalloc", "mpm_set_warm_start", "mpm_nn_pack_weights",
    "mpm_nn_conv3d", "mpm_nn_conv3d_wgrad", "mpm_nn_bias_grad", "mpm_nn_adam", "mpm_nn_features", "mpm_nn_mse",
]

WARM_START_WEIGHTS = 27 * (16 * 32 + 32 * 32 + 32 * 32 + 32 * 16)
WARM_START_FEATURES = 16
WARM_START_BIASES = 32 + 32 + 32 + 3

STATUS = {
    0: "MPM_OK", 1: "MPM_ERR_INVALID_ARGUMENT", 2: "MPM_ERR_CUDA", 3: "MPM_ERR_NO_DEVICE", 4: "MPM_ERR_NAN_MASSES",
    5: "MPM_ERR_NAN_VELOCITIES", 6: "MPM_ERR_NAN_MOMENTA", 7: "MPM_ERR_NAN_STRESS", 8: "MPM_ERR_INFINITE_HARDNESS",
    9: "MPM_ERR_NAN_PARTICLE_VELOCITY", 10: "MPM_ERR_GRID_TOO_BIG", 11: "MPM_ERR_UNKNOWN_VARIABLE",
    12: "MPM_ERR_WRONG_SIZE", 13: "MPM_ERR_UNSUPPORTED", 14: "MPM_ERR_CANCELLED", 15: "MPM_ERR_INTERNAL",
    16: "MPM_ERR_OUT_OF_MEMORY", 17: "MPM_ERR_TOO_MANY_PARTICLES",
}


class MpmCollider(C.Structure):
    _fields_ = [("kind", C.c_int), ("coeffs", C.c_float * 4), ("velocity", C.c_float * 3), ("friction", C.c_float),
                ("sticky", C.c_int), ("grid_dims", C.c_int * 3), ("grid_phi", C.POINTER(C.c_float)),
                ("grid_velocity", C.POINTER(C.c_float))]


class MpmSceneDesc(C.Structure):
    _fields_ = [("grid_size", C.c_float), ("dimension", C.c_int), ("shape_function", C.c_int),
                ("youngs_modulus", C.c_float), ("poisson_ratio", C.c_float), ("hardening", C.c_float),
                ("compressive_strength", C.c_float), ("tensile_strength", C.c_float), ("num_colliders", C.c_int),
                ("colliders", C.POINTER(MpmCollider)), ("num_gravity_fields", C.c_int),
                ("gravity", C.POINTER(C.c_float)), ("device", C.c_int)]


class MpmSolveParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("tolerance", C.c_float)]


class MpmStepStats(C.Structure):
    _fields_ = [("num_bodies", C.c_int), ("num_ballistic", C.c_int), ("max_iterations_used", C.c_int),
                ("total_iterations", C.c_int), ("iterations", C.c_int * 64), ("b_norm2", C.c_double * 64),
                ("r_norm2", C.c_double * 64), ("exit_reason", C.c_int * 64), ("fp64_svd_particles", C.c_int),
                ("kernel_launches", C.c_int)]


class MpmPhaseProfile(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int), ("total_ms", C.c_double), ("particles", C.c_double),
                ("nodes", C.c_double)]


class MpmWarmStart(C.Structure):
    _fields_ = [("weights", C.POINTER(C.c_float)), ("biases", C.POINTER(C.c_float)), ("feature_scale", C.c_float * 16),
                ("output_scale", C.c_float), ("light_mass", C.c_float), ("density", C.c_float), ("min_nodes", C.c_int),
                ("use_history", C.c_int)]


CANCEL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)
ITERATE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_size_t)

_lib = None


def load():
    """Load the library (built in-tree by ``mpmsnow_b200/build.py``).  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python mpmsnow_b200/build.py` "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    vp = C.c_void_p
    L.mpm_abi_version.restype = C.c_int
    L.mpm_status_string.restype = C.c_char_p
    L.mpm_status_string.argtypes = [C.c_int]
    L.mpm_last_error.restype = C.c_char_p
    L.mpm_last_error.argtypes = [vp]
    L.mpm_create.argtypes = [C.POINTER(MpmSceneDesc), C.c_size_t, fp, fp, C.POINTER(vp)]
    L.mpm_destroy.argtypes = [vp]
    L.mpm_step.argtypes = [vp, C.c_float, C.POINTER(MpmSolveParams), C.POINTER(MpmStepStats)]
    L.mpm_step_ex.argtypes = [vp, C.c_float, C.POINTER(MpmSolveParams), C.c_int, CANCEL_FN, vp, ITERATE_FN, vp,
                              C.POINTER(MpmStepStats)]
    L.mpm_num_particles.restype = C.c_size_t
    L.mpm_num_particles.argtypes = [vp]
    L.mpm_variable_info.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int)]
    L.mpm_get_variable.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
    L.mpm_set_variable.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
    L.mpm_get_variable_device.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
    L.mpm_set_variable_device.argtypes = [vp, C.c_char_p, vp, C.c_size_t]
    L.mpm_get_bodies.argtypes = [vp, vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.mpm_debug_grid_info.argtypes = [vp, C.c_int, fp, ip, fp, C.POINTER(C.c_int)]
    L.mpm_debug_grid_get.argtypes = [vp, C.c_int, C.c_char_p, fp, C.c_size_t]
    L.mpm_debug_apply.argtypes = [vp, C.c_int, C.c_char_p, fp, fp, C.c_size_t, C.c_float]
    L.mpm_debug_particle_cells.argtypes = [vp, ip, ip, ip]
    L.mpm_get_stream.restype = vp
    L.mpm_get_stream.argtypes = [vp]
    L.mpm_profile_enable.restype = C.c_int
    L.mpm_profile_enable.argtypes = [vp, C.c_int]
    L.mpm_profile_read.restype = C.c_int
    L.mpm_profile_read.argtypes = [vp, C.POINTER(MpmPhaseProfile), C.c_int]
    L.mpm_calculate_bodies_noalloc_max.restype = C.c_int
    L.mpm_calculate_bodies_noalloc.restype = C.c_int
    L.mpm_calculate_bodies_noalloc.argtypes = [vp, C.c_size_t, C.c_float, vp, vp, vp]
    i32, f32, ll = C.c_int, C.c_float, C.c_longlong
    L.mpm_set_warm_start.argtypes = [vp, C.POINTER(MpmWarmStart)]
    L.mpm_set_collider.argtypes = [vp, C.c_int, C.POINTER(MpmCollider)]
    L.mpm_set_colliders.argtypes = [vp, C.c_int, C.POINTER(MpmCollider)]
    L.mpm_seed_particles.argtypes = [C.POINTER(MpmCollider), fp, fp, C.c_float, C.c_float, C.c_int, vp, vp, vp,
                                     C.c_size_t, C.POINTER(C.c_size_t)]
    L.mpm_nn_pack_weights.argtypes = [vp, i32, i32, i32, i32, vp, vp, vp]
    L.mpm_nn_conv3d.argtypes = [vp, i32, vp, vp, i32, i32, i32, i32, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp]
    L.mpm_nn_conv3d_wgrad.argtypes = [vp, i32, vp, i32, vp, i32, i32, i32, i32, vp, vp]
    L.mpm_nn_bias_grad.argtypes = [vp, i32, i32, ll, vp, vp]
    L.mpm_nn_adam.argtypes = [vp, vp, vp, vp, i32, f32, f32, f32, f32, i32, f32, vp]
    L.mpm_nn_features.argtypes = [vp, vp, vp, vp, vp, vp, ll, f32, f32, f32, f32, vp, vp, vp, vp]
    L.mpm_nn_mse.argtypes = [vp, i32, vp, vp, ll, f32, vp, vp, vp]
    for name in ("mpm_set_warm_start", "mpm_nn_pack_weights", "mpm_nn_conv3d", "mpm_nn_conv3d_wgrad", "mpm_nn_bias_grad",
                 "mpm_nn_adam", "mpm_nn_features", "mpm_nn_mse"):
        getattr(L, name).restype = C.c_int
    for name in ("mpm_create", "mpm_step", "mpm_step_ex", "mpm_variable_info", "mpm_get_variable", "mpm_set_variable",
                 "mpm_get_variable_device", "mpm_set_variable_device", "mpm_get_bodies", "mpm_debug_grid_info",
                 "mpm_debug_grid_get", "mpm_debug_apply", "mpm_debug_particle_cells"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


class MpmError(RuntimeError):
    """A non-OK mpm_status; ``message`` is the reference's std::runtime_error text where it has one."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message
