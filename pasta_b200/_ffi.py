"""ctypes binding of libpasta_b200.so (the C ABI in include/pasta_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpasta_b200.so")

WL_LINSPACE, WL_LOGSPACE, WL_NONUNIFORM = 0, 1, 2
DISP_NONE, DISP_FIXED, DISP_VARIABLE = 0, 1, 2
CONT_CHUNK, CONT_LINEAR, CONT_FIXED, CONT_CONSTANT = 0, 1, 2, 3
FIT_BATCHED, FIT_PLAIN = 0, 1


class PsoSettingsC(C.Structure):
    _fields_ = [("num_particles", C.c_int32), ("max_iters", C.c_int32), ("inertia_factor", C.c_double),
                ("cognitive_factor", C.c_double), ("social_factor", C.c_double), ("delta", C.c_double),
                ("vsini_lo", C.c_double), ("vsini_hi", C.c_double), ("rv_lo", C.c_double),
                ("rv_hi", C.c_double), ("ckind", C.c_int32 * 5), ("ca", C.c_double * 5), ("cb", C.c_double * 5)]


class FitResultC(C.Structure):
    _fields_ = [("label", C.c_double * 5), ("chi2", C.c_double), ("time", C.c_double),
                ("iterations", C.c_int32), ("status", C.c_int32), ("n_params", C.c_int32),
                ("_pad", C.c_int32)]


class BinarySettingsC(C.Structure):
    _fields_ = [("num_particles", C.c_int32), ("max_iters", C.c_int32), ("inertia_factor", C.c_double),
                ("cognitive_factor", C.c_double), ("social_factor", C.c_double), ("delta", C.c_double),
                ("vsini_lo", C.c_double), ("vsini_hi", C.c_double), ("rv_lo", C.c_double),
                ("rv_hi", C.c_double), ("ckind", C.c_int32 * 11), ("ca", C.c_double * 11),
                ("cb", C.c_double * 11)]


class BinaryResultC(C.Structure):
    _fields_ = [("label1", C.c_double * 5), ("label2", C.c_double * 5), ("light_ratio", C.c_double),
                ("chi2", C.c_double), ("time", C.c_double), ("iterations", C.c_int32), ("status", C.c_int32),
                ("n_params", C.c_int32), ("_pad", C.c_int32)]


# name -> (restype, argtypes); every symbol of include/pasta_b200.h
P, D, I64, I, F = C.c_void_p, C.c_double, C.c_int64, C.c_int, C.c_float
SIGNATURES = {
    "pasta_abi_version": (I, []),
    "pasta_last_error": (C.c_char_p, []),
    "pasta_set_device": (I, [I]),
    "pasta_kernel_launch_count": (I64, []),
    "pasta_set_linear_tensor_cores": (I, [I]),
    "pasta_set_interp_tensor_cores": (I, [I]),
    "pasta_grid_create": (I, [P, P, P, I64, I64, I, D, D, P, P]),
    "pasta_grid_destroy": (I, [P]),
    "pasta_grid_direct_max": (I, [P, P]),
    "pasta_grid_set_direct_max": (I, [P, C.c_int32]),
    "pasta_grid_tc_min": (I, [P, P]),
    "pasta_grid_set_tc_min": (I, [P, I]),
    "pasta_grid_shape": (I, [P, P]),
    "pasta_grid_axis": (I, [P, I, P]),
    "pasta_grid_logg_limits": (I, [P, P, P]),
    "pasta_grid_cumulative_size": (I, [P, P]),
    "pasta_grid_clamp_1d": (I, [P, D, D, D, I, P]),
    "pasta_grid_is_teff_logg_between_bounds": (I, [P, D, D, P]),
    "pasta_grid_coefficients": (I, [P, D, D, D, P, P, P, P, P]),
    "pasta_interpolate": (I, [P, P, I64, P, P]),
    "pasta_dispersion_create": (I, [I, D, D, I64, P, I, P, I64, D, P, P]),
    "pasta_dispersion_destroy": (I, [P]),
    "pasta_dispersion_convolve": (I, [P, P, I64, P]),
    "pasta_dispersion_kernels": (I, [P, P, P]),
    "pasta_dispersion_convolve_resample": (I, [P, I, D, D, I64, P, I64, P]),
    "pasta_continuum_create": (I, [I, P, I64, I, I, D, P, I, P, I, P]),
    "pasta_continuum_destroy": (I, [P]),
    "pasta_continuum_nparams": (I, [P]),
    "pasta_continuum_fit": (I, [P, P, P, P, I64, P, P]),
    "pasta_continuum_build": (I, [P, P, I64, P]),
    "pasta_produce_model": (I, [P, P, P, I64, P, P]),
    "pasta_interpolate_and_convolve": (I, [P, P, P, I64, P, P]),
    "pasta_chi2": (I, [P, P, P, P, P, I64, P, I64, P, P]),
    "pasta_chi2_noalloc": (I, [P, P, P, P, P, I64, P, I64, P, P, P]),
    "pasta_chi2_many": (I, [P, I64, P, P, P, P, P, P, P, P]),
    "pasta_ccf": (I, [P, P, P, I64, D, D, D, P, I64, P, P]),
    "pasta_fit": (I, [P, P, P, P, P, P, I64, I64, P, I, P, P, P]),
    "pasta_fit_many": (I, [P, I64, P, P, P, P, P, P, P, I, P, P]),
    "pasta_compute_uncertainty": (I, [P, P, P, I64, P, P, I64, D, P, P, P, P, P]),
    "pasta_batch_create": (I, [P, I64, P, P, P, P, P, P, P, P]),
    "pasta_batch_step": (I, [P, I, P]),
    "pasta_batch_profile_step": (I, [P, P]),
    "pasta_batch_info": (I, [P, P]),
    "pasta_batch_finish": (I, [P, P, P]),
    "pasta_batch_destroy": (I, [P]),
    "pasta_server_create": (I, [P, I, I64, P]),
    "pasta_server_submit": (I, [P, P, P, P, P, P, I64, C.c_uint64, P]),
    "pasta_server_step": (I, [P]),
    "pasta_server_poll": (I, [P, P, P, P, I64, I, P]),
    "pasta_server_pending": (I, [P, P, P, P]),
    "pasta_server_memory": (I, [P, P, P]),
    "pasta_server_destroy": (I, [P]),
    "pasta_server_run": (I, [P, I, P]),
    "pasta_server_stats": (I, [P, P]),
    "pasta_interpolate_linear": (I, [P, P, I64, P, P]),
    "pasta_binary_model": (I, [P, P, P, P, I64, P, P]),
    "pasta_binary_chi2": (I, [P, P, P, P, P, P, I64, P, I64, P, P]),
    "pasta_binary_fit": (I, [P, P, P, P, P, P, P, I64, C.c_uint64, P, P, P]),
}

_lib = None


class PastaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def lib():
    """Load the CUDA library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"pasta_b200 CUDA library not found at {LIB_PATH}; build it with "
                "`python -m pasta_b200.build` (there is no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def check(rc):
    if rc < 0:
        raise PastaError(rc, lib().pasta_last_error().decode(errors="replace"))
    return rc


def ptr(a):
    return None if a is None else a.ctypes.data


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def loaded_path():
    return LIB_PATH if _lib is not None else None
