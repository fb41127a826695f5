"""ctypes binding of ``libcorrct_b200.so`` (declared in ``include/corrct_b200.h``).

The library is loaded lazily on first use.  There is no CPU fallback: a missing
library or a missing CUDA device raises immediately.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcorrct_b200.so")

ABI_VERSION = 7  # CCT_ABI_VERSION of include/corrct_b200.h

CCT_OK = 0
CCT_ERR_VALUE = 1
CCT_ERR_CUDA = 2
CCT_ERR_UNSUPPORTED = 3

CCT_DTYPE_F32 = 0
CCT_DTYPE_BF16 = 1
CCT_DTYPE_FIELDS_F32 = 2

CCT_BP_REFERENCE = 0
CCT_BP_SYMMETRIC = 1
CCT_BP_ADJOINT = 2

CCT_VARIANT_FP_TMA = 1
CCT_VARIANT_FP_SLICES2 = 2

CCT_METHOD_MLEM = 0
CCT_METHOD_SIRT = 1

c_float_p = ctypes.c_void_p  # device pointers are passed as integers


class XrfDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("n_angles", ctypes.c_int32),
        ("n_det", ctypes.c_int32),
        ("n_slices", ctypes.c_int32),
        ("maps_dtype", ctypes.c_int32),
        ("variant", ctypes.c_int32),
        ("fp_matrix", ctypes.c_void_p),
        ("bp_trig", ctypes.c_void_p),
        ("weights", ctypes.c_void_p),
        ("line_scale", ctypes.c_void_p),
        ("psf", ctypes.c_void_p),
        ("psf_len", ctypes.c_int32),
        ("n_channels", ctypes.c_int32),
        ("maps_slice_stride", ctypes.c_int64),
        ("channel_scale", ctypes.c_void_p),
        ("fp_box_strides", ctypes.c_void_p),
    ]


class MapsDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("n_angles", ctypes.c_int32),
        ("n_det", ctypes.c_int32),
        ("n_slices", ctypes.c_int32),
        ("n_sub", ctypes.c_int32),
        ("maps_dtype", ctypes.c_int32),
        ("has_in", ctypes.c_int32),
        ("has_out", ctypes.c_int32),
        ("rot_in", ctypes.c_void_p),
        ("rot_out", ctypes.c_void_p),
        ("pairs", ctypes.c_void_p),
        ("n_entries", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("quads", ctypes.c_void_p),
        ("n_quads", ctypes.c_int32),
        ("emitted_scale", ctypes.c_float),
    ]


class NoiseDesc(ctypes.Structure):
    _fields_ = [
        ("num_photons", ctypes.c_double),
        ("detection_efficiency", ctypes.c_double),
        ("background_avg", ctypes.c_double),
        ("background_std", ctypes.c_double),
        ("readout_std", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("add_poisson", ctypes.c_int32),
        ("has_background", ctypes.c_int32),
        ("has_readout", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ConvDesc(ctypes.Structure):
    _fields_ = [
        ("batch", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("cin", ctypes.c_int32),
        ("cout", ctypes.c_int32),
    ]


class SolverState(ctypes.Structure):
    _fields_ = [
        ("x", ctypes.c_void_p),
        ("x_relax", ctypes.c_void_p),
        ("b", ctypes.c_void_p),
        ("tau", ctypes.c_void_p),
        ("sigma", ctypes.c_void_p),
        ("sino_buf", ctypes.c_void_p),
        ("vol_buf", ctypes.c_void_p),
        ("tv_dual", ctypes.c_void_p),
        ("partials", ctypes.c_void_p),
        ("residuals", ctypes.c_void_p),
        ("active", ctypes.c_void_p),
        ("iterations", ctypes.c_void_p),
        ("tolerance", ctypes.c_void_p),
        ("x_mask", ctypes.c_void_p),
        ("lower_limit", ctypes.c_float),
        ("upper_limit", ctypes.c_float),
        ("has_lower", ctypes.c_int32),
        ("has_upper", ctypes.c_int32),
        ("background", ctypes.c_float),
        ("has_background", ctypes.c_int32),
        ("tv_lambda", ctypes.c_float),
        ("tau_shared", ctypes.c_int32),
        ("sino_tmp", ctypes.c_void_p),
        ("residual_history", ctypes.c_void_p),
        ("history_len", ctypes.c_int32),
        ("x_mask_per_slice", ctypes.c_int32),
        ("joint_stop", ctypes.c_int32),
        ("b_mask", ctypes.c_void_p),
        ("b_test_mask", ctypes.c_void_p),
        ("partials_test", ctypes.c_void_p),
        ("residuals_test", ctypes.c_void_p),
        ("history_test", ctypes.c_void_p),
    ]


# name -> (restype, argtypes); every symbol declared in include/corrct_b200.h
SIGNATURES = {
    "cct_abi_version": (ctypes.c_int, []),
    "cct_last_error": (ctypes.c_char_p, []),
    "cct_device_error": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "cct_fp": (ctypes.c_int, [ctypes.POINTER(XrfDesc), c_float_p, c_float_p, c_float_p, ctypes.c_void_p]),
    "cct_bp": (
        ctypes.c_int,
        [ctypes.POINTER(XrfDesc), ctypes.c_int32, c_float_p, c_float_p, c_float_p, ctypes.c_void_p],
    ),
    "cct_maps_workspace_size": (
        ctypes.c_int,
        [ctypes.POINTER(MapsDesc), ctypes.c_int32, ctypes.POINTER(ctypes.c_size_t)],
    ),
    "cct_compute_maps": (
        ctypes.c_int,
        [ctypes.POINTER(MapsDesc), c_float_p, c_float_p, c_float_p, c_float_p, ctypes.c_size_t, ctypes.c_void_p],
    ),
    "cct_compute_maps_noalloc": (
        ctypes.c_int,
        [ctypes.POINTER(MapsDesc), c_float_p, c_float_p, c_float_p, ctypes.c_void_p],
    ),
    "cct_solver_partials_count": (ctypes.c_int, [ctypes.POINTER(XrfDesc), ctypes.POINTER(ctypes.c_int64)]),
    "cct_mlem_step": (
        ctypes.c_int,
        [ctypes.POINTER(XrfDesc), c_float_p, ctypes.POINTER(SolverState), ctypes.c_void_p],
    ),
    "cct_mlem_fp": (
        ctypes.c_int,
        [ctypes.POINTER(XrfDesc), c_float_p, ctypes.POINTER(SolverState), ctypes.c_void_p],
    ),
    "cct_mlem_update": (ctypes.c_int, [ctypes.POINTER(XrfDesc), ctypes.POINTER(SolverState), ctypes.c_void_p]),
    "cct_sirt_step": (
        ctypes.c_int,
        [ctypes.POINTER(XrfDesc), c_float_p, ctypes.c_int32, ctypes.POINTER(SolverState), ctypes.c_void_p],
    ),
    "cct_pdhg_step": (
        ctypes.c_int,
        [ctypes.POINTER(XrfDesc), c_float_p, ctypes.c_int32, ctypes.POINTER(SolverState), ctypes.c_void_p],
    ),
    "cct_reduce_norm": (
        ctypes.c_int,
        [c_float_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, c_float_p, c_float_p, ctypes.c_void_p],
    ),
    "cct_conv3x3_fwd": (
        ctypes.c_int,
        [ctypes.POINTER(ConvDesc), c_float_p, c_float_p, c_float_p, ctypes.c_int32, c_float_p, ctypes.c_void_p],
    ),
    "cct_conv3x3_wgrad": (ctypes.c_int, [ctypes.POINTER(ConvDesc), c_float_p, c_float_p, c_float_p, ctypes.c_void_p]),
    "cct_net_flip_weights": (ctypes.c_int, [c_float_p, c_float_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    "cct_net_relu_bwd": (ctypes.c_int, [c_float_p, c_float_p, c_float_p, ctypes.c_int64, ctypes.c_void_p]),
    "cct_net_avgpool2": (
        ctypes.c_int,
        [c_float_p, c_float_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p],
    ),
    "cct_net_upsample2": (
        ctypes.c_int,
        [c_float_p, c_float_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p],
    ),
    "cct_net_add": (ctypes.c_int, [c_float_p, c_float_p, c_float_p, ctypes.c_int64, ctypes.c_void_p]),
    "cct_net_bias_grad": (ctypes.c_int, [c_float_p, c_float_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p]),
    "cct_net_mse": (
        ctypes.c_int,
        [c_float_p, c_float_p, c_float_p, c_float_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p],
    ),
    "cct_net_adam": (
        ctypes.c_int,
        [c_float_p, c_float_p, c_float_p, c_float_p, c_float_p, ctypes.c_int64, ctypes.c_float, ctypes.c_float,
         ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_void_p],
    ),
    "cct_net_pack_nhwc": (
        ctypes.c_int,
        [c_float_p, ctypes.c_int32, c_float_p, ctypes.c_int64, ctypes.c_int32, c_float_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "cct_net_unpack_c0": (
        ctypes.c_int,
        [c_float_p, ctypes.c_int32, c_float_p, c_float_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_float, c_float_p,
         ctypes.c_int64, ctypes.c_void_p],
    ),
    "cct_net_ratio": (ctypes.c_int, [c_float_p, c_float_p, c_float_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p]),
    "cct_net_timeout": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "cct_ragged_workspace_size": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_size_t)]),
    "cct_ragged_plan_create": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(XrfDesc), ctypes.POINTER(ctypes.c_void_p),
         ctypes.POINTER(SolverState), ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p],
    ),
    "cct_ragged_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cct_ragged_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cct_noise_partials_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int64)]),
    "cct_add_noise": (
        ctypes.c_int,
        [ctypes.POINTER(NoiseDesc), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
}

_lib = None
_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Load the shared library (once) and bind the C signatures."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m pycorrectedemissionct_b200.build` "
                    "(there is no CPU fallback)"
                )
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            if lib.cct_abi_version() != ABI_VERSION:
                raise RuntimeError("libcorrct_b200.so ABI version mismatch")
            _lib = lib
    return _lib


def check(status: int) -> None:
    """Map a status code to the reference's exception types."""
    if status == CCT_OK:
        return
    msg = load().cct_last_error().decode(errors="replace")
    if status == CCT_ERR_VALUE:
        raise ValueError(msg)
    if status == CCT_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(f"CUDA error: {msg}")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
