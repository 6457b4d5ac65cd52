"""ctypes binding of liblucem_b200.so (the C ABI in include/lucem_b200.h).

The library is built in-tree by ``python -m lucem_b200.build``.  There is no
fallback: if the library is missing, importing the ops raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblucem_b200.so")

MAX_DIMS = 8

# lucem_status
STATUS_NAMES = {
    0: "OK", 1: "SHAPE_MISMATCH", 2: "ALIASED_BUFFERS", 3: "INVALID_DIMENSION", 4: "UNKNOWN_PAD_MODE",
    5: "INVALID_ORIGIN", 6: "INVALID_WEIGHTS", 7: "INVALID_PARAMETER", 8: "EMPTY_INPUT",
    9: "AXIS_OUT_OF_BOUNDS", 10: "REPEATED_AXIS", 11: "TOO_MANY_ELEMENTS", 12: "OUT_OF_DEVICE_MEMORY",
    13: "UNSUPPORTED_DTYPE", 14: "CUDA", 15: "DEVICE_TIMEOUT", 16: "INVALID_HANDLE",
}
U8, U16, F32, U32 = 1, 2, 3, 4
PAD_REFLECT, PAD_CONSTANT, PAD_NEAREST, PAD_MIRROR, PAD_WRAP = 0, 1, 2, 3, 4
RESP_GAUSSIAN, RESP_DOG, RESP_LAPLACE, RESP_GRAD_MAG, RESP_UNSHARP = 0, 1, 2, 3, 4


class Tensor(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int32), ("ndim", C.c_int32),
                ("dims", C.c_int64 * MAX_DIMS)]


class GaussianSettings(C.Structure):
    _fields_ = [("orders", C.POINTER(C.c_uint32)), ("n_orders", C.c_int32), ("mode", C.c_int32),
                ("cval", C.c_double), ("truncate", C.c_double), ("radii", C.POINTER(C.c_int64)),
                ("n_radii", C.c_int32), ("axes", C.POINTER(C.c_int64)), ("n_axes", C.c_int32),
                ("has_channel_axis", C.c_int32), ("channel_axis", C.c_int64), ("input_scale", C.c_double)]


class Gaussian1dSettings(C.Structure):
    _fields_ = [("axis", C.c_int64), ("order", C.c_uint32), ("mode", C.c_int32), ("cval", C.c_double),
                ("truncate", C.c_double), ("radius", C.c_int64)]


class Correlate1dSettings(C.Structure):
    _fields_ = [("axis", C.c_int64), ("mode", C.c_int32), ("cval", C.c_double), ("origin", C.c_int32)]


class Response(C.Structure):
    _fields_ = [("kind", C.c_int32), ("sigma", C.c_double), ("sigma2", C.c_double), ("amount", C.c_double),
                ("out", Tensor)]


class Block(C.Structure):
    _fields_ = [("index", C.c_int64), ("origin", C.c_int64 * 3), ("size", C.c_int64 * 3),
                ("read_origin", C.c_int64 * 3), ("read_size", C.c_int64 * 3)]


class RlSettings(C.Structure):
    _fields_ = [("num_iter", C.c_int32), ("clip", C.c_int32), ("has_filter_epsilon", C.c_int32),
                ("filter_epsilon", C.c_double), ("mode", C.c_int32), ("grid", C.c_int64 * 3)]


class WienerSettings(C.Structure):
    _fields_ = [("balance", C.c_double), ("clip", C.c_int32)]


class PhaseCorrelationSettings(C.Structure):
    _fields_ = [("upsample_factor", C.c_int64), ("normalize_phase", C.c_int32)]


class PhaseCorrelationResult(C.Structure):
    _fields_ = [("shift", C.c_double * MAX_DIMS), ("error", C.c_double), ("phasediff", C.c_double)]


class RidgeSettings(C.Structure):
    _fields_ = [("sigmas", C.POINTER(C.c_double)), ("n_sigmas", C.c_int32), ("black_ridges", C.c_int32),
                ("mode", C.c_int32), ("cval", C.c_double), ("beta", C.c_double), ("gamma", C.c_double)]


class PyramidSettings(C.Structure):
    _fields_ = [("downscale", C.c_double), ("sigma", C.c_double), ("order", C.c_int32), ("mode", C.c_int32),
                ("cval", C.c_double)]


class BlobSettings(C.Structure):
    _fields_ = [("min_sigma", C.c_double), ("max_sigma", C.c_double), ("num_sigma", C.c_int64),
                ("sigma_ratio", C.c_double), ("threshold", C.c_double), ("overlap", C.c_double),
                ("log_scale", C.c_int32), ("exclude_border", C.c_int64)]


class CannySettings(C.Structure):
    _fields_ = [("sigma", C.c_double), ("has_low", C.c_int32), ("low_threshold", C.c_double),
                ("has_high", C.c_int32), ("high_threshold", C.c_double), ("use_quantiles", C.c_int32),
                ("mode", C.c_int32), ("cval", C.c_double)]


class BlobC(C.Structure):
    _fields_ = [("y", C.c_int64), ("x", C.c_int64), ("sigma", C.c_double), ("response", C.c_double)]


class UnsupervisedWienerSettings(C.Structure):
    _fields_ = [("num_iter", C.c_int64), ("burnin", C.c_int64), ("clip", C.c_int32), ("seed", C.c_uint64)]


# name -> (restype, argtypes); every function include/lucem_b200.h declares.
P = C.c_void_p
PP = C.POINTER(C.c_void_p)
TP = C.POINTER(Tensor)
D = C.c_double
I32 = C.c_int32
I64 = C.c_int64
DP = C.POINTER(C.c_double)
I64P = C.POINTER(C.c_int64)
SIGNATURES = {
    "lucem_abi_version": (I32, []),
    "lucem_last_error_message": (C.c_char_p, []),
    "lucem_ctx_create": (I32, [I32, PP]),
    "lucem_ctx_destroy": (None, [P]),
    "lucem_workspace_create": (I32, [P, PP]),
    "lucem_workspace_destroy": (None, [P]),
    "lucem_workspace_capacity_bytes": (C.c_size_t, [P]),
    "lucem_workspace_set_timing": (I32, [P, I32]),
    "lucem_workspace_set_wait_limit": (I32, [P, I64]),
    "lucem_fft_nd": (I32, [P, TP, TP, TP, TP, I32, P, P]),
    "lucem_fft_1d": (I32, [P, TP, TP, TP, TP, I32, I32, P, P]),
    "lucem_complex_mul": (I32, [TP, TP, TP, TP, TP, TP, I32, P]),
    "lucem_wiener_settings_default": (None, [C.POINTER(WienerSettings)]),
    "lucem_wiener_deconvolve": (I32, [P, TP, TP, C.POINTER(WienerSettings), TP, P, P]),
    "lucem_fourier_gaussian": (I32, [P, TP, TP, DP, I32, P]),
    "lucem_fourier_box": (I32, [P, TP, TP, DP, I32, P]),
    "lucem_fourier_shift": (I32, [P, TP, TP, DP, I32, P]),
    "lucem_butterworth": (I32, [P, TP, D, I32, D, TP, P, P]),
    "lucem_phase_correlation_settings_default": (None, [C.POINTER(PhaseCorrelationSettings)]),
    "lucem_phase_correlation": (I32, [P, TP, TP, C.POINTER(PhaseCorrelationSettings),
                                      C.POINTER(PhaseCorrelationResult), P, P]),
    "lucem_hessian_matrix": (I32, [P, TP, D, I32, D, TP, TP, TP, P, P]),
    "lucem_hessian_det": (I32, [P, TP, D, I32, D, TP, P, P]),
    "lucem_hessian_eigvals": (I32, [P, TP, D, I32, D, TP, TP, P, P]),
    "lucem_shape_index": (I32, [P, TP, D, I32, D, TP, P, P]),
    "lucem_structure_tensor": (I32, [P, TP, D, I32, D, TP, TP, TP, P, P]),
    "lucem_structure_tensor_eigvals": (I32, [TP, TP, TP, TP, TP, P]),
    "lucem_ridge_settings_default": (None, [C.POINTER(RidgeSettings)]),
    "lucem_frangi": (I32, [P, TP, C.POINTER(RidgeSettings), TP, P, P]),
    "lucem_sato": (I32, [P, TP, C.POINTER(RidgeSettings), TP, P, P]),
    "lucem_meijering": (I32, [P, TP, C.POINTER(RidgeSettings), TP, P, P]),
    "lucem_pyramid_settings_default": (None, [C.POINTER(PyramidSettings)]),
    "lucem_pyramid_reduce": (I32, [P, TP, C.POINTER(PyramidSettings), TP, P, P]),
    "lucem_pyramid_expand": (I32, [P, TP, C.POINTER(PyramidSettings), TP, P, P]),
    "lucem_laplacian_band": (I32, [P, TP, TP, C.POINTER(PyramidSettings), TP, P, P]),
    "lucem_canny_settings_default": (None, [C.POINTER(CannySettings)]),
    "lucem_canny": (I32, [P, TP, C.POINTER(CannySettings), TP, P, P]),
    "lucem_blob_settings_default": (None, [C.POINTER(BlobSettings)]),
    "lucem_blobs_log": (I32, [P, TP, C.POINTER(BlobSettings), C.POINTER(BlobC), I64, I64P, P, P]),
    "lucem_blobs_dog": (I32, [P, TP, C.POINTER(BlobSettings), C.POINTER(BlobC), I64, I64P, P, P]),
    "lucem_blobs_doh": (I32, [P, TP, C.POINTER(BlobSettings), C.POINTER(BlobC), I64, I64P, P, P]),
    "lucem_unsupervised_wiener_settings_default": (None, [C.POINTER(UnsupervisedWienerSettings)]),
    "lucem_unsupervised_wiener": (I32, [P, TP, TP, C.POINTER(UnsupervisedWienerSettings), TP, DP, P, P]),
    "lucem_workspace_wait_status": (I32, [P, P, I64P]),
    "lucem_workspace_timings": (I32, [P, C.c_char_p, DP, I64P, I32, C.POINTER(I32)]),
    "lucem_pad_mode_parse": (I32, [C.c_char_p, C.POINTER(I32)]),
    "lucem_gaussian_kernel_1d": (I32, [D, C.c_uint32, I64, DP]),
    "lucem_gaussian_radius": (I64, [D, D]),
    "lucem_pad_index": (I64, [I64, I64, I32]),
    "lucem_gaussian_settings_default": (None, [C.POINTER(GaussianSettings)]),
    "lucem_gaussian_blur": (I32, [P, TP, DP, I32, C.POINTER(GaussianSettings), TP, P, P]),
    "lucem_gaussian_blur_adjoint": (I32, [P, TP, DP, I32, C.POINTER(GaussianSettings), TP, P, P]),
    "lucem_gaussian_blur_noalloc": (I32, [TP, DP, I32, C.POINTER(GaussianSettings), TP, P]),
    "lucem_gaussian_1d_settings_default": (None, [C.POINTER(Gaussian1dSettings)]),
    "lucem_gaussian_1d": (I32, [P, TP, D, C.POINTER(Gaussian1dSettings), TP, P]),
    "lucem_correlate_1d": (I32, [P, TP, DP, I64, C.POINTER(Correlate1dSettings), TP, P]),
    "lucem_difference_of_gaussians": (I32, [P, TP, DP, I32, DP, I32, C.POINTER(GaussianSettings), TP, P, P]),
    "lucem_gaussian_laplace": (I32, [P, TP, DP, I32, I32, D, D, TP, P, P]),
    "lucem_gaussian_grad_mag": (I32, [P, TP, DP, I32, I32, D, D, TP, P, P]),
    "lucem_unsharp_mask": (I32, [P, TP, DP, I32, D, C.POINTER(GaussianSettings), TP, P, P]),
    "lucem_gaussian_family": (I32, [P, TP, C.POINTER(Response), I32, I32, D, D, D, P, P]),
    "lucem_schedule": (I32, [I64P, I64P, I64P, C.POINTER(Block), I64, I64P]),
    "lucem_gaussian_family_tiles": (I32, [P, TP, C.POINTER(Block), I64, C.POINTER(Response), I32, I32, D, D,
                                          D, I32, P, P]),
    "lucem_rl_settings_default": (None, [C.POINTER(RlSettings)]),
    "lucem_richardson_lucy": (I32, [P, TP, TP, C.POINTER(RlSettings), TP, P, P]),
    "lucem_rl_grid": (I32, [I64P, I64P, I32, I32, I64P, I64P]),
    "lucem_richardson_lucy_backward": (I32, [P, TP, TP, C.POINTER(RlSettings), TP, I32, TP, TP, P, P]),
    "lucem_fft_convolve": (I32, [P, TP, TP, I32, I64P, TP, P, P]),
    "lucem_fft_convolve_backward": (I32, [P, TP, TP, I32, I64P, TP, TP, TP, P, P]),
    "lucem_gaussian_batch": (I32, [P, I32, TP, TP, C.POINTER(I32), I32, DP, I32, C.c_double, C.c_double,
                                    C.c_double, P, P]),
    "lucem_rl_batch_create": (I32, [P, I32, TP, TP, C.POINTER(RlSettings), TP, P, P, C.POINTER(P)]),
    "lucem_rl_batch_run": (I32, [P, I32, P, P]),
    "lucem_rl_batch_info": (I32, [P, I64P, C.POINTER(I32), C.POINTER(I32)]),
    "lucem_rl_batch_destroy": (None, [P]),
    "lucem_autotune_fft": (I32, [P, I64P, I32, P, P]),
    "lucem_autotune_query": (I32, [P, I32, I64, C.POINTER(C.c_double)]),
    "lucem_autotune_save": (I32, [P, C.c_char_p]),
    "lucem_autotune_load": (I32, [P, C.c_char_p]),
    "lucem_autotune_enable": (I32, [P, I32]),
    "lucem_autotune_plans": (I32, [P, C.c_char_p, C.POINTER(I32), I32, C.POINTER(I32)]),
    "lucem_graph_begin": (I32, [P]),
    "lucem_graph_end": (I32, [P, C.POINTER(P)]),
    "lucem_graph_launch": (I32, [P, P]),
    "lucem_graph_destroy": (None, [P]),
    "lucem_fft_good_length": (I64, [I64, I32]),
}

_lib = None
_lock = threading.Lock()


class LucemError(ValueError):
    """A non-OK lucem_status; `status` is the code, `name` its enumerator."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.name}: {message}")


def lib():
    """The loaded library; raises if it was not built (there is no fallback)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(f"{LIB_PATH} is missing: build it with `python -m lucem_b200.build`")
                L = C.CDLL(LIB_PATH)
                for name, (res, args) in SIGNATURES.items():
                    f = getattr(L, name)
                    f.restype = res
                    f.argtypes = args
                _lib = L
    return _lib


def check(status: int):
    if status != 0:
        msg = lib().lucem_last_error_message().decode("utf-8", "replace")
        raise LucemError(status, msg)


def exported_symbols():
    return list(SIGNATURES)
