"""ctypes binding of ``libpytme_b200.so`` (declared in ``include/pytme_b200.h``).

The library is required: importing this module raises if it is missing, and no
operation of the package falls back to a CPU implementation. Status codes are
mapped to the exception types the reference raises for the same conditions
(``ValueError`` for bad arguments, ``MemoryError`` for allocation failures,
``NotImplementedError`` for unsupported requests, ``TimeoutError`` for a device wait
that gave up, ``RuntimeError`` otherwise).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_float, c_int, c_int32, c_int64
from ctypes import c_size_t, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PYTME_B200_LIB", os.path.join(_HERE, "libpytme_b200.so"))

TM_OK = 0
TM_E_INVALID = -1
TM_E_OOM = -2
TM_E_CUFFT = -3
TM_E_CUDA = -4
TM_E_TIMEOUT = -5
TM_E_UNSUPPORTED = -6

TM_SCORE_CC = 0
TM_SCORE_FLC = 1
TM_SCORE_FLCSM = 2
TM_PREC_FP32 = 0
TM_PREC_MIXED = 1
STAGES = ("prepare", "template", "xpass", "ypass", "zpass")

EXPORTED = (
    "tm_version", "tm_last_error", "tm_set_device_memory_limit", "tm_rigid_transform", "tm_normalize_template_workspace",
    "tm_normalize_template", "tm_norm_scores", "tm_max_score_over_rotations",
    "tm_fft_plan_create", "tm_fft_plan_destroy", "tm_fft_r2c", "tm_fft_c2r",
    "tm_scan_create", "tm_scan_destroy", "tm_scan_device_bytes", "tm_scan_set_template",
    "tm_scan_set_target", "tm_scan_run", "tm_scan_set_timing", "tm_scan_set_graph",
    "tm_scan_get_timing",
    "tm_scan_stage_bytes", "tm_max_filter_peaks",
    "tm_find_candidate_indices_workspace", "tm_find_candidate_indices",
    "tm_find_candidate_indices_noalloc", "tm_fft_filter",
    "tm_euler_zyz", "tm_refine_rotate", "tm_refine_forward", "tm_refine_grad_filtered",
    "tm_refine_backward", "tm_spline_prefilter", "tm_rigid_transform_cubic",
    "tm_scan_set_interpolation", "tm_build_filter", "tm_whitening_bins", "tm_whitening_filter",
    "tm_scan_set_xpass", "tm_scan_check", "tm_scan_xpass_mode", "tm_scan_set_zpass",
    "tm_scan_zpass_mode", "tm_scan_set_ypass", "tm_scan_ypass_mode", "tm_scan_set_wait_budget",
)
# exported for the test suite only (pytme_b200/csrc/diagnostics.h), not public interface
DIAGNOSTICS = ("tm_line_fft_test", "tm_xcorr_tc_test")


class ScanDesc(Structure):
    _fields_ = [
        ("score", c_int),
        ("precision", c_int),
        ("fast_shape", c_int * 3),
        ("template_shape", c_int * 3),
        ("batch", c_int),
        ("plain", c_int),
        ("has_template_filter", c_int),
    ]


TM_FILTER_CTF = 1
TM_FILTER_WEDGE = 2
TM_FILTER_MAX_COMPONENTS = 4


class FilterComponent(Structure):
    _fields_ = [("kind", c_int), ("p", c_double * 8)]


class RefineDesc(Structure):
    _fields_ = [
        ("tmpl", c_void_p),
        ("mask", c_void_p),
        ("template_shape", c_int * 3),
        ("target", c_void_p),
        ("target_shape", c_int * 3),
        ("target_outside", c_float),
        ("rot", c_void_p),
        ("shifts", c_void_p),
        ("corners", c_void_p),
        ("n_peaks", c_int),
        ("eps", c_double),
    ]


class NativeError(RuntimeError):
    """Error status from the CUDA library that maps to no more specific type."""


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"pytme_b200: CUDA library not found at {LIB_PATH}; build it with "
            "`python pytme_b200/build.py` (there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    vp, f32p, i32p, i64 = c_void_p, c_void_p, c_void_p, c_int64
    sig = {
        "tm_version": (c_int, []),
        "tm_last_error": (c_int, [c_char_p, c_size_t]),
        "tm_set_device_memory_limit": (c_int, [c_int64]),
        "tm_rigid_transform": (c_int, [f32p, f32p, c_int, c_int, c_int, f32p, c_int, f32p, f32p,
                                       c_int, c_int, c_int, vp]),
        "tm_normalize_template_workspace": (c_int64, [c_int]),
        "tm_normalize_template": (c_int, [f32p, f32p, i64, c_int, i64, c_double, vp, vp]),
        "tm_norm_scores": (c_int, [f32p, f32p, f32p, c_double, f32p, c_double, f32p, i64, vp]),
        "tm_max_score_over_rotations": (c_int, [f32p, f32p, i32p, c_int32, i64, vp]),
        "tm_fft_plan_create": (c_int, [c_int, POINTER(c_int), c_int, c_int, POINTER(c_void_p)]),
        "tm_fft_plan_destroy": (c_int, [vp]),
        "tm_fft_r2c": (c_int, [vp, vp, vp, vp]),
        "tm_fft_c2r": (c_int, [vp, vp, vp, c_double, vp]),
        "tm_scan_create": (c_int, [POINTER(ScanDesc), POINTER(c_void_p)]),
        "tm_scan_destroy": (c_int, [vp]),
        "tm_scan_device_bytes": (c_int64, [vp]),
        "tm_scan_set_template": (c_int, [vp, f32p, f32p, f32p, vp]),
        "tm_scan_set_target": (c_int, [vp, f32p, vp]),
        "tm_scan_run": (c_int, [vp, f32p, c_int, c_int32, f32p, i32p, vp]),
        "tm_scan_set_timing": (c_int, [vp, c_int]),
        "tm_scan_set_graph": (c_int, [vp, c_int]),
        "tm_scan_get_timing": (c_int, [vp, vp, vp]),
        "tm_scan_stage_bytes": (c_int64, [vp, c_int, c_int]),
        "tm_max_filter_peaks": (c_int, [f32p, c_int, c_int, c_int, c_int, f32p, f32p, vp, vp]),
        "tm_find_candidate_indices_workspace": (c_int64, [c_int]),
        "tm_find_candidate_indices": (c_int, [vp, c_int, c_int64, i32p, i32p, vp, vp]),
        "tm_find_candidate_indices_noalloc": (c_int, [vp, c_int, c_int64, i32p, i32p, vp]),
        "tm_line_fft_test": (c_int, [vp, vp, c_int, c_int, c_int, vp]),
        "tm_fft_filter": (c_int, [vp, f32p, vp, f32p, vp]),
        "tm_spline_prefilter": (c_int, [f32p, vp, c_int, c_int, c_int, c_int, vp]),
        "tm_rigid_transform_cubic": (c_int, [vp, vp, c_int, c_int, c_int, f32p, c_int, f32p,
                                             f32p, c_int, c_int, c_int, vp]),
        "tm_scan_set_interpolation": (c_int, [vp, c_int, vp]),
        "tm_scan_set_xpass": (c_int, [vp, c_int]),
        "tm_scan_check": (c_int, [vp, vp]),
        "tm_scan_xpass_mode": (c_int, [vp]),
        "tm_scan_set_zpass": (c_int, [vp, c_int]),
        "tm_scan_zpass_mode": (c_int, [vp]),
        "tm_scan_set_ypass": (c_int, [vp, c_int]),
        "tm_scan_ypass_mode": (c_int, [vp]),
        "tm_scan_set_wait_budget": (c_int, [vp, ctypes.c_uint32]),
        "tm_build_filter": (c_int, [vp, c_int, POINTER(c_int), c_int, f32p, vp]),
        "tm_whitening_bins": (c_int, [POINTER(c_int), c_int]),
        "tm_whitening_filter": (c_int, [vp, POINTER(c_int), c_int, POINTER(c_int), c_int, vp,
                                        vp, f32p, vp]),
        "tm_xcorr_tc_test": (c_int, [vp, vp, c_int, c_int, c_int, c_int, c_int, c_float, vp,
                                     c_int, vp]),
        "tm_euler_zyz": (c_int, [f32p, c_int, f32p, f32p, vp]),
        "tm_refine_rotate": (c_int, [POINTER(RefineDesc), f32p, vp]),
        "tm_refine_forward": (c_int, [POINTER(RefineDesc), f32p, vp, f32p, vp]),
        "tm_refine_grad_filtered": (c_int, [POINTER(RefineDesc), f32p, vp, f32p, f32p, vp]),
        "tm_refine_backward": (c_int, [POINTER(RefineDesc), f32p, f32p, vp, f32p, f32p, vp, vp,
                                       vp, f32p, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib.tm_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, what: str = "") -> None:
    """Raise the exception that matches a TM_E_* status."""
    if status == TM_OK:
        return
    msg = f"{what}: {last_error()}" if what else last_error()
    if status == TM_E_INVALID:
        raise ValueError(msg)
    if status == TM_E_OOM:
        raise MemoryError(msg)
    if status == TM_E_UNSUPPORTED:
        raise NotImplementedError(msg)
    if status == TM_E_TIMEOUT:
        raise TimeoutError(msg)
    raise NativeError(f"{msg} (status {status})")


def ptr(t) -> int:
    """Device address of a CUDA torch tensor (None for None). A host tensor raises
    ValueError: every kernel argument of the library is device memory."""
    if t is None:
        return None
    if not getattr(t, "is_cuda", False):
        raise ValueError("pytme_b200 kernels take CUDA tensors; got "
                         f"{type(t).__name__} on {getattr(t, 'device', 'host')}")
    return t.data_ptr()


def stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
