"""Score setup/scoring pairs with the reference's registry interface.

``MATCHING_EXHAUSTIVE_REGISTER`` maps "CC", "FLC" and "FLCSphericalMask" to
``(setup, scoring)`` pairs with the signatures of tme/matching_scores.py. The
setup functions build a ``ScanPlan`` (the ``tm_scan`` plan of the CUDA library)
and hand it the reversed template, mask, template filter and the padded,
filtered target; the scoring functions stream a rotation chunk through it.

When the callback is a ``MaxScoreOverRotations`` proxy (the reference's or this
package's) the whole chunk runs fused on the device and the proxy's state is
left exactly as B sequential ``callback(scores, rotation_matrix=R)`` calls would
leave it under ``inversion_mapping``. Any other analyzer receives one score map
per rotation, as in the reference loop.
"""
from __future__ import annotations

import os
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _native as N
from .matching import rigid_transform_matrices

__all__ = [
    "ScanPlan",
    "cc_setup",
    "flc_setup",
    "flcSphericalMask_setup",
    "corr_scoring",
    "flc_scoring",
    "MATCHING_EXHAUSTIVE_REGISTER",
    "register_matching_exhaustive",
    "default_precision",
]

_SCORE_CODES = {"CC": N.TM_SCORE_CC, "FLC": N.TM_SCORE_FLC, "FLCSphericalMask": N.TM_SCORE_FLCSM}


def default_precision() -> Dict:
    """Plan options taken from the active backend (``change_backend("b200", ...)``)."""
    from .backend import current_options

    return current_options()


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("pytme_b200 needs a CUDA device; there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def _to_device(arr, dtype=torch.float32) -> torch.Tensor:
    if isinstance(arr, torch.Tensor):
        return arr.to(device=_device(), dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype, device=_device()).contiguous()


class ScanPlan:
    """Owner of one ``tm_scan`` plan (device scratch, spectra and cuFFT plans)."""

    def __init__(self, score: str, fast_shape, template_shape, precision: str = "fp32",
                 batch: int = 32, plain: bool = False):
        desc = N.ScanDesc()
        desc.score = _SCORE_CODES[score]
        desc.precision = N.TM_PREC_MIXED if precision == "mixed" else N.TM_PREC_FP32
        for i in range(3):
            desc.fast_shape[i] = int(fast_shape[i])
            desc.template_shape[i] = int(template_shape[i])
        desc.batch = int(batch)
        desc.plain = int(bool(plain))
        desc.has_template_filter = 0
        self.score = score
        self.fast_shape = tuple(int(x) for x in fast_shape)
        self.template_shape = tuple(int(x) for x in template_shape)
        self.precision = precision
        self.batch = int(batch)
        self.plain = bool(plain)
        handle = N.c_void_p()
        _device()
        st = N.lib.tm_scan_create(N.ctypes.byref(desc), N.ctypes.byref(handle))
        if st == N.TM_E_UNSUPPORTED and not plain:
            # shapes outside the fused kernels' range run on the plain path
            desc.plain = 1
            desc.precision = N.TM_PREC_FP32
            self.plain, self.precision = True, "fp32"
            st = N.lib.tm_scan_create(N.ctypes.byref(desc), N.ctypes.byref(handle))
        N.check(st, "tm_scan_create")
        self._h = handle
        self._keep = []

    @property
    def device_bytes(self) -> int:
        return int(N.lib.tm_scan_device_bytes(self._h))

    def set_template(self, template_rev, mask_rev=None, template_filter=None, stream=None):
        t = _to_device(template_rev)
        m = None if mask_rev is None else _to_device(mask_rev)
        f = None if template_filter is None else _to_device(template_filter)
        if f is not None and f.numel() == 1:
            f = None
        self._keep = [t, m, f]
        N.check(N.lib.tm_scan_set_template(self._h, N.ptr(t), N.ptr(m), N.ptr(f),
                                           N.stream_ptr(stream)), "tm_scan_set_template")

    def set_interpolation(self, order: int, stream=None):
        """Template rotation order: 1 trilinear, 3 cubic B-spline (SciPy's prefiltered
        spline for the template, unfiltered for the FLC mask)."""
        order = int(order)
        if order == getattr(self, "_order", 1):
            return
        N.check(N.lib.tm_scan_set_interpolation(self._h, order, N.stream_ptr(stream)),
                "tm_scan_set_interpolation")
        self._order = order

    def set_target(self, target_fast, stream=None):
        t = _to_device(target_fast)
        if tuple(t.shape) != self.fast_shape:
            raise ValueError(f"target has shape {tuple(t.shape)}, plan expects {self.fast_shape}")
        N.check(N.lib.tm_scan_set_target(self._h, N.ptr(t), N.stream_ptr(stream)),
                "tm_scan_set_target")

    def run(self, matrices: torch.Tensor, first_index: int, max_scores: torch.Tensor,
            argmax: torch.Tensor, stream=None):
        if tuple(max_scores.shape) != self.fast_shape or tuple(argmax.shape) != self.fast_shape:
            raise ValueError("state arrays must have the plan's fast shape")
        if max_scores.dtype != torch.float32 or argmax.dtype != torch.int32:
            raise ValueError("state arrays must be float32 scores and int32 indices")
        if not (max_scores.is_contiguous() and argmax.is_contiguous()):
            raise ValueError("state arrays must be contiguous")
        n = int(matrices.shape[0])
        N.check(N.lib.tm_scan_run(self._h, N.ptr(matrices), n, int(first_index),
                                  N.ptr(max_scores), N.ptr(argmax), N.stream_ptr(stream)),
                "tm_scan_run")

    def set_xpass(self, mode: str = "auto"):
        """x pass on the tensor cores ("tensor"), as FFTs on the CUDA cores ("fft"), or
        the plan's default ("auto": tensor cores for mixed precision where supported)."""
        code = {"tensor": 0, "fft": 1, "auto": 2}[mode]
        N.check(N.lib.tm_scan_set_xpass(self._h, code), "tm_scan_set_xpass")

    def set_zpass(self, mode: str = "auto"):
        """z pass on the tensor cores ("tensor"), as FFTs on the CUDA cores ("fft"), or
        the plan's default ("auto": tensor cores for mixed precision where supported)."""
        code = {"tensor": 0, "fft": 1, "auto": 2}[mode]
        N.check(N.lib.tm_scan_set_zpass(self._h, code), "tm_scan_set_zpass")

    def set_ypass(self, mode: str = "auto"):
        """y pass on the tensor cores ("tensor": radix 16 in FP32 registers, radix n1/16 on
        the tensor cores; behind the warp-specialised tensor-core x pass it reads spectra
        stored with x' innermost and writes row-major rows into a second buffer), the same
        in place on row-major spectra ("tensor-inplace"), with both DFT stages on the
        tensor cores ("tensor2"; needs the tensor-core x pass), as FFTs on the CUDA cores
        ("fft"), or the plan's default ("auto")."""
        code = {"tensor": 0, "fft": 1, "auto": 2, "tensor2": 3, "tensor-inplace": 4}[mode]
        N.check(N.lib.tm_scan_set_ypass(self._h, code), "tm_scan_set_ypass")

    @property
    def ypass(self) -> str:
        """The y pass this plan runs: "tensor", "tensor-inplace", "tensor2" or "fft"."""
        return {0: "tensor", 1: "fft", 3: "tensor2", 4: "tensor-inplace"}[
            N.lib.tm_scan_ypass_mode(self._h)]

    def set_wait_budget(self, iters: int = 0):
        """Polls of every data wait in the tensor-core kernels (0: the default). A wait
        that runs out makes ``check`` raise TimeoutError and invalidates that run."""
        N.check(N.lib.tm_scan_set_wait_budget(self._h, int(iters)), "tm_scan_set_wait_budget")

    @property
    def zpass(self) -> str:
        """The z pass this plan runs: "tensor" or "fft"."""
        return "tensor" if N.lib.tm_scan_zpass_mode(self._h) == 0 else "fft"

    @property
    def xpass(self) -> str:
        """The x pass this plan runs: "tensor" or "fft"."""
        return "tensor" if N.lib.tm_scan_xpass_mode(self._h) == 0 else "fft"

    def check(self, stream=None):
        """Synchronise and raise if a bounded wait of a tensor-core kernel gave up."""
        N.check(N.lib.tm_scan_check(self._h, N.stream_ptr(stream)), "tm_scan_check")

    def set_graph(self, enable: bool = True):
        """Replay full launch groups from one captured CUDA graph."""
        N.check(N.lib.tm_scan_set_graph(self._h, int(bool(enable))), "tm_scan_set_graph")

    def set_timing(self, enable: bool = True):
        """Bracket each fused-path stage with CUDA events (resets the counters)."""
        N.check(N.lib.tm_scan_set_timing(self._h, int(bool(enable))), "tm_scan_set_timing")

    def get_timing(self) -> Dict[str, Tuple[float, int]]:
        """{stage: (total ms, launches)} accumulated since ``set_timing``."""
        ms = (N.ctypes.c_double * 5)()
        cnt = (N.ctypes.c_int64 * 5)()
        N.check(N.lib.tm_scan_get_timing(self._h, N.ctypes.cast(ms, N.c_void_p),
                                         N.ctypes.cast(cnt, N.c_void_p)), "tm_scan_get_timing")
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(N.STAGES)}

    def stage_bytes(self, stage: str, nb: int) -> int:
        """Algorithmic HBM bytes of one launch of ``stage`` for ``nb`` rotations."""
        return int(N.lib.tm_scan_stage_bytes(self._h, N.STAGES.index(stage), int(nb)))

    def close(self):
        if getattr(self, "_h", None):
            N.lib.tm_scan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ target preparation
def _prepare_target(target, fast_shape, target_filter=None) -> torch.Tensor:
    """Top-left pad to the transform shape; with a target filter, multiply it into the
    spectrum once and keep the top-left target-shaped crop of the inverse
    (tme/matching_exhaustive.py:84-117), then pad again."""
    from .backend import fft_plan

    t = _to_device(target)
    pad = torch.zeros(fast_shape, dtype=torch.float32, device=t.device)
    pad[tuple(slice(0, min(a, b)) for a, b in zip(t.shape, fast_shape))] = \
        t[tuple(slice(0, min(a, b)) for a, b in zip(t.shape, fast_shape))]
    if target_filter is None:
        return pad
    filt = _to_device(target_filter)
    plan = fft_plan(tuple(fast_shape))
    spec = plan.rfftn(pad)
    spec *= filt.reshape(spec.shape)
    full = plan.irfftn(spec)
    out = torch.zeros_like(pad)
    box = tuple(slice(0, min(a, b)) for a, b in zip(t.shape, fast_shape))
    out[box] = full[box]
    return out


def _template_arrays(matching_data):
    tmpl = np.ascontiguousarray(np.asarray(_host(matching_data.template), dtype=np.float32))
    mask = matching_data.template_mask
    if mask is not None:
        mask = np.ascontiguousarray(np.asarray(_host(mask), dtype=np.float32))
    return tmpl, mask


def _host(arr):
    if isinstance(arr, torch.Tensor):
        return arr.detach().cpu().numpy()
    return np.asarray(arr)


def _setup(score: str, matching_data, fast_shape, template_filter=None, target_filter=None,
           **kwargs) -> Dict:
    opts = default_precision()
    tmpl, mask = _template_arrays(matching_data)
    if score in ("FLC", "FLCSphericalMask") and mask is None:
        raise ValueError(f"{score} requires a template mask")
    plan = ScanPlan(score, fast_shape, tmpl.shape, precision=opts["precision"],
                    batch=opts["rotation_batch"], plain=opts["plain"])
    if opts.get("xpass", "auto") != "auto" and not plan.plain and score != "FLC":
        try:
            plan.set_xpass(opts["xpass"])
        except NotImplementedError:
            pass  # shapes the tensor-core x pass does not cover keep the FFT x pass
    if opts.get("zpass", "auto") != "auto" and not plan.plain and score != "FLC":
        try:
            plan.set_zpass(opts["zpass"])
        except NotImplementedError:
            pass
    if opts.get("ypass", "auto") != "auto" and not plan.plain and score != "FLC":
        try:
            plan.set_ypass(opts["ypass"])
        except NotImplementedError:
            pass
    tf = None
    if template_filter is not None:
        tf = template_filter if isinstance(template_filter, torch.Tensor) else \
            np.asarray(_host(template_filter), dtype=np.float32)
        n_tf = tf.numel() if isinstance(tf, torch.Tensor) else tf.size
        if n_tf <= 1:
            tf = None
    if tf is not None:
        expect = (tmpl.shape[0], tmpl.shape[1], tmpl.shape[2] // 2 + 1)
        n_tf = tf.numel() if isinstance(tf, torch.Tensor) else tf.size
        if n_tf != int(np.prod(expect)):
            raise NotImplementedError(
                f"template filter of shape {tuple(tf.shape)} is not at the template's rfft "
                f"shape {expect}; only pad_template_filter=False filters are supported")
        tf = tf.reshape(expect)
    plan.set_template(tmpl, mask, tf)
    target = _prepare_target(_host(matching_data.target), tuple(fast_shape), target_filter)
    plan.set_target(target)
    return {"plan": plan, "fast_shape": tuple(fast_shape),
            "template_shape": tuple(tmpl.shape), "score": score}


def cc_setup(matching_data, fast_shape, fast_ft_shape=None, shm_handler=None, **kwargs) -> Dict:
    """cc_setup (tme/matching_scores.py:153-189): raw cross-correlation."""
    return _setup("CC", matching_data, fast_shape, **kwargs)


def flc_setup(matching_data, fast_shape, fast_ft_shape=None, shm_handler=None, **kwargs) -> Dict:
    """flc_setup (tme/matching_scores.py:357-387): spectra of f and f^2 for the
    per-rotation local statistics under the rotated mask."""
    return _setup("FLC", matching_data, fast_shape, **kwargs)


def flcSphericalMask_setup(matching_data, fast_shape, fast_ft_shape=None, shm_handler=None,
                           **kwargs) -> Dict:
    """flcSphericalMask_setup (tme/matching_scores.py:390-450): target spectrum and
    the inverse local-variance denominator under the unrotated mask (FP64)."""
    return _setup("FLCSphericalMask", matching_data, fast_shape, **kwargs)


# ------------------------------------------------------------------ scoring
def _fused_state(callback):
    """(scores, rotations, mapping) of a MaxScoreOverRotations proxy that uses
    inversion mapping, else None."""
    if callback is None:
        return None
    analyzer = getattr(callback, "_analyzer", None)
    state = getattr(callback, "_state", None)
    if analyzer is None or state is None or getattr(callback, "_shared", False):
        return None
    if type(analyzer).__name__ != "MaxScoreOverRotations":
        return None
    if not getattr(analyzer, "_inversion_mapping", False):
        return None
    scores, rotations, mapping = state
    if not (isinstance(scores, torch.Tensor) and scores.is_cuda):
        return None
    return scores, rotations, mapping


def _matrices(rotations, template_shape) -> Tuple[torch.Tensor, np.ndarray]:
    rot = np.ascontiguousarray(_host(rotations), dtype=np.float32).reshape(-1, 3, 3)
    center = np.divide(np.asarray(template_shape) - 1, 2)
    mats = rigid_transform_matrices(rot, center)
    return _to_device(mats), rot


def _score_chunk(plan: "ScanPlan", rotations, callback, interpolation_order: int):
    plan.set_interpolation(interpolation_order)
    mats, rot = _matrices(rotations, plan.template_shape)
    n = rot.shape[0]
    if n == 0:
        return callback
    fused = _fused_state(callback)
    if fused is not None:
        scores, rotidx, mapping = fused
        first = len(mapping)
        plan.run(mats, first, scores, rotidx)
        for i in range(n):
            mapping[first + i] = rot[i]
        return callback
    scratch_s = torch.empty(plan.fast_shape, dtype=torch.float32, device=mats.device)
    scratch_r = torch.empty(plan.fast_shape, dtype=torch.int32, device=mats.device)
    for i in range(n):
        scratch_s.fill_(-float("inf"))
        plan.run(mats[i:i + 1], 0, scratch_s, scratch_r)
        if callback is not None:
            callback(scratch_s, rotation_matrix=rot[i])
    return callback


def corr_scoring(plan: "ScanPlan", rotations, callback, interpolation_order: int = 3,
                 template_filter=None, **kwargs):
    """corr_scoring (tme/matching_scores.py:491-626) for CC and FLCSphericalMask."""
    return _score_chunk(plan, rotations, callback, interpolation_order)


def flc_scoring(plan: "ScanPlan", rotations, callback, interpolation_order: int = 3,
                template_filter=None, **kwargs):
    """flc_scoring (tme/matching_scores.py:629-759): rotated mask, per-rotation local
    statistics."""
    return _score_chunk(plan, rotations, callback, interpolation_order)


MATCHING_EXHAUSTIVE_REGISTER = {
    "CC": (cc_setup, corr_scoring),
    "FLC": (flc_setup, flc_scoring),
    "FLCSphericalMask": (flcSphericalMask_setup, corr_scoring),
}


def register_matching_exhaustive(matching: str, matching_setup, matching_scoring,
                                 memory_class=None) -> None:
    """tme/matching_exhaustive.py:468-501: add a score; duplicates raise ValueError."""
    if matching in MATCHING_EXHAUSTIVE_REGISTER:
        raise ValueError(f"A method with name '{matching}' is already registered.")
    MATCHING_EXHAUSTIVE_REGISTER[matching] = (matching_setup, matching_scoring)
