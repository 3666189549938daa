"""Exhaustive-matching driver with the reference's call signatures.

``MatchingData``, ``scan`` and ``scan_subsets`` mirror
tme/matching_data.py and tme/matching_exhaustive.py for unbatched 3D targets and
templates: target splitting with reflect padding (``pad_target_edges``), Fourier
padding and shifts, the template/target filters, the score setup and scoring
functions of the registry, analyzer proxies, ``result`` and ``merge``. The work
inside each split runs on the GPU through the score functions in
``pytme_b200.scores``; everything here is host-side bookkeeping on small arrays.
"""
from __future__ import annotations

import warnings
from itertools import product
from typing import Callable, Dict, Optional, Tuple

import numpy as np
import torch

__all__ = [
    "next_fast_len",
    "compute_convolution_shapes",
    "fourier_padding",
    "rigid_transform_matrices",
    "split_shape",
    "apply_convolution_mode",
    "MatchingData",
    "scan",
    "scan_subsets",
]


def next_fast_len(n: int) -> int:
    """Smallest length >= n of the form 2^a 3^b 5^c 7^d 11^e 13^f with e + f <= 1
    (pyFFTW's rule, used by compute_convolution_shapes in
    tme/backends/npfftw_backend.py:317-324)."""
    n = max(int(n), 1)
    while True:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m in (1, 11, 13):
            return n
        n += 1


def compute_convolution_shapes(arr1_shape, arr2_shape):
    """tme/backends/npfftw_backend.py:317-324."""
    conv = [int(x + y - 1) for x, y in zip(arr1_shape, arr2_shape)]
    fast = [next_fast_len(x) for x in conv]
    fast_ft = list(fast[:-1]) + [fast[-1] // 2 + 1]
    return conv, fast, fast_ft


def fourier_padding(target_shape, template_shape, pad_target: bool = False):
    """``MatchingData._fourier_padding`` (tme/matching_data.py:489-532) without batch
    dimensions: (convolution, fast, fast_ft, fourier_shift)."""
    target_shape = np.asarray(target_shape, dtype=int)
    template_shape = np.asarray(template_shape, dtype=int)
    pad_shape = np.maximum(target_shape, template_shape)
    conv, fast, fast_ft = compute_convolution_shapes(pad_shape, np.ones_like(pad_shape))
    template_mod = np.mod(template_shape, 2)
    shift = 1 - np.divide(template_shape, 2).astype(int)
    shift = np.subtract(shift, template_mod)
    diff = np.subtract(target_shape, template_shape)
    smask = diff < 0
    if np.sum(smask):
        warnings.warn("Template is larger than target and padding is turned off. Consider "
                      "swapping them or activate padding. Correcting the shift for now.")
        sshift = np.divide(diff, 2)
        offset = np.mod(diff, 2)
        sshift = np.multiply(np.add(sshift, offset), smask)
        shift = np.subtract(shift, sshift).astype(int)
    if pad_target:
        shift = np.subtract(shift, np.subtract(1, template_mod))
    return tuple(conv), tuple(fast), tuple(fast_ft), tuple(int(x) for x in shift)


def rigid_transform_matrices(rotations: np.ndarray, center) -> np.ndarray:
    """Homogeneous pull matrices ``T(c) . R^-1 . T(-c)`` for a stack of rotations, built
    with the float32 arithmetic of ``NumpyFFTWBackend._rigid_transform_matrix``
    (tme/backends/npfftw_backend.py:326-355): LAPACK float32 inverse, then float32
    BLAS products. Returns (n, 4, 4) float32, row-major."""
    rot = np.ascontiguousarray(rotations, dtype=np.float32).reshape(-1, 3, 3)
    n = rot.shape[0]
    inv = np.linalg.inv(rot)
    center = np.asarray(center, dtype=np.float32)
    cmat = np.identity(4, dtype=np.float32)
    cmat[:3, 3] = center
    rmat = np.zeros((n, 4, 4), dtype=np.float32)
    rmat[:, :3, :3] = inv
    rmat[:, 3, 3] = 1
    left = np.matmul(cmat, rmat)
    cneg = cmat.copy()
    cneg[:3, 3] = -cneg[:3, 3]
    out = np.matmul(left, cneg)
    out /= out[:, 3:4, 3:4]
    return np.ascontiguousarray(out, dtype=np.float32)


def split_shape(shape, splits: Dict, equal_shape: bool = True):
    """The split slices of tme/matching_utils.py:573-618. Axis ``a`` is cut into
    ``p = max(splits.get(a, 1), 1)`` parts of length ``ceil(n/p)`` (``equal_shape``; the
    last part is moved back to end at the edge, overlapping its neighbour) or
    ``floor(n/p)`` (the last part runs to the edge); the result lists every combination
    of the axes' parts with the last axis varying fastest."""
    per_axis = []
    for axis, n in enumerate(int(x) for x in shape):
        parts = max(int(splits.get(axis, 1)), 1)
        step = -(-n // parts) if equal_shape else n // parts
        starts = [i * step for i in range(parts - 1)]
        cuts = [slice(a, a + step) for a in starts]
        cuts.append(slice(n - step, n) if equal_shape else slice((parts - 1) * step, n))
        per_axis.append(tuple(cuts))
    return tuple(product(*per_axis))


def _center_slice(current_shape, new_shape):
    starts = [(c - n) // 2 for c, n in zip(current_shape, new_shape)]
    return tuple(slice(s, s + n) for s, n in zip(starts, new_shape))


def apply_convolution_mode(arr, convolution_mode: str, s1, s2, convolution_shape=None):
    """tme/matching_utils.py:469-524 (slicing only; works on NumPy and torch arrays)."""
    if convolution_shape is None:
        convolution_shape = [s1[i] + s2[i] - 1 for i in range(len(s1))]
    arr = arr[tuple(slice(0, x) for x in convolution_shape)]
    if convolution_mode not in ("full", "same", "valid"):
        raise ValueError("Supported convolution_mode are 'full', 'same' and 'valid'.")
    if convolution_mode == "full":
        return arr
    if convolution_mode == "same":
        return arr[_center_slice(arr.shape, s1)]
    valid = [s1[i] - s2[i] + 1 for i in range(arr.ndim)]
    return arr[_center_slice(arr.shape, valid)]


class MatchingData:
    """Target, template, masks, rotations and filters of one matching problem
    (tme/matching_data.py:23-852, unbatched). ``template`` and ``template_mask``
    return the arrays reversed along every axis, as the reference does, so the
    Fourier product needs no conjugation."""

    def __init__(self, target, template, template_mask=None, target_mask=None,
                 rotations=None, invert_target: bool = False, **kwargs):
        self._target = np.asarray(target)
        self._template = np.asarray(template)
        self._template_mask = None if template_mask is None else np.asarray(template_mask)
        self._target_mask = None if target_mask is None else np.asarray(target_mask)
        self._invert_target = bool(invert_target)
        self.template_filter = None
        self.target_filter = None
        self.rotations = rotations

    # ---- attributes with the reference's semantics
    @property
    def rotations(self):
        return self._rotations

    @rotations.setter
    def rotations(self, rotations):
        if rotations is None:
            rotations = np.eye(self._target.ndim)
        rotations = np.asarray(rotations)
        if rotations.ndim not in (2, 3):
            raise ValueError("Rotations have to be a rank 2 or 3 array.")
        if rotations.ndim == 2:
            rotations = rotations.reshape(1, *rotations.shape)
        self._rotations = rotations.astype(np.float32)

    @property
    def target(self):
        return self._target

    @target.setter
    def target(self, arr):
        self._target = np.asarray(arr)

    @property
    def template(self):
        return self._template[::-1, ::-1, ::-1]

    @template.setter
    def template(self, arr):
        self._template = np.asarray(arr)

    @property
    def template_mask(self):
        if self._template_mask is None:
            return None
        return self._template_mask[::-1, ::-1, ::-1]

    @template_mask.setter
    def template_mask(self, arr):
        self._template_mask = None if arr is None else np.asarray(arr)

    @property
    def target_mask(self):
        return self._target_mask

    @target_mask.setter
    def target_mask(self, arr):
        self._target_mask = None if arr is None else np.asarray(arr)

    def target_padding(self, pad_target: bool = False):
        """tme/matching_data.py:459-487."""
        if pad_target:
            return tuple(int(x) for x in np.subtract(self._template.shape, 1))
        return tuple(0 for _ in self._target.shape)

    @staticmethod
    def _subset_array(arr, arr_slice, padding, invert=False):
        """``subset_array`` (tme/matching_data.py:96-168): slice plus reflect padding
        that uses real neighbouring data where the array has it."""
        padding = np.maximum(np.asarray(padding), 0).astype(int)
        start = np.array([x.start for x in arr_slice], dtype=int)
        stop = np.array([x.stop for x in arr_slice], dtype=int)
        right = np.divide(padding, 2).astype(int)
        left = np.add(right, np.mod(padding, 2))
        data_left = np.minimum(start, left)
        data_right = np.minimum(np.subtract(arr.shape, stop), right).astype(int)
        a0 = np.subtract(start, data_left)
        a1 = np.add(stop, data_right)
        out = np.asarray(arr[tuple(slice(int(a), int(b)) for a, b in zip(a0, a1))])
        pads = tuple((int(l), int(r)) for l, r in zip(np.subtract(left, data_left),
                                                     np.subtract(right, data_right)))
        if any(l or r for l, r in pads):  # without padding the slice is used as it is
            out = np.pad(out, pads, mode="reflect")
        if invert:
            out = -out
        return out

    def subset_by_slice(self, target_slice=None, template_slice=None, target_pad=None):
        """tme/matching_data.py:170-268 (unbatched)."""
        if target_slice is None:
            target_slice = tuple(slice(0, s) for s in self._target.shape)
        if template_slice is None:
            template_slice = tuple(slice(0, s) for s in self._template.shape)
        if target_pad is None:
            target_pad = np.zeros(self._target.ndim, dtype=int)
        tgt = self._subset_array(self._target, target_slice, target_pad, self._invert_target)
        tmpl = self._subset_array(self._template, template_slice, np.zeros(3, int))
        tmask = None
        if self._template_mask is not None:
            tmask = self._subset_array(self._template_mask, template_slice, np.zeros(3, int))
        ret = MatchingData(tgt, tmpl, template_mask=tmask, rotations=self._rotations)
        ret.template_filter = self.template_filter
        ret.target_filter = self.target_filter
        offset = tuple(int(x.start) for x in target_slice)
        return ret, offset

    def fourier_padding(self, pad_target: bool = False):
        return fourier_padding(self._target.shape, self._template.shape, pad_target)

    def _split_rotations_on_jobs(self, n_jobs: int):
        """tme/matching_data.py:822-844."""
        per = self.rotations.shape[0] // n_jobs
        out = []
        for n in range(n_jobs):
            lo = n * per
            hi = None if n == n_jobs - 1 else lo + per
            out.append(self.rotations[lo:hi])
        return out


class TargetSpectrum:
    """The complex64 rfft of the target padded (top-left) to the fast shape, computed on
    the device the first time a filter asks for it: the ``data_rfft`` that the
    reference's filter set-up hands to every filter (tme/matching_exhaustive.py:84-90)."""

    def __init__(self, target, fast_shape):
        self._target, self._fast = target, tuple(int(x) for x in fast_shape)
        self._ft = None

    def get(self):
        if self._ft is None:
            from .backend import backend as be

            t = torch.as_tensor(np.asarray(self._target, dtype=np.float32)) \
                if not isinstance(self._target, torch.Tensor) else self._target
            self._ft = be.rfftn(t.to(torch.float32), s=self._fast)
        return self._ft


def _evaluate_filter(filt, shape, data_rfft=None, **kwargs):
    """A filter is either an array (already at the right rfft shape) or a callable
    with the reference's filter interface (``__call__(shape=..., return_real_fourier=
    True, data_rfft=..., ...)`` returning a dict with ``data``). ``data_rfft`` is the
    target's spectrum, or a ``TargetSpectrum`` that computes it when a filter needs it
    (whitening)."""
    if filt is None:
        return None
    if callable(filt):
        from .filters import device_filter, needs_spectrum

        spec = None
        if data_rfft is not None and needs_spectrum(filt):
            spec = data_rfft.get() if isinstance(data_rfft, TargetSpectrum) else data_rfft
        try:
            # CTFs, continuous wedges, whitening and their Compose are built on the GPU
            return device_filter(filt, shape, return_real_fourier=True, data_rfft=spec,
                                 **kwargs)
        except NotImplementedError:
            pass
        if isinstance(spec, torch.Tensor):
            from .analyzer import download

            spec = download(spec)
        ret = filt(shape=shape, return_real_fourier=True, shape_is_real_fourier=False,
                   data_rfft=spec, batch_dimension=None, **kwargs)
        return np.asarray(ret["data"], dtype=np.float32)
    if isinstance(filt, torch.Tensor):
        return filt.to(torch.float32)
    return np.asarray(filt, dtype=np.float32)


def scan(matching_data: MatchingData, matching_setup: Callable, matching_score: Callable,
         n_jobs: int = 1, callback_class=None, callback_class_args: Optional[Dict] = None,
         pad_target: bool = True, pad_template_filter: bool = False,
         interpolation_order: int = 3, jobs_per_callback_class: int = 8, target_slice=None,
         template_slice=None, process_group=None, **kwargs):
    """One split of the search (tme/matching_exhaustive.py:144-295). Rotations are
    scored in one process on the current GPU; ``n_jobs`` only shapes the rotation
    chunks handed to the scoring function, as in the reference. With ``process_group``
    (a torch.distributed group of more than one rank, one process per GPU), each rank
    scores its contiguous share of the rotations and one MAX all-reduce merges the
    (score, rotation) states (``distributed.score_rotation_shares``); every rank then
    holds the analyzer state of the whole scan."""
    from . import scores as _scores  # noqa: F401  (registers the default scores)
    from .analyzer import SharedAnalyzerProxy

    callback_class_args = dict(callback_class_args or {})
    md, offset = matching_data.subset_by_slice(
        target_slice=target_slice, template_slice=template_slice,
        target_pad=matching_data.target_padding(pad_target=pad_target))
    conv, fwd, inv, shift = md.fourier_padding(pad_target=pad_target)

    spectrum = TargetSpectrum(md._target, fwd)
    template_filter = _evaluate_filter(md.template_filter, md._template.shape, data_rfft=spectrum)
    target_filter = _evaluate_filter(md.target_filter, fwd, data_rfft=spectrum, weight_type=None)
    del spectrum
    if template_filter is not None and pad_template_filter:
        raise NotImplementedError("pad_template_filter=True is not supported; the "
                                  "template filter is applied at template shape")

    default_args = {
        "shape": fwd, "offset": offset, "fourier_shift": shift, "fast_shape": fwd,
        "targetshape": md._target.shape, "templateshape": md._template.shape,
        "convolution_shape": conv, "thread_safe": False,
        "convolution_mode": "valid" if pad_target else "same",
        "only_unique_rotations": True, "aggregate_axis": None,
        "n_rotations": md.rotations.shape[0],
    }
    callback_class_args["inversion_mapping"] = n_jobs == 1
    default_args.update(callback_class_args)

    setup = matching_setup(matching_data=md, template_filter=template_filter,
                           target_filter=target_filter, fast_shape=fwd, fast_ft_shape=inv,
                           shm_handler=None)
    setup["interpolation_order"] = interpolation_order
    setup["template_filter"] = template_filter

    callback = SharedAnalyzerProxy(callback_class, default_args) if callback_class else None
    sharded = False
    if process_group is not None:
        import torch.distributed as dist

        sharded = dist.is_initialized() and dist.get_world_size(
            None if process_group == "default" else process_group) > 1
    if sharded:
        from .distributed import score_rotation_shares

        score_rotation_shares(matching_score, setup, md.rotations, callback,
                              group=None if process_group == "default" else process_group)
    else:
        for rotation in md._split_rotations_on_jobs(max(int(n_jobs), 1)):
            matching_score(rotations=rotation, callback=callback, **setup)
    if "plan" in setup:
        setup["plan"].close()
    if callback_class is None:
        return None
    result = callback.result(**default_args)
    return callback_class.merge([result], **default_args)


def scan_subsets(matching_data: MatchingData, matching_score: Callable,
                 matching_setup: Callable, callback_class=None,
                 callback_class_args: Optional[Dict] = None, job_schedule=(1, 1),
                 target_splits: Optional[Dict] = None, template_splits: Optional[Dict] = None,
                 pad_target_edges: bool = False, pad_template_filter: bool = False,
                 interpolation_order: int = 3, jobs_per_callback_class: int = 8,
                 backend_name: str = None, backend_args: Optional[Dict] = None,
                 verbose: bool = False, process_group=None, **kwargs):
    """tme/matching_exhaustive.py:298-465. Splits run one after another on the
    current device; their analyzer results are merged with ``callback_class.merge``.
    ``process_group`` ("default" or a torch.distributed group; one process per GPU)
    shards every split's rotations over the group's ranks (see ``scan``)."""
    callback_class_args = dict(callback_class_args or {})
    template_splits = split_shape(matching_data._template.shape, splits=template_splits or {})
    target_splits = split_shape(matching_data._target.shape, splits=target_splits or {})
    if len(target_splits) > 1 and not pad_target_edges:
        warnings.warn("Target splitting without padding target edges leads to unreliable "
                      "similarity estimates around the split border.")
    outer, inner = job_schedule
    results = []
    for target_split, template_split in product(target_splits, template_splits):
        results.append(scan(
            matching_data=matching_data, matching_score=matching_score,
            matching_setup=matching_setup, n_jobs=inner, callback_class=callback_class,
            callback_class_args=callback_class_args, interpolation_order=interpolation_order,
            pad_target=pad_target_edges, pad_template_filter=pad_template_filter,
            target_slice=target_split, template_slice=template_split,
            process_group=process_group))
    if callback_class is not None:
        return callback_class.merge(results, **callback_class_args)
    return None
