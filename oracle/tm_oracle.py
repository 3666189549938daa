"""CPU oracle for the exhaustive template-matching hot path.

TEST INFRASTRUCTURE ONLY. This module restates, in NumPy/SciPy, the reference's
per-rotation scan loop so the CUDA path can be checked against it. Only the test
suite, ``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py``
import it, and only as the checker or the timed CPU baseline; the product path
in ``pytme_b200`` never calls it.

Each function follows the reference (KosinskiLab/pyTME 0.3.b0) step by step,
with the same dtypes and operation order, and cites the file:line it restates.
The third-party arithmetic the reference calls is called here too:
``scipy.ndimage.affine_transform`` (order 1, ``mode="constant"``) for rotations,
``scipy.ndimage.maximum_filter`` for peak calling and ``scipy.fft`` for FFTs
(the reference calls pyFFTW; FFTW is not installed here, so FFT rounding is
pocketfft's). The oracle is pinned against golden vectors produced by running
the reference package itself (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math
from typing import Dict, Optional, Tuple

import numpy as np
import scipy.fft as sfft
from scipy.ndimage import affine_transform, maximum_filter

__all__ = [
    "next_fast_len",
    "fourier_padding",
    "rigid_transform_matrix",
    "rotate_order1",
    "rotate",
    "normalize_template",
    "norm_scores",
    "apply_template_filter",
    "apply_target_filter",
    "scan",
    "scan_parallel",
    "raw_index",
    "result_map",
    "max_filter_coordinates",
    "find_candidate_indices",
    "topk_indices",
    "peak_caller_maximum_filter",
    "euler_zyz_to_matrix",
    "score_box_corner",
    "refine_flc_score",
]


# --------------------------------------------------------------------------- shapes
def next_fast_len(n: int) -> int:
    """pyFFTW's fast length: 2^a 3^b 5^c 7^d 11^e 13^f, e + f <= 1
    (called by tme/backends/npfftw_backend.py:317-324)."""
    n = max(int(n), 1)
    while True:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m in (1, 11, 13):
            return n
        n += 1


def fourier_padding(target_shape, template_shape, pad_target: bool = False):
    """Restates ``MatchingData._fourier_padding`` (tme/matching_data.py:489-532) and
    ``compute_convolution_shapes`` (tme/backends/npfftw_backend.py:317-324) for
    unbatched 3D data. Returns (convolution, fast, fast_ft, fourier_shift)."""
    target_shape = np.asarray(target_shape, dtype=int)
    template_shape = np.asarray(template_shape, dtype=int)
    pad_shape = np.maximum(target_shape, template_shape)
    conv = [int(x + 1 - 1) for x in pad_shape]
    fast = [next_fast_len(x) for x in conv]
    fast_ft = list(fast[:-1]) + [fast[-1] // 2 + 1]

    template_mod = np.mod(template_shape, 2)
    shift = 1 - np.divide(template_shape, 2).astype(int)
    shift = np.subtract(shift, template_mod)
    diff = np.subtract(target_shape, template_shape)
    smask = diff < 0
    if np.sum(smask):
        sshift = np.divide(diff, 2)
        offset = np.mod(diff, 2)
        sshift = np.multiply(np.add(sshift, offset), smask)
        shift = np.subtract(shift, sshift).astype(int)
    if pad_target:
        shift = np.subtract(shift, np.subtract(1, template_mod))
    return tuple(conv), tuple(fast), tuple(fast_ft), tuple(int(x) for x in shift)


# --------------------------------------------------------------------------- rotation
def rigid_transform_matrix(rotation: np.ndarray, center, dtype=np.float32) -> np.ndarray:
    """Homogeneous pull matrix ``T(c) . R^-1 . T(-c)`` built like
    ``NumpyFFTWBackend._rigid_transform_matrix`` (tme/backends/npfftw_backend.py:326-355):
    float dtype of the backend, LAPACK inverse and BLAS dot per rotation."""
    ndim = rotation.shape[0]
    matrix = np.identity(ndim + 1, dtype=dtype)
    translation_matrix = np.identity(ndim + 1, dtype=dtype)
    translation_matrix[:ndim, ndim] = -np.zeros(ndim)
    np.dot(matrix, translation_matrix, out=matrix)
    center_matrix = np.identity(ndim + 1, dtype=dtype)
    center_matrix[:ndim, ndim] = center
    np.dot(matrix, center_matrix, out=matrix)
    rmat = np.identity(ndim + 1, dtype=dtype)
    rmat[:ndim, :ndim] = np.linalg.inv(rotation.astype(dtype))
    np.dot(matrix, rmat, out=matrix)
    center_matrix[:ndim, ndim] = -center_matrix[:ndim, ndim]
    np.dot(matrix, center_matrix, out=matrix)
    matrix /= matrix[ndim, ndim]
    return matrix


def rotate_order1(data: np.ndarray, matrix: np.ndarray, output: np.ndarray) -> np.ndarray:
    """``_rigid_transform`` (tme/backends/npfftw_backend.py:357-388): order-1
    ``affine_transform`` in constant mode into the top-left ``data.shape`` box of
    ``output``."""
    return rotate(data, matrix, output, order=1, prefilter=True)


def rotate(data: np.ndarray, matrix: np.ndarray, output: np.ndarray, order: int = 1,
           prefilter: bool = True) -> np.ndarray:
    """``_rigid_transform`` (tme/backends/npfftw_backend.py:357-388) at any spline order:
    ``rigid_transform`` (:390-449) prefilters the data and not the mask."""
    out_slice = tuple(slice(0, s) for s in data.shape)
    affine_transform(input=data, matrix=matrix, mode="constant", output=output[out_slice],
                     order=order, prefilter=prefilter)
    return output


# --------------------------------------------------------------------------- scores
def normalize_template(template, mask, n_obs):
    """tme/matching_utils.py:61-99 (in place, backend dtype)."""
    masked_mean = np.sum(np.multiply(template, mask), axis=None, keepdims=True)
    masked_mean = np.divide(masked_mean, n_obs)
    masked_std = np.sum(np.multiply(np.square(template), mask), axis=None, keepdims=True)
    masked_std = np.subtract(masked_std / n_obs, np.square(masked_mean))
    masked_std = np.sqrt(np.maximum(masked_std, 0))
    np.subtract(template, masked_mean, out=template)
    np.divide(template, masked_std, out=template)
    return np.multiply(template, mask, out=template)


def norm_scores(arr, exp_sq, sq_exp, n_obs, eps, out):
    """``NumpyFFTWBackend.norm_scores`` (tme/backends/npfftw_backend.py:537-587)."""
    sq_exp = np.divide(sq_exp, n_obs, out=sq_exp)
    sq_exp = np.square(sq_exp, out=sq_exp)
    exp_sq = np.divide(exp_sq, n_obs, out=exp_sq)
    sq_exp = np.subtract(exp_sq, sq_exp, out=sq_exp)
    sq_exp = np.maximum(sq_exp, 0.0, out=sq_exp)
    sq_exp = np.sqrt(sq_exp, out=sq_exp)
    sq_exp[sq_exp < eps] = 1
    sq_exp = np.multiply(sq_exp, n_obs, out=sq_exp)
    return np.divide(arr, sq_exp, out=out)


def apply_template_filter(template_t: np.ndarray, template_filter: Optional[np.ndarray]):
    """``_apply_filter_subset`` of ``_create_filter_func`` for a filter at template
    rfft shape (tme/matching_scores.py:90-135): rfftn -> multiply -> irfftn of the
    template-sized box, written back in place."""
    if template_filter is None or template_filter.size == 1:
        return template_t
    ft = sfft.rfftn(template_t)
    ft = np.multiply(ft, template_filter, out=ft)
    template_t[...] = sfft.irfftn(ft, s=template_t.shape)
    return template_t


def apply_target_filter(target: np.ndarray, fast_shape, target_filter: Optional[np.ndarray]):
    """Target part of ``_setup_template_filter_apply_target_filter``
    (tme/matching_exhaustive.py:84-117): the filter is multiplied into the rfft of the
    top-left padded target once, and the cropped inverse replaces the target."""
    if target_filter is None:
        return target
    pad = np.zeros(fast_shape, dtype=target.dtype)
    pad[tuple(slice(0, s) for s in target.shape)] = target
    ft = sfft.rfftn(pad)
    ft = np.multiply(ft, target_filter.reshape(ft.shape), out=ft)
    full = sfft.irfftn(ft, s=pad.shape)
    return np.ascontiguousarray(full[tuple(slice(0, s) for s in target.shape)])


def _topleft_pad(arr, shape, dtype):
    b = np.zeros(shape, dtype=dtype)
    b[tuple(slice(0, min(a, s)) for a, s in zip(arr.shape, shape))] = arr[
        tuple(slice(0, min(a, s)) for a, s in zip(arr.shape, shape))]
    return b


def _max_update(scores, max_scores, rotations, index):
    """``max_score_over_rotations`` (tme/backends/npfftw_backend.py:503-535): strict >."""
    idx = scores > max_scores
    max_scores[idx] = scores[idx]
    rotations[idx] = index


def _setup(score, target, template_rev, mask_rev, fast, dtype, cdtype):
    """``cc_setup`` / ``flc_setup`` / ``flcSphericalMask_setup``
    (tme/matching_scores.py:153-189, 357-387, 390-450)."""
    eps = np.finfo(dtype).eps
    target_pad = _topleft_pad(target, fast, dtype)
    if score == "CC":
        return {"ft_target": sfft.rfftn(target_pad)}
    if score == "FLC":
        ft_target = sfft.rfftn(target_pad)
        ft_target2 = sfft.rfftn(np.square(target_pad))
        return {"ft_target": ft_target, "ft_target2": ft_target2}
    if score == "FLCSphericalMask":
        n_obs = np.sum(mask_rev.astype(dtype), axis=None, keepdims=True)
        mask_pad = _topleft_pad(mask_rev, fast, dtype)
        ft_mask = sfft.rfftn(mask_pad, s=fast)
        ft_target = sfft.rfftn(np.square(target_pad))
        ft_temp = np.multiply(ft_target, ft_mask)
        temp2 = sfft.irfftn(ft_temp, s=fast)
        ft_target = sfft.rfftn(target_pad)
        ft_temp = np.multiply(ft_target, ft_mask)
        temp = sfft.irfftn(ft_temp, s=fast)
        inv_den = norm_scores(1, temp2, temp, n_obs, eps, temp2)
        return {"ft_target": ft_target, "inv_denominator": inv_den}
    raise ValueError(f"unknown score {score}")


def _loop(score, setup, template_rev, mask_rev, rotations, fast, dtype, cdtype,
          template_filter, first_index, max_scores, argmax, order=1, on_scores=None):
    """Per-rotation loops ``corr_scoring`` (tme/matching_scores.py:600-624) and
    ``flc_scoring`` (tme/matching_scores.py:727-757) with ``MaxScoreOverRotations``
    state updates (tme/analyzer/aggregation.py:142-189). ``on_scores(i, scores)``, when
    given, sees every rotation's full score map before the update (the callback
    position of the reference loops)."""
    eps = np.finfo(dtype).eps
    tshape = template_rev.shape
    center = np.divide(np.asarray(tshape) - 1, 2)
    unpadded = tuple(slice(0, s) for s in tshape)
    arr = np.zeros(fast, dtype=dtype)
    if score == "FLC":
        temp = np.zeros(fast, dtype=dtype)
        for i in range(rotations.shape[0]):
            matrix = rigid_transform_matrix(rotations[i], center, dtype)
            arr.fill(0)
            temp.fill(0)
            rotate(template_rev, matrix, arr, order, prefilter=True)
            rotate(mask_rev, matrix, temp, order, prefilter=False)
            n_obs = np.sum(temp)
            apply_template_filter(arr[unpadded], template_filter)
            normalize_template(arr, temp, n_obs)
            ft_temp = sfft.rfftn(temp)
            cc_m = sfft.irfftn(setup["ft_target"] * ft_temp, s=fast)
            cc_m2 = sfft.irfftn(setup["ft_target2"] * ft_temp, s=fast)
            ft_temp = sfft.rfftn(arr)
            cc = sfft.irfftn(setup["ft_target"] * ft_temp, s=fast).astype(dtype, copy=False)
            cc = norm_scores(cc, cc_m2.astype(dtype, copy=False), cc_m.astype(dtype, copy=False),
                             n_obs, eps, cc)
            if on_scores is not None:
                on_scores(i, cc)
            _max_update(cc, max_scores, argmax, first_index + i)
        return
    template_rot = np.zeros(tshape, dtype=dtype)
    mask_sum = None
    if score == "FLCSphericalMask":
        mask_sum = np.sum(mask_rev)
    for i in range(rotations.shape[0]):
        matrix = rigid_transform_matrix(rotations[i], center, dtype)
        rotate(template_rev, matrix, template_rot, order, prefilter=True)
        apply_template_filter(template_rot, template_filter)
        if mask_sum is not None:
            normalize_template(template_rot, mask_rev, mask_sum)
        arr.fill(0)
        arr[unpadded] = template_rot
        ft_temp = sfft.rfftn(arr)
        ft_temp = np.multiply(setup["ft_target"], ft_temp, out=ft_temp)
        arr = sfft.irfftn(ft_temp, s=fast).astype(dtype, copy=False)
        if "inv_denominator" in setup:
            arr = np.multiply(arr, setup["inv_denominator"], out=arr)
        if on_scores is not None:
            on_scores(i, arr)
        _max_update(arr, max_scores, argmax, first_index + i)
        arr = np.ascontiguousarray(arr)


def _prepare(target, template, template_mask, pad_target_edges, target_filter, dtype):
    """Target padding (``subset_array`` reflect padding, tme/matching_data.py:96-168,
    with ``target_padding`` :459-487), template/mask reversal (``template`` property,
    :698-715) and the target filter."""
    target = np.asarray(target, dtype=dtype)
    template = np.asarray(template, dtype=dtype)
    if pad_target_edges:
        padding = np.subtract(template.shape, 1)
        right = np.divide(padding, 2).astype(int)
        left = np.add(right, np.mod(padding, 2))
        target = np.pad(target, tuple(zip(left, right)), mode="reflect")
    template_rev = np.ascontiguousarray(template[::-1, ::-1, ::-1])
    mask_rev = None
    if template_mask is not None:
        mask_rev = np.ascontiguousarray(np.asarray(template_mask, dtype=dtype)[::-1, ::-1, ::-1])
    return target, template_rev, mask_rev


def scan(target: np.ndarray, template: np.ndarray, rotations: np.ndarray,
         score: str = "FLCSphericalMask", template_mask: Optional[np.ndarray] = None,
         template_filter: Optional[np.ndarray] = None,
         target_filter: Optional[np.ndarray] = None, pad_target_edges: bool = False,
         dtype=np.float32, score_threshold: float = 0.0, interpolation_order: int = 1) -> Dict:
    """One split of ``scan`` (tme/matching_exhaustive.py:144-295) with
    ``MaxScoreOverRotations`` and ``job_schedule=(1, 1)``; returns the raw state and the
    post-processed ``result`` maps (tme/analyzer/aggregation.py:207-277)."""
    cdtype = np.complex128 if dtype == np.float64 else np.complex64
    rotations = np.asarray(rotations, dtype=np.float32)
    tgt, t_rev, m_rev = _prepare(target, template, template_mask, pad_target_edges,
                                 target_filter, dtype)
    conv, fast, fast_ft, shift = fourier_padding(tgt.shape, t_rev.shape, pad_target_edges)
    if target_filter is not None:
        tgt = apply_target_filter(tgt, fast, target_filter).astype(dtype)
    if score in ("FLC", "FLCSphericalMask") and m_rev is None:
        raise ValueError(f"{score} needs a template mask")
    setup = _setup(score, tgt, t_rev, m_rev, fast, dtype, cdtype)
    max_scores = np.full(fast, score_threshold, dtype=dtype)
    argmax = np.full(fast, -1, dtype=np.int32)
    tf = None if template_filter is None else np.asarray(template_filter, dtype=dtype)
    _loop(score, setup, t_rev, m_rev, rotations, fast, dtype, cdtype, tf, 0, max_scores,
          argmax, order=interpolation_order)
    scores, rot = result_map(max_scores, argmax, shift, conv, tgt.shape, t_rev.shape,
                             "valid" if pad_target_edges else "same")
    return {"scores": scores, "rotations": rot, "fast_shape": fast, "fourier_shift": shift,
            "raw_scores": max_scores, "raw_rotations": argmax}


def _scan_chunk(args):
    (score, tgt, t_rev, m_rev, rotations, fast, dtype, tf, first, thr, order, probe) = args
    cdtype = np.complex128 if dtype == np.float64 else np.complex64
    setup = _setup(score, tgt, t_rev, m_rev, fast, dtype, cdtype)
    ms = np.full(fast, thr, dtype=dtype)
    am = np.full(fast, -1, dtype=np.int32)
    vals = None
    hook = None
    if probe is not None:
        vals = np.zeros((rotations.shape[0], probe.size), dtype=np.float64)

        def hook(i, arr):
            vals[i] = np.asarray(arr).reshape(-1)[probe]
    _loop(score, setup, t_rev, m_rev, rotations, fast, dtype, cdtype, tf, first, ms, am,
          order=order, on_scores=hook)
    return ms, am, vals


def raw_index(result_coords, fast, shift, conv, target_shape, template_shape, mode="same"):
    """Flat indices into the raw (fast-shaped) state of the voxels at ``result_coords``
    ((m, 3) coordinates of the map ``result_map`` returns): ``result_map`` applied to the
    index volume."""
    idx = np.arange(int(np.prod(fast)), dtype=np.int64).reshape(fast)
    ridx, _ = result_map(idx, idx, shift, conv, target_shape, template_shape, mode)
    c = np.asarray(result_coords, dtype=np.int64).reshape(-1, len(fast))
    return np.ascontiguousarray(ridx[tuple(c.T)])


def scan_parallel(target, template, rotations, score="FLCSphericalMask", template_mask=None,
                  template_filter=None, target_filter=None, dtype=np.float32,
                  n_workers: int = 1, score_threshold: float = 0.0,
                  interpolation_order: int = 1, probe=None):
    """``scan`` with the rotation set split into contiguous chunks over ``n_workers``
    spawned processes (the reference's inner joblib parallelism,
    tme/matching_exhaustive.py:276-285 and ``_split_rotations_on_jobs``
    tme/matching_data.py:822-844); chunk states are merged in rotation order, which
    keeps the first rotation on ties. ``probe`` ((m, 3) coordinates in the returned
    ``same``-mode map) adds ``"probe"``: every rotation's score at those voxels,
    (rotations, m) float64."""
    import multiprocessing as mp

    rotations = np.asarray(rotations, dtype=np.float32)
    tgt, t_rev, m_rev = _prepare(target, template, template_mask, False, None, dtype)
    conv, fast, fast_ft, shift = fourier_padding(tgt.shape, t_rev.shape, False)
    if target_filter is not None:
        tgt = apply_target_filter(tgt, fast, target_filter).astype(dtype)
    tf = None if template_filter is None else np.asarray(template_filter, dtype=dtype)
    pidx = None
    if probe is not None:
        pidx = raw_index(probe, fast, shift, conv, tgt.shape, t_rev.shape)
    n = rotations.shape[0]
    n_workers = max(1, min(int(n_workers), n))
    per = n // n_workers
    chunks = []
    for j in range(n_workers):
        lo = j * per
        hi = n if j == n_workers - 1 else lo + per
        chunks.append((score, tgt, t_rev, m_rev, rotations[lo:hi], fast, dtype, tf, lo,
                       score_threshold, interpolation_order, pidx))
    if n_workers == 1:
        outs = [_scan_chunk(chunks[0])]
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(n_workers) as pool:
            outs = pool.map(_scan_chunk, chunks)
    ms, am, _ = outs[0]
    for ms2, am2, _ in outs[1:]:
        upd = ms2 > ms
        ms[upd] = ms2[upd]
        am[upd] = am2[upd]
    scores, rot = result_map(ms, am, shift, conv, tgt.shape, t_rev.shape, "same")
    out = {"scores": scores, "rotations": rot}
    if probe is not None:
        out["probe"] = np.concatenate([o[2] for o in outs], axis=0)
    return out


def _center_slice(current_shape, new_shape):
    starts = [(c - n) // 2 for c, n in zip(current_shape, new_shape)]
    return tuple(slice(s, s + n) for s, n in zip(starts, new_shape))


def result_map(max_scores, argmax, shift, conv, target_shape, template_shape, mode):
    """``MaxScoreOverRotations.result`` (tme/analyzer/aggregation.py:207-277): roll by
    the Fourier shift, then ``apply_convolution_mode`` (tme/matching_utils.py:469-524)."""
    axis = tuple(range(len(shift)))
    s = np.roll(max_scores, shift=shift, axis=axis)
    r = np.roll(argmax, shift=shift, axis=axis)
    s = s[tuple(slice(0, x) for x in conv)]
    r = r[tuple(slice(0, x) for x in conv)]
    if mode == "same":
        box = _center_slice(s.shape, target_shape)
    elif mode == "valid":
        box = _center_slice(s.shape, [a - b + 1 for a, b in zip(target_shape, template_shape)])
    else:
        box = tuple(slice(None) for _ in s.shape)
    return s[box], r[box]


# --------------------------------------------------------------------------- peaks
def max_filter_coordinates(scores: np.ndarray, min_distance: int) -> np.ndarray:
    """``NumpyFFTWBackend.max_filter_coordinates`` (tme/backends/npfftw_backend.py:200-206)."""
    box = tuple(min_distance for _ in range(scores.ndim))
    mf = maximum_filter(scores, size=box, mode="constant")
    return np.array(np.nonzero(mf == scores)).T


def find_candidate_indices(coordinates: np.ndarray, min_distance) -> np.ndarray:
    """Greedy min-distance filter of ``find_candidate_indices``
    (tme/external/bindings.cpp:85-126): point 0 is kept; each later point is kept when
    its distance to every kept point is ``> min_distance``. The reference computes the
    distance in the coordinates' type; for integer coordinates (the int64 overload the
    peak callers reach, bindings.cpp:251-256) the squared distance and its square root
    are truncated to integers, so a point is rejected iff
    ``floor(sqrt(d2)) <= min_distance``. Each point is tested against the kept list at
    once (integer squared distances; the floor of the float64 square root equals the
    integer square root for the squared distances of coordinates below 2**24)."""
    coords = np.asarray(coordinates)
    n = coords.shape[0]
    if n == 0:
        return np.zeros(0, dtype=np.int64)
    integer = np.issubdtype(coords.dtype, np.integer)
    c = coords.astype(np.int64 if integer else np.float64)
    if integer and np.abs(c).max(initial=0) >= 2 ** 24:
        raise ValueError("integer coordinates beyond 2**24 are outside the oracle's range")
    kept_c = np.empty_like(c)
    kept = [0]
    kept_c[0] = c[0]
    k = 1
    for i in range(1, n):
        d = kept_c[:k] - c[i]
        d2 = np.einsum("ij,ij->i", d, d)
        dist = np.floor(np.sqrt(d2.astype(np.float64))) if integer else np.sqrt(d2)
        if not np.any(dist <= min_distance):
            kept.append(i)
            kept_c[k] = c[i]
            k += 1
    return np.asarray(kept, dtype=np.int64)


def topk_indices(arr: np.ndarray, k: int):
    """``NumpyFFTWBackend.topk_indices`` (tme/backends/npfftw_backend.py:177-182)."""
    temp = arr.reshape(-1)
    indices = np.argpartition(temp, -k)[-k:][:k]
    sorted_indices = indices[np.argsort(temp[indices])][::-1]
    return np.unravel_index(sorted_indices, arr.shape)


def peak_caller_maximum_filter(scores: np.ndarray, num_peaks: int = 1000,
                               min_distance: int = 1, min_boundary_distance: int = 0,
                               min_score=None, max_score=None):
    """``PeakCallerMaximumFilter`` applied once to a score map with an identity rotation
    (tme/analyzer/peaks.py:327-384 ``__call__``, :241-290 ``_get_peak_mask``,
    :531-583 ``_update``, :68-106 ``filter_points_indices``). Returns positions and
    scores of the state (including unfilled ``-1`` rows, as the reference state does)."""
    ndim = scores.ndim
    translations = np.full((num_peaks, ndim), -1, dtype=np.int32)
    state_scores = np.full((num_peaks,), -1, dtype=np.float32)
    peaks = max_filter_coordinates(scores, min_distance)
    if len(peaks) == 0:
        return translations, state_scores
    upper = np.subtract(np.asarray(scores.shape), min_boundary_distance)
    valid = np.multiply(peaks < upper, peaks >= min_boundary_distance)
    valid = np.sum(valid, axis=1) == peaks.shape[1]
    pscores = scores[tuple(peaks.T)]
    valid = np.multiply(pscores == pscores, valid)
    if min_score is not None:
        valid = np.multiply(pscores >= min_score, valid)
    if max_score is not None:
        valid = np.multiply(pscores <= max_score, valid)
    if np.sum(valid) == 0:
        return translations, state_scores
    if np.sum(valid) > num_peaks or pscores.shape[0] > num_peaks:
        top = min(pscores.size, 2 * num_peaks)
        idx, *_ = topk_indices(pscores * valid, top)
        valid = np.full(pscores.shape, 0, bool)
        valid[idx] = True
        if min_score is not None:
            valid = np.multiply(pscores >= min_score, valid)
        if max_score is not None:
            valid = np.multiply(pscores <= max_score, valid)
    peaks = peaks[valid].astype(np.int32)
    pscores = scores[tuple(peaks.T)]
    positions = np.concatenate((translations, peaks))
    all_scores = np.concatenate((state_scores, pscores.astype(np.float32)))
    if min_distance <= 0:
        order = np.arange(positions.shape[0])
    else:
        sorted_idx = np.argsort(-all_scores)
        kept = find_candidate_indices(positions[sorted_idx], min_distance)
        order = sorted_idx[kept]
    s = all_scores[order]
    top_n = min(s.size, num_peaks)
    top, *_ = topk_indices(s, top_n)
    final = order[top]
    return positions[final], all_scores[final]


# --------------------------------------------------------------------------- refinement
def euler_zyz_to_matrix(angles) -> np.ndarray:
    """``euler_to_rotationmatrix`` (tme/rotations.py:171-196): SciPy's extrinsic "zyz"
    sequence in degrees, R = Rz(angles[2]) . Ry(angles[1]) . Rz(angles[0]); float64
    here (the reference casts to float32)."""
    from scipy.spatial.transform import Rotation

    return Rotation.from_euler("zyz", np.asarray(angles, dtype=np.float64),
                               degrees=True).as_matrix()


def score_box_corner(position, target_shape, template_shape) -> np.ndarray:
    """Target voxel of template voxel 0 for the score-map voxel ``position`` of a
    "same"-mode ``MaxScoreOverRotations.result`` (target at least as large as the
    template on every axis): the scan correlates with the reversed template, so the
    box starts t - 1 before the raw correlation index, and ``result`` rolls by
    ``1 - t//2 - t%2`` (tme/matching_data.py:510-512) and crops from
    (min(conv, fast) - T) // 2 (tme/matching_utils.py:469-524)."""
    conv, fast, _, _ = fourier_padding(target_shape, template_shape)
    start = [(min(c, f) - n) // 2 for c, f, n in zip(conv, fast, target_shape)]
    return (np.asarray(position, dtype=np.int64) + np.asarray(start)
            - np.asarray(template_shape) // 2)


def refine_flc_score(target, template, mask, corner, rotation, shift=(0.0, 0.0, 0.0),
                     template_filter=None, dtype=np.float64) -> float:
    """The FLC score of ``flc_scoring`` (tme/matching_scores.py:629-759) at one pose,
    written in real space. The template and mask are rotated by ``rotation`` about the
    template centre (t - 1)/2 with order-1 constant-mode interpolation
    (``_rigid_transform``, tme/backends/npfftw_backend.py:357-388) and moved by the
    sub-voxel ``shift`` in the target frame, so template voxel o samples
    R^T (o - c - shift) + c. The template filter is applied at template shape
    (``_apply_filter_subset``, tme/matching_scores.py:131-135), the filtered template is
    normalised under the rotated mask (tme/matching_utils.py:61-99), correlated with the
    target box starting at ``corner`` (zero outside the target) and divided by the
    masked local standard deviation times n_obs (``norm_scores``,
    tme/backends/npfftw_backend.py:537-587, eps = float32 eps). At shift 0 this is the
    exhaustive FLC map value at the score-map voxel whose ``score_box_corner`` is
    ``corner``, because correlating with the reversed, rotated template equals
    correlating the rotated template in real space."""
    template = np.asarray(template, dtype=dtype)
    mask = np.asarray(mask, dtype=dtype)
    t = np.asarray(template.shape)
    c = (t - 1) / 2.0
    rt = np.asarray(rotation, dtype=np.float64).T
    offset = c - rt @ (c + np.asarray(shift, dtype=np.float64))
    tr = affine_transform(template, rt, offset=offset, order=1, mode="constant",
                          prefilter=False)
    mr = affine_transform(mask, rt, offset=offset, order=1, mode="constant", prefilter=False)
    if template_filter is not None:
        tr = apply_template_filter(tr, np.asarray(template_filter, dtype=dtype))
    box = np.zeros(template.shape, dtype=dtype)
    corner = np.asarray(corner, dtype=np.int64)
    src = tuple(slice(max(k, 0), min(k + n, m)) for k, n, m in zip(corner, t, target.shape))
    dst = tuple(slice(s.start - k, s.stop - k) for s, k in zip(src, corner))
    if all(s.stop > s.start for s in src):
        box[dst] = np.asarray(target, dtype=dtype)[src]
    n_obs = np.sum(mr)
    tn = normalize_template(tr, mr, n_obs)
    numerator = np.sum(tn * box)
    exp_sq = np.sum(box * box * mr)
    sq_exp = np.sum(box * mr)
    eps = np.finfo(np.float32).eps
    out = norm_scores(np.asarray([numerator]), np.asarray([exp_sq]), np.asarray([sq_exp]),
                      n_obs, eps, np.zeros(1, dtype=dtype))
    return float(out[0])
