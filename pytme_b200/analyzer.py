"""Analyzers with the reference's callback API (tme/analyzer).

``MaxScoreOverRotations`` keeps its (scores, rotations, mapping) state on the
device; the fused scan updates it directly, any other caller goes through
``__call__`` and ``tm_max_score_over_rotations``. ``result`` and ``merge`` follow
tme/analyzer/aggregation.py:207-432. ``PeakCaller`` and its subclasses follow
tme/analyzer/peaks.py:146-941 with the maximum filter, top-k and greedy
distance filter running on the GPU (``pytme_b200.peaks``).
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np
import torch

from .backend import backend as be
from .matching import apply_convolution_mode

_NUMPY_DTYPES = {torch.float32: np.float32, torch.int32: np.int32, torch.float64: np.float64,
                 torch.int64: np.int64}
_CHUNK = 16 << 20
_staging: Dict[str, torch.Tensor] = {}


def download(t: torch.Tensor) -> np.ndarray:
    """A device tensor as a new host array.

    Large tensors go through two pinned 16 MiB chunks, kept for the life of the process:
    the copy engine fills one while the host copies the other into the result. A plain
    ``.cpu()`` stages through pageable memory and moved the 420 MB state of a
    512x512x200 scan at about 2 GB/s."""
    t = t.contiguous()
    nbytes = t.numel() * t.element_size()
    if not t.is_cuda or nbytes < 2 * _CHUNK or t.dtype not in _NUMPY_DTYPES:
        return t.cpu().numpy()
    stage = _staging.get("pinned")
    if stage is None:
        stage = torch.empty(2 * _CHUNK, dtype=torch.uint8, pin_memory=True)
        _staging["pinned"] = stage
    out = np.empty(tuple(t.shape), dtype=_NUMPY_DTYPES[t.dtype])
    src = t.view(-1).view(torch.uint8)
    dst = out.reshape(-1).view(np.uint8)
    stream = torch.cuda.current_stream(t.device)
    done = [torch.cuda.Event(), torch.cuda.Event()]
    pending = None
    for i, off in enumerate(range(0, nbytes, _CHUNK)):
        m = min(_CHUNK, nbytes - off)
        # chunk i - 2 used this half and was copied out in the previous iteration
        stage[(i % 2) * _CHUNK:(i % 2) * _CHUNK + m].copy_(src[off:off + m], non_blocking=True)
        done[i % 2].record(stream)
        if pending is not None:
            j, poff, pm = pending
            done[j % 2].synchronize()
            dst[poff:poff + pm] = stage[(j % 2) * _CHUNK:(j % 2) * _CHUNK + pm].numpy()
        pending = (i, off, m)
    j, poff, pm = pending
    done[j % 2].synchronize()
    dst[poff:poff + pm] = stage[(j % 2) * _CHUNK:(j % 2) * _CHUNK + pm].numpy()
    return out

__all__ = [
    "SharedAnalyzerProxy",
    "MaxScoreOverRotations",
    "PeakCaller",
    "PeakCallerSort",
    "PeakCallerMaximumFilter",
]


class SharedAnalyzerProxy:
    """Holds an analyzer and its state so scoring loops can call
    ``callback(scores, rotation_matrix=R)`` (tme/analyzer/proxy.py:92-123). Work
    stays in one process, so the state is never shared."""

    def __init__(self, analyzer_class, analyzer_params: Dict, shm_handler=None, **kwargs):
        self._shared = False
        self._analyzer = analyzer_class(**analyzer_params)
        self._state = self._analyzer.init_state()

    def __call__(self, *args, **kwargs):
        self._state = self._analyzer(self._state, *args, **kwargs)

    def result(self, **kwargs):
        return self._analyzer.result(self._state, **kwargs)

    def merge(self, *args, **kwargs):
        return self._analyzer.merge(*args, **kwargs)


class MaxScoreOverRotations:
    """Maximum score over rotations per translation with the index of the rotation
    that reached it (tme/analyzer/aggregation.py:31-432)."""

    def __init__(self, shape, offset=None, score_threshold: float = 0,
                 shm_handler=None, use_memmap: bool = False, inversion_mapping: bool = False,
                 jax_mode: bool = False, **kwargs):
        self._use_memmap = use_memmap
        self._score_threshold = score_threshold
        self._shape = tuple(int(x) for x in shape)
        self._inversion_mapping = inversion_mapping
        if offset is None:
            offset = np.zeros(len(self._shape), dtype=int)
        self._offset = np.asarray(offset).astype(int)

    @property
    def shareable(self):
        return True

    def init_state(self):
        dev = torch.device("cuda", torch.cuda.current_device())
        scores = torch.full(self._shape, float(self._score_threshold), dtype=torch.float32,
                            device=dev)
        rotations = torch.full(self._shape, -1, dtype=torch.int32, device=dev)
        return scores, rotations, {}

    def __call__(self, state, scores, rotation_matrix, **kwargs):
        prev, rotations, mapping = state
        index = len(mapping)
        rot = np.asarray(be.to_numpy_array(rotation_matrix), dtype=np.float32)
        if self._inversion_mapping:
            mapping[index] = rot
        else:
            index = mapping.setdefault(rot.tobytes(), index)
        if not isinstance(scores, torch.Tensor):
            scores = torch.as_tensor(np.asarray(scores, dtype=np.float32), device=prev.device)
        be.max_score_over_rotations(scores.to(torch.float32), prev, rotations, index)
        return prev, rotations, mapping

    @staticmethod
    def _invert_rmap(mapping: dict) -> dict:
        new_map, ndim = {}, None
        for k, v in mapping.items():
            rmat = np.frombuffer(k, dtype=np.float32)
            if ndim is None:
                ndim = int(np.sqrt(rmat.size))
            new_map[v] = rmat.reshape(ndim, ndim)
        return new_map

    def result(self, state, targetshape=None, templateshape=None, convolution_shape=None,
               fourier_shift=None, convolution_mode=None, **kwargs):
        scores, rotations, mapping = state
        if fourier_shift is not None:
            axis = tuple(range(len(fourier_shift)))
            scores = torch.roll(scores, shifts=tuple(int(s) for s in fourier_shift), dims=axis)
            rotations = torch.roll(rotations, shifts=tuple(int(s) for s in fourier_shift),
                                   dims=axis)
        if convolution_mode is not None:
            args = dict(s1=targetshape, s2=templateshape, convolution_mode=convolution_mode,
                        convolution_shape=convolution_shape)
            scores = apply_convolution_mode(scores, **args)
            rotations = apply_convolution_mode(rotations, **args)
        scores = download(scores)
        rotations = download(rotations)
        if self._inversion_mapping:
            mapping = {np.asarray(v, dtype=np.float32).tobytes(): k for k, v in mapping.items()}
        return scores, np.asarray(self._offset), rotations, self._invert_rmap(mapping)

    @staticmethod
    def _harmonize_states(states: List[Tuple]):
        new_map, out_shape = {}, None
        for i in range(len(states)):
            if states[i] is None:
                continue
            scores, offset, rotations, mapping = states[i]
            if out_shape is None:
                out_shape = np.zeros(scores.ndim, int)
            out_shape = np.maximum(out_shape, np.add(offset, scores.shape))
            new_param = {}
            for key, value in mapping.items():
                b = np.asarray(value, dtype=np.float32).tobytes()
                new_param[b] = key
                if b not in new_map:
                    new_map[b] = len(new_map)
            states[i] = (scores, offset, rotations, new_param)
        out_shape = None if out_shape is None else tuple(int(x) for x in out_shape)
        return new_map, out_shape, states

    @classmethod
    def merge(cls, results: List[Tuple], **kwargs):
        """tme/analyzer/aggregation.py:305-432 (in-memory)."""
        results = [r for r in results]
        if len(results) == 1:
            return results[0]
        master, out_shape, results = cls._harmonize_states(results)
        if out_shape is None:
            return None
        sd, rd = results[0][0].dtype, results[0][2].dtype
        scores_out = np.full(out_shape, fill_value=kwargs.get("score_threshold", 0), dtype=sd)
        rot_out = np.full(out_shape, fill_value=-1, dtype=rd)
        for i in range(len(results)):
            if results[i] is None:
                continue
            scores, offset, rotations, mapping = results[i]
            stops = np.add(offset, scores.shape).astype(int)
            idx = tuple(slice(*pos) for pos in zip(offset, stops))
            upd = scores > scores_out[idx]
            scores_out[idx][upd] = scores[upd]
            lut = np.arange(len(mapping) + 1, dtype=rot_out.dtype)
            for key, value in mapping.items():
                lut[value] = master[key]
            ur = rotations[upd]
            if len(ur):
                rot_out[idx][upd] = lut[ur]
            results[i] = None
        return (scores_out, np.zeros(scores_out.ndim, dtype=int), rot_out,
                cls._invert_rmap(master))


class PeakCaller:
    """Base class of the peak callers (tme/analyzer/peaks.py:146-620): candidate
    peaks per score map, validity masking, greedy minimum-distance filtering and
    top-k selection against the running state."""

    def __init__(self, shape, num_peaks: int = 1000, min_distance: int = 1,
                 min_boundary_distance: int = 0, min_score: float = None,
                 max_score: float = None, batch_dims=None, shm_handler=None, **kwargs):
        if num_peaks <= 0:
            raise ValueError("num_peaks has to be larger than 0.")
        if min_distance < 0:
            raise ValueError("min_distance has to be non-negative.")
        if min_boundary_distance < 0:
            raise ValueError("min_boundary_distance has to be non-negative.")
        if batch_dims is not None:
            raise NotImplementedError("batched peak calling is not supported")
        self.shape = shape
        self.num_peaks = int(num_peaks)
        self.min_distance = int(min_distance)
        self.min_boundary_distance = int(min_boundary_distance)
        self.batch_dims = None
        self.min_score, self.max_score = min_score, max_score

    @property
    def shareable(self):
        return False

    def call_peaks(self, scores, **kwargs):
        raise NotImplementedError

    def init_state(self):
        ndim = len(self.shape)
        translations = np.full((self.num_peaks, ndim), -1, dtype=np.int32)
        rotations = np.zeros((self.num_peaks, ndim, ndim), dtype=np.float32)
        for i in range(ndim):
            rotations[:, i, i] = 1.0
        scores = np.full((self.num_peaks,), -1, dtype=np.float32)
        details = np.full((self.num_peaks,), -1, dtype=np.float32)
        return translations, rotations, scores, details

    def _get_peak_mask(self, peaks: np.ndarray, ps: np.ndarray, shape):
        """tme/analyzer/peaks.py:241-290, given the candidates' scores ``ps`` (the
        reference gathers them from the map inside; here they come gathered from the
        device) and the map's ``shape``."""
        from .peaks import topk_indices

        if not len(peaks):
            return None
        upper = np.subtract(np.asarray(shape), self.min_boundary_distance)
        valid = np.multiply(peaks < upper, peaks >= self.min_boundary_distance)
        valid = np.sum(valid, axis=1) == peaks.shape[1]
        valid = np.multiply(ps == ps, valid)
        if self.min_score is not None:
            valid = np.multiply(ps >= self.min_score, valid)
        if self.max_score is not None:
            valid = np.multiply(ps <= self.max_score, valid)
        if np.sum(valid) == 0:
            return None
        if np.sum(valid) > self.num_peaks or ps.shape[0] > self.num_peaks:
            top = topk_indices(ps * valid, min(ps.size, 2 * self.num_peaks))
            valid = np.full(ps.shape, 0, bool)
            valid[top] = True
            if self.min_score is not None:
                valid = np.multiply(ps >= self.min_score, valid)
            if self.max_score is not None:
                valid = np.multiply(ps <= self.max_score, valid)
        return valid

    def call_candidates(self, scores, **kwargs):
        """(positions, their scores, details) of this caller's candidate peaks. The
        default gathers the scores of ``call_peaks``'s positions from the map on the
        device; callers that produce scores with their positions override it."""
        positions, details = self.call_peaks(scores=scores, **kwargs)
        if positions is None or len(positions) == 0:
            return None, None, details
        positions = np.asarray(positions).astype(np.int64)
        s = scores if isinstance(scores, torch.Tensor) else torch.as_tensor(np.asarray(scores))
        s = s.to(device=torch.device("cuda", torch.cuda.current_device()))
        idx = torch.as_tensor(positions, device=s.device)
        ps = s[tuple(idx.T)].to(torch.float32).cpu().numpy()
        return positions, ps, details

    def __call__(self, state, scores, rotation_matrix, **kwargs):
        """tme/analyzer/peaks.py:327-384 for one score map. The map stays on the device:
        only the candidates (positions and scores) come to the host for the reference's
        selection and greedy-filter bookkeeping."""
        positions, ps, details = self.call_candidates(
            scores=scores, rotation_matrix=rotation_matrix, min_score=self.min_score,
            max_score=self.max_score)
        if positions is None or len(positions) == 0:
            return state
        valid = self._get_peak_mask(positions, ps, tuple(scores.shape))
        if valid is None:
            return state
        positions = positions[valid]
        pscores = ps[valid]
        pdetails = np.full(pscores.shape, -1, dtype=np.float32) if details is None else \
            np.asarray(details)[valid]
        rot = np.asarray(be.to_numpy_array(rotation_matrix), dtype=np.float32)
        rots = np.repeat(rot.reshape(1, *rot.shape), positions.shape[0], axis=0)
        return self._update(state, positions, pdetails, pscores, rots)

    def _update(self, state, peak_positions, peak_details, peak_scores, peak_rotations,
                offset=None):
        """tme/analyzer/peaks.py:531-583."""
        from .peaks import filter_points_indices, topk_indices

        translations, rotations, scores, details = state
        peak_positions = np.asarray(peak_positions)
        if offset is not None:
            peak_positions = np.add(peak_positions, np.asarray(offset).astype(peak_positions.dtype))
        positions = np.concatenate((translations, peak_positions))
        rotations = np.concatenate((rotations, peak_rotations))
        scores = np.concatenate((scores, np.asarray(peak_scores, dtype=np.float32)))
        details = np.concatenate((details, np.asarray(peak_details, dtype=np.float32)))
        order = filter_points_indices(positions, self.min_distance, scores=scores)
        top = topk_indices(scores[order], min(len(order), self.num_peaks))
        final = np.asarray(order)[top]
        return positions[final], rotations[final], scores[final], details[final]

    def result(self, state, fast_shape=None, targetshape=None, templateshape=None,
               convolution_shape=None, fourier_shift=None, convolution_mode=None, **kwargs):
        """tme/analyzer/peaks.py:585-620 with score_to_cart (tme/analyzer/_utils.py:120-191):
        wrap by the Fourier shift, crop to the convolution mode's output box and drop
        rows with negative coordinates."""
        translations, rotations, scores, details = state
        positions = np.asarray(translations).astype(np.int64)
        valid = np.ones(positions.shape[0], dtype=bool)
        if fourier_shift is not None:
            positions = np.mod(positions + np.asarray(fourier_shift), np.asarray(fast_shape))
        if convolution_mode is not None:
            conv = np.asarray(convolution_shape)
            if convolution_mode == "same":
                out_shape = np.asarray(targetshape)
            elif convolution_mode == "valid":
                out_shape = np.subtract(targetshape, templateshape) + 1
            else:
                out_shape = conv
            starts = np.divide(np.subtract(conv, out_shape), 2).astype(np.int32)
            stops = starts + out_shape
            valid = np.sum(np.multiply(positions >= starts, positions < stops), axis=1) \
                == positions.shape[1]
            positions = positions - starts
        valid = np.multiply(np.sum(positions >= 0, axis=1) == positions.shape[1], valid)
        valid = valid.astype(bool)
        return positions[valid], rotations[valid], scores[valid], details[valid]

    @classmethod
    def merge(cls, results=List[Tuple], **kwargs):
        """tme/analyzer/peaks.py:386-426."""
        if "shape" not in kwargs:
            kwargs["shape"] = tuple(1 for _ in range(results[0][0].shape[1]))
        base = cls(**kwargs)
        state = base.init_state()
        for r in results:
            if len(r) == 0:
                continue
            pos, rot, sc, det = r
            state = base._update(state, np.asarray(pos), np.asarray(det), np.asarray(sc),
                                 np.asarray(rot), offset=kwargs.get("offset", None))
        return state


class PeakCallerSort(PeakCaller):
    """The ``num_peaks`` highest scores (tme/analyzer/peaks.py:641-659)."""

    def call_peaks(self, scores, **kwargs):
        from .peaks import topk_indices_device

        coords = topk_indices_device(scores, min(self.num_peaks, int(np.prod(scores.shape))))
        return coords, None


class PeakCallerMaximumFilter(PeakCaller):
    """Local maxima of a box maximum filter with edge ``min_distance``
    (tme/analyzer/peaks.py:662-670)."""

    def call_peaks(self, scores, **kwargs):
        from .peaks import max_filter_coordinates

        return max_filter_coordinates(scores, self.min_distance), None

    def call_candidates(self, scores, **kwargs):
        from .peaks import max_filter_candidates

        positions, ps = max_filter_candidates(scores, self.min_distance)
        return positions, ps, None
