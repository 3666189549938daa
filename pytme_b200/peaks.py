"""Peak-calling helpers: maximum-filter peaks and the greedy distance filter on the
device, plus the reference's top-k ordering.

``max_filter_coordinates`` follows NumpyFFTWBackend.max_filter_coordinates
(tme/backends/npfftw_backend.py:200-206) through ``tm_max_filter_peaks``;
``filter_points_indices`` follows tme/analyzer/peaks.py:68-106 with the greedy
filter of find_candidate_indices (tme/external/bindings.cpp:85-126) running as
``tm_find_candidate_indices``; ``topk_indices`` is the reference's
argpartition/argsort ordering (tme/backends/npfftw_backend.py:177-182) on the
small candidate arrays.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N

__all__ = ["max_filter_coordinates", "max_filter_candidates", "find_candidate_indices",
           "filter_points_indices", "filter_bucket", "topk_indices", "topk_indices_device"]


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def max_filter_coordinates(scores, min_distance: int) -> np.ndarray:
    """(n, 3) int64 coordinates where the box maximum filter of edge ``min_distance``
    equals the score, in C order (as ``np.nonzero`` returns them)."""
    s = scores if isinstance(scores, torch.Tensor) else torch.as_tensor(
        np.ascontiguousarray(scores, dtype=np.float32))
    s = s.to(device=_dev(), dtype=torch.float32).contiguous()
    if s.ndim != 3:
        raise NotImplementedError("peak calling is implemented for 3D score maps")
    a = torch.empty_like(s)
    b = torch.empty_like(s)
    mask = torch.empty(s.shape, dtype=torch.uint8, device=s.device)
    N.check(N.lib.tm_max_filter_peaks(N.ptr(s), *s.shape, int(min_distance), N.ptr(a), N.ptr(b),
                                      N.ptr(mask), N.stream_ptr()), "tm_max_filter_peaks")
    return torch.nonzero(mask).cpu().numpy().astype(np.int64)


def max_filter_candidates(scores, min_distance: int):
    """Peaks of the box maximum filter with their scores: (n, 3) int64 coordinates in C
    order and their n float32 scores. The filter, the compaction and the gather of the
    scores run on the device; only the candidates travel to the host (a few thousand
    values for a 512x512x200 map, not the map)."""
    s = scores if isinstance(scores, torch.Tensor) else torch.as_tensor(
        np.ascontiguousarray(scores, dtype=np.float32))
    s = s.to(device=_dev(), dtype=torch.float32).contiguous()
    if s.ndim != 3:
        raise NotImplementedError("peak calling is implemented for 3D score maps")
    a = torch.empty_like(s)
    b = torch.empty_like(s)
    mask = torch.empty(s.shape, dtype=torch.uint8, device=s.device)
    N.check(N.lib.tm_max_filter_peaks(N.ptr(s), *s.shape, int(min_distance), N.ptr(a), N.ptr(b),
                                      N.ptr(mask), N.stream_ptr()), "tm_max_filter_peaks")
    del a, b
    flat = torch.nonzero(mask.reshape(-1)).reshape(-1)
    vals = s.reshape(-1)[flat]
    idx = flat.cpu().numpy()
    coords = np.stack(np.unravel_index(idx, tuple(s.shape)), axis=1).astype(np.int64)
    return coords, vals.cpu().numpy()


def find_candidate_indices(coordinates, min_distance: int) -> np.ndarray:
    """Greedy filter on the device; returns the kept indices in input order."""
    c = np.ascontiguousarray(np.asarray(coordinates), dtype=np.int64)
    n = int(c.shape[0])
    if n == 0:
        return np.zeros(0, dtype=np.int64)
    if c.ndim != 2 or c.shape[1] != 3:
        raise NotImplementedError("the greedy filter is implemented for 3D coordinates")
    dev = _dev()
    ct = torch.as_tensor(c, device=dev)
    out = torch.empty(n, dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    ws_bytes = int(N.lib.tm_find_candidate_indices_workspace(n))
    ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=dev)
    N.check(N.lib.tm_find_candidate_indices(N.ptr(ct), n, int(min_distance), N.ptr(out),
                                            N.ptr(cnt), N.ptr(ws), N.stream_ptr()),
            "tm_find_candidate_indices")
    k = int(cnt.item())
    return out[:k].cpu().numpy().astype(np.int64)


def filter_bucket(coordinates, min_distance: float, scores=None) -> np.ndarray:
    """One point per grid cell of edge ``min_distance`` (the reference's rule for large
    point sets, tme/analyzer/peaks.py:39-64): cells from the integer part of
    (coordinate - minimum) / min_distance, flattened with per-axis strides of
    (max cell + 1)^axis. With scores, each cell keeps its highest-scoring point (an
    argsort of cell rank minus the score scaled into [0, 1)), listed by cell; without,
    the first point of each cell in input order."""
    c = np.asarray(coordinates)
    c = c - c.min(axis=0)
    cells = (c / min_distance).astype(int)
    strides = np.power(cells.max(axis=0) + 1, np.arange(cells.shape[1]))
    flat = (cells * strides).sum(axis=1)
    if scores is None:
        _, first = np.unique(flat, return_index=True)
        return first[np.argsort(first)]
    _, rank = np.unique(flat, return_inverse=True)
    sc = np.asarray(scores)
    sc = sc - sc.min()
    sc = sc / (sc.max() + 0.1)
    order = np.argsort(rank - sc)
    cell_of = rank[order]
    first_of_cell = np.concatenate(([True], cell_of[1:] != cell_of[:-1]))
    return order[first_of_cell]


def _filter_lower_triangle(coordinates, min_distance: float) -> np.ndarray:
    """The reference's rule at exactly its point cutoff (tme/analyzer/peaks.py:101-106):
    point i is kept when every earlier point lies farther than ``min_distance`` (Euclidean,
    float64), in input order; evaluated on the device in blocks of rows."""
    c = torch.as_tensor(np.asarray(coordinates), device=_dev(), dtype=torch.float64)
    n = c.shape[0]
    keep = np.zeros(n, dtype=bool)
    block = 2048
    for i0 in range(0, n, block):
        i1 = min(n, i0 + block)
        d = torch.cdist(c[i0:i1], c[:i1], compute_mode="donot_use_mm_for_euclid_dist")
        earlier = (torch.arange(i1, device=c.device)[None, :] <
                   torch.arange(i0, i1, device=c.device)[:, None])
        far = ((d > min_distance) | ~earlier).all(dim=1)
        keep[i0:i1] = far.cpu().numpy()
    return np.nonzero(keep)[0]


def filter_points_indices(coordinates, min_distance: float, scores=None,
                          bucket_cutoff: int = 100000) -> np.ndarray:
    """tme/analyzer/peaks.py:68-106 (unbatched). Below ``bucket_cutoff`` points: the
    greedy filter on the device in descending score order; above it: ``filter_bucket``;
    at exactly the cutoff the reference falls through to its lower-triangle distance
    rule in input order, reproduced by ``_filter_lower_triangle``."""
    coordinates = np.asarray(coordinates)
    if min_distance <= 0:
        return np.arange(coordinates.shape[0])
    n = coordinates.shape[0]
    if n == 0:
        return np.zeros(0, dtype=np.int64)
    if n > bucket_cutoff:
        return filter_bucket(coordinates, min_distance, scores)
    if n == bucket_cutoff:
        return _filter_lower_triangle(coordinates, min_distance)
    if scores is not None:
        order = np.argsort(-np.asarray(scores))
        kept = find_candidate_indices(coordinates[order], int(min_distance))
        return order[kept]
    return _filter_lower_triangle(coordinates, min_distance)


def topk_indices(arr, k: int) -> np.ndarray:
    """Indices of the k largest entries of a 1D array, largest first."""
    temp = np.asarray(arr).reshape(-1)
    k = min(int(k), temp.size)
    if k <= 0:
        return np.zeros(0, dtype=np.int64)
    idx = np.argpartition(temp, -k)[-k:][:k]
    return idx[np.argsort(temp[idx])][::-1]


def topk_indices_device(scores, k: int) -> np.ndarray:
    """(k, ndim) coordinates of the k largest scores of a device score map."""
    s = scores if isinstance(scores, torch.Tensor) else torch.as_tensor(np.asarray(scores))
    s = s.to(device=_dev(), dtype=torch.float32)
    vals, idx = torch.topk(s.reshape(-1), int(k), largest=True, sorted=True)
    return np.stack(np.unravel_index(idx.cpu().numpy(), tuple(s.shape)), axis=1)
