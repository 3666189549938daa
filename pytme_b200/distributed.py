"""Rotation sharding across ranks and the single exchange step of a sharded scan.

Each rank scores a contiguous share of the rotation set over the whole target
(the reference's rotation split, tme/matching_data.py:822-844) and keeps its own
(max score, rotation index) state. ``merge_max_argmax`` combines the states with
one MAX all-reduce on a packed int64 key: the high 32 bits hold the score's bits
mapped to an order-preserving signed integer, the low 32 bits ``2^32 - 1 - index``
(0 for "no rotation"), so the maximum key is the highest score and, among equal
scores, the lowest rotation index — the result of scoring all rotations in order
with the strict ``>`` update (tme/backends/npfftw_backend.py:503-535).
"""
from __future__ import annotations

import torch
import torch.distributed as dist

__all__ = ["rotation_share", "pack_keys", "unpack_keys", "merge_max_argmax",
           "score_rotation_shares"]


def rotation_share(n_rotations: int, rank: int, world: int):
    """[start, stop) of this rank's contiguous share (the last rank takes the rest)."""
    per = n_rotations // world
    start = rank * per
    stop = n_rotations if rank == world - 1 else start + per
    return start, stop


def pack_keys(scores: torch.Tensor, rotations: torch.Tensor) -> torch.Tensor:
    """Order-preserving int64 keys of (score, rotation). A NaN score gets the smallest
    key, so it never wins over a number (the strict ``>`` update never stores one)."""
    bits = scores.contiguous().view(torch.int32).to(torch.int64)
    hi = torch.where(bits < 0, bits ^ 0x7FFFFFFF, bits)
    rot = rotations.to(torch.int64)
    lo = torch.where(rot < 0, torch.zeros_like(rot), 0xFFFFFFFF - rot)
    nan = torch.isnan(scores)
    hi = torch.where(nan, torch.full_like(hi, -(1 << 31)), hi)
    lo = torch.where(nan, torch.zeros_like(lo), lo)
    return (hi << 32) | lo


def unpack_keys(keys: torch.Tensor):
    hi = keys >> 32
    bits = torch.where(hi < 0, hi ^ 0x7FFFFFFF, hi).to(torch.int32)
    scores = bits.view(torch.float32)
    lo = keys & 0xFFFFFFFF
    rot = torch.where(lo == 0, torch.full_like(lo, -1), 0xFFFFFFFF - lo).to(torch.int32)
    return scores, rot


def merge_max_argmax(scores: torch.Tensor, rotations: torch.Tensor, group=None):
    """In-place merge of per-rank (max, argmax) states over the process group."""
    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return scores, rotations
    keys = pack_keys(scores, rotations)
    dist.all_reduce(keys, op=dist.ReduceOp.MAX, group=group)
    s, r = unpack_keys(keys)
    scores.copy_(s)
    rotations.copy_(r)
    return scores, rotations


def score_rotation_shares(matching_score, setup, rotations, callback, group=None):
    """Scores this rank's contiguous share of ``rotations`` into ``callback`` and merges
    the ranks' states, leaving every rank's analyzer as one process scoring all
    rotations in order would have left it (the reference's multi-device rotation split,
    tme/matching_exhaustive.py:131-133 with tme/matching_data.py:822-844, and the merge of
    tme/analyzer/aggregation.py:305-432 reduced to one collective).

    The callback must hold a MaxScoreOverRotations-style state (scores, rotation
    indices, {index: rotation}) under inversion mapping: rotation i is recorded as index
    i, so the mapping is pre-filled with the rotations before this rank's share (the
    scoring function takes len(mapping) as its first index), and completed with those
    after it once the states are merged."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    analyzer = getattr(callback, "_analyzer", None)
    state = getattr(callback, "_state", None)
    if analyzer is None or state is None or not getattr(analyzer, "_inversion_mapping", False) \
            or not isinstance(state[0], torch.Tensor):
        raise NotImplementedError("rotation sharding needs a MaxScoreOverRotations callback "
                                  "with inversion mapping (job_schedule inner jobs = 1)")
    rot = rotations
    n = int(rot.shape[0])
    lo, hi = rotation_share(n, rank, world)
    scores, indices, mapping = state
    if len(mapping) != 0:
        raise ValueError("rotation sharding starts from an empty analyzer state")
    as_matrix = (lambda i: rot[i]) if isinstance(rot, torch.Tensor) else \
        (lambda i: __import__("numpy").asarray(rot[i], dtype="float32"))
    for i in range(lo):
        mapping[i] = as_matrix(i)
    if hi > lo:
        matching_score(rotations=rot[lo:hi], callback=callback, **setup)
    scores, indices, mapping = callback._state
    if len(mapping) != hi:
        raise RuntimeError(f"rank {rank} recorded {len(mapping)} rotations, expected {hi}")
    merge_max_argmax(scores, indices, group=group)
    for i in range(hi, n):
        mapping[i] = as_matrix(i)
    return callback
