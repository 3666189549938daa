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

__all__ = ["rotation_share", "pack_keys", "unpack_keys", "merge_max_argmax"]


def rotation_share(n_rotations: int, rank: int, world: int):
    """[start, stop) of this rank's contiguous share (the last rank takes the rest)."""
    per = n_rotations // world
    start = rank * per
    stop = n_rotations if rank == world - 1 else start + per
    return start, stop


def pack_keys(scores: torch.Tensor, rotations: torch.Tensor) -> torch.Tensor:
    bits = scores.contiguous().view(torch.int32).to(torch.int64)
    hi = torch.where(bits < 0, bits ^ 0x7FFFFFFF, bits)
    rot = rotations.to(torch.int64)
    lo = torch.where(rot < 0, torch.zeros_like(rot), 0xFFFFFFFF - rot)
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
