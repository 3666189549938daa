"""Sharded-scan merge on CPU with two gloo ranks: the packed-key MAX all-reduce must
reproduce a sequential strict-> scan over all rotations (highest score, lowest
index on ties)."""
import os

import numpy as np
import torch
import torch.multiprocessing as mp

from pytme_b200.distributed import merge_max_argmax, pack_keys, rotation_share, unpack_keys


def _sequential(per_rot_scores, threshold=0.0):
    best = np.full(per_rot_scores.shape[1:], threshold, np.float32)
    arg = np.full(per_rot_scores.shape[1:], -1, np.int32)
    for i, s in enumerate(per_rot_scores):
        upd = s > best
        best[upd] = s[upd]
        arg[upd] = i
    return best, arg


def _worker(rank, world, port, data, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world)
    lo, hi = rotation_share(data.shape[0], rank, world)
    best = np.full(data.shape[1:], 0.0, np.float32)
    arg = np.full(data.shape[1:], -1, np.int32)
    for i in range(lo, hi):
        upd = data[i] > best
        best[upd] = data[i][upd]
        arg[upd] = i
    s, r = torch.from_numpy(best), torch.from_numpy(arg)
    merge_max_argmax(s, r)
    if rank == 0:
        out.put((s.numpy(), r.numpy()))
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()


def test_pack_roundtrip_and_order():
    s = torch.tensor([-3.5, -0.0, 0.0, 1e-30, 2.0, 2.0, float("inf")], dtype=torch.float32)
    r = torch.tensor([4, -1, 7, 0, 9, 3, 1], dtype=torch.int32)
    k = pack_keys(s, r)
    s2, r2 = unpack_keys(k)
    assert torch.equal(s2.view(torch.int32), s.view(torch.int32)) and torch.equal(r2, r)
    assert k[5] > k[4]  # equal score: lower rotation index wins
    assert torch.all(k[1:] >= k[:-1])


def test_two_rank_merge_equals_sequential_scan():
    rng = np.random.default_rng(0)
    data = rng.normal(size=(37, 6, 5, 4)).astype(np.float32)
    data[20] = data[3]  # exact ties across ranks
    data[30, 0, 0, 0] = data[2, 0, 0, 0] = 9.0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(i, 2, port, data, q)) for i in range(2)]
    for p in procs:
        p.start()
    s, r = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    best, arg = _sequential(data)
    assert np.array_equal(s, best)
    assert np.array_equal(r, arg)
