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


# ---------------------------------------------------------------- sharded public API
def _stub_score_map(rot, shape, field):
    # a deterministic score map per rotation, quantised to produce exact ties across
    # rotations (the lower index must win them)
    m = np.cos(field * (float(np.asarray(rot, np.float64).sum()) + 3.0))
    return torch.from_numpy((np.round(m * 8) / 8).astype(np.float32))


def _stub_setup(matching_data, fast_shape, **kwargs):
    rng = np.random.default_rng(5)
    return {"fast_shape": tuple(fast_shape), "field": rng.uniform(0, 7, size=tuple(fast_shape))}


def _stub_score(rotations, callback, fast_shape, field, **kwargs):
    """The fused scoring contract on the host: strict-> updates of the analyzer state
    with rotation i of the chunk recorded as len(mapping) + i."""
    scores, idx, mapping = callback._state
    first = len(mapping)
    for i, r in enumerate(np.asarray(rotations)):
        m = _stub_score_map(r, fast_shape, field)
        upd = m > scores
        scores[upd] = m[upd]
        idx[upd] = first + i
        mapping[first + i] = np.asarray(r, np.float32)
    return callback


def _cpu_max_score_class():
    from pytme_b200.analyzer import MaxScoreOverRotations

    class CpuMaxScore(MaxScoreOverRotations):
        """The analyzer with its state in host tensors (these ranks have no GPU)."""

        def init_state(self):
            return (torch.full(self._shape, float(self._score_threshold), dtype=torch.float32),
                    torch.full(self._shape, -1, dtype=torch.int32), {})

    return CpuMaxScore


def _sharded_inputs():
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(9)
    target = rng.normal(size=(12, 10, 9)).astype(np.float32)
    template = rng.normal(size=(4, 4, 4)).astype(np.float32)
    rots = syn.random_rotation_matrices(23, rng)
    return target, template, rots


def _run_scan(process_group=None):
    import pytme_b200 as P

    target, template, rots = _sharded_inputs()
    md = P.MatchingData(target, template)
    md.rotations = rots
    return P.scan_subsets(md, matching_score=_stub_score, matching_setup=_stub_setup,
                          callback_class=_cpu_max_score_class(),
                          callback_class_args={"score_threshold": 0}, job_schedule=(1, 1),
                          interpolation_order=1, process_group=process_group)


def _sharded_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world)
    res = _run_scan(process_group="default")
    out.put((rank, res[0], res[2], {k: v.tolist() for k, v in res[3].items()}))
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()


def test_scan_subsets_shards_rotations_over_two_ranks():
    """scan_subsets(process_group=...) on two gloo ranks with a host stub scorer: every
    rank ends with the analyzer state of one process scoring all rotations in order
    (scores, rotation indices and the index -> rotation mapping)."""
    seq = _run_scan()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_sharded_worker, args=(i, 2, port, q)) for i in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, s, r, mapping in got:
        assert np.array_equal(s, seq[0]), rank
        assert np.array_equal(r, seq[2]), rank
        assert mapping == {k: v.tolist() for k, v in seq[3].items()}, rank


def test_pack_keys_nan_never_wins():
    s = torch.tensor([float("nan"), -5.0, float("nan")], dtype=torch.float32)
    r = torch.tensor([0, 3, -1], dtype=torch.int32)
    k = pack_keys(s, r)
    assert k[1] > k[0] and k[1] > k[2]
    s2, r2 = unpack_keys(torch.maximum(k[0:1], k[1:2]))
    assert float(s2[0]) == -5.0 and int(r2[0]) == 3
