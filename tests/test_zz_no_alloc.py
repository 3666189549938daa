"""The allocation-free greedy filter, called through the C ABI.

tm_find_candidate_indices_noalloc serves callers that cannot allocate device
memory while they run: it keeps its scratch in a fixed array inside the library
instead of asking for a workspace. Its results must equal those of
tm_find_candidate_indices (integer indices, so exactly) on consecutive calls, since
every call reuses the same scratch array. This file is collected last so a run that
stops at the first failure has already run everything else."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(fn_name, coords, md, use_workspace):
    import torch

    from pytme_b200 import _native as N

    dev = torch.device("cuda", 0)
    c = torch.as_tensor(np.ascontiguousarray(coords, dtype=np.int64), device=dev)
    n = int(coords.shape[0])
    out = torch.full((max(n, 1),), -7, dtype=torch.int32, device=dev)
    cnt = torch.full((1,), -7, dtype=torch.int32, device=dev)
    if use_workspace:
        ws = torch.empty(max(int(N.lib.tm_find_candidate_indices_workspace(n)), 8),
                         dtype=torch.uint8, device=dev)
        st = N.lib.tm_find_candidate_indices(c.data_ptr(), n, int(md), out.data_ptr(),
                                             cnt.data_ptr(), ws.data_ptr(), N.stream_ptr())
    else:
        st = getattr(N.lib, fn_name)(c.data_ptr(), n, int(md), out.data_ptr(), cnt.data_ptr(),
                                     N.stream_ptr())
    N.check(st, fn_name)
    torch.cuda.synchronize()
    k = int(cnt.item())
    return out[:k].cpu().numpy()


def test_noalloc_filter_matches_workspace_entry_point_on_consecutive_calls():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    rng = np.random.default_rng(99)
    # first call: beyond the shared-memory capacity, so the fixed scratch is used
    a = rng.integers(0, 300, size=(6000, 3)).astype(np.int64)
    # second call: a different, smaller point set reusing the same scratch
    b = rng.integers(0, 120, size=(2500, 3)).astype(np.int64)
    for coords, md in ((a, 8), (b, 5)):
        ref = _run("tm_find_candidate_indices", coords, md, use_workspace=True)
        got = _run("tm_find_candidate_indices_noalloc", coords, md, use_workspace=False)
        assert len(ref) > 1
        assert np.array_equal(got, ref)


def test_noalloc_filter_fills_its_whole_scratch():
    """TM_NOALLOC_MAX_POINTS well-separated points (a grid of spacing 2 with minimum
    distance 1): every point is kept, so the scratch array is written to its last
    entry; the result must equal the workspace entry point's, on two calls in a row.
    A negative minimum distance keeps every point, as the reference's integer rule
    floor(sqrt(d2)) <= min_distance never holds then."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    n = 65536
    g = np.stack(np.meshgrid(np.arange(64), np.arange(64), np.arange(16), indexing="ij"),
                 axis=-1).reshape(-1, 3).astype(np.int64) * 2
    assert g.shape[0] == n
    g = g[np.random.default_rng(5).permutation(n)]
    for _ in range(2):
        ref = _run("tm_find_candidate_indices", g, 1, use_workspace=True)
        got = _run("tm_find_candidate_indices_noalloc", g, 1, use_workspace=False)
        assert len(ref) == n
        assert np.array_equal(got, ref)
    close = np.random.default_rng(6).integers(0, 4, size=(3000, 3)).astype(np.int64)
    got = _run("tm_find_candidate_indices_noalloc", close, -3, use_workspace=False)
    assert np.array_equal(got, np.arange(3000))


def test_noalloc_filter_rejects_sizes_beyond_its_scratch():
    from pytme_b200 import _native as N

    n = 65537
    st = N.lib.tm_find_candidate_indices_noalloc(None, n, 3, None, None, None)
    assert st == N.TM_E_INVALID
    assert "fixed scratch" in N.last_error()
