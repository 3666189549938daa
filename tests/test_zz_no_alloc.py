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


def test_noalloc_filter_rejects_sizes_beyond_its_scratch():
    from pytme_b200 import _native as N

    n = 65537
    st = N.lib.tm_find_candidate_indices_noalloc(None, n, 3, None, None, None)
    assert st == N.TM_E_INVALID
    assert "fixed scratch" in N.last_error()
