"""The tensor-core x pass (tcgen05; BF16 head/tail operands for FP32 output, FP16
Hankel operands for half output) against a direct
evaluation of the circular correlation it computes, for each column:
H[b][x'] = sum_{x < t0} scale * C[(x' - x) mod n0] * G[b][x]."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference(G, C, t0, scale):
    nb = G.shape[0]
    n0 = C.shape[0]
    H = np.zeros((nb,) + C.shape, np.complex128)
    for x in range(t0):
        H += scale * np.roll(C, x, axis=0)[None] * G[:, x][:, None]
    return H


@pytest.mark.parametrize("n0,n1,h2,t0,nb,half", [
    (64, 2, 5, 12, 8, False),
    (128, 3, 9, 48, 32, False),
    (128, 2, 7, 20, 20, False),
    (64, 2, 6, 16, 40, False),
    (128, 2, 9, 48, 32, True),
    (128, 2, 5, 48, 128, False),
    (64, 2, 5, 24, 100, True),
    (256, 2, 9, 48, 32, True),
    (512, 1, 7, 40, 64, True),
    (256, 2, 5, 20, 120, True),
    # persistent warp-specialised kernel: several items per CTA, both operand buffers
    # reused, 16- and 32-rotation groups, t0 up to 64
    (128, 40, 65, 48, 32, True),
    (256, 40, 33, 20, 7, True),
    (512, 16, 24, 64, 16, True),
    (384, 12, 101, 48, 29, True),
])
def test_xcorr_tc_matches_direct(n0, n1, h2, t0, nb, half):
    import torch

    from pytme_b200 import _native as N

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(n0 + t0 + nb)
    G = (rng.normal(size=(nb, t0, n1, h2)) + 1j * rng.normal(size=(nb, t0, n1, h2)))
    C = (rng.normal(size=(n0, n1, h2)) + 1j * rng.normal(size=(n0, n1, h2)))
    G = G.astype(np.complex64)
    C = C.astype(np.complex64)
    scale = 0.37
    g = torch.from_numpy(G.view(np.float32)).cuda()
    c = torch.from_numpy(C.view(np.float32)).cuda()
    dt = torch.float16 if half else torch.float32
    h = torch.zeros((nb, n0, n1, h2, 2), dtype=dt, device="cuda")
    N.check(N.lib.tm_xcorr_tc_test(N.ptr(g), N.ptr(c), nb, t0, n0, n1, h2, scale, N.ptr(h),
                                   int(half), N.stream_ptr()), "tm_xcorr_tc_test")
    got = h.float().cpu().numpy()
    got = got[..., 0] + 1j * got[..., 1]
    want = _reference(G.astype(np.complex128), C.astype(np.complex128), t0, scale)
    err = np.abs(got - want).max() / np.abs(want).max()
    # BF16 head + tail operands: about 16 significant bits per product; the half-output
    # path takes FP16 operands (11 bits) and FP16 storage
    assert err < (2e-3 if half else 5e-5), err
