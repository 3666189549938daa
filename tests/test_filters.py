"""Fourier filters against the reference's arrays (tests/golden/filters.npz): the host
restatement (no GPU) and the device builder (GPU)."""
import numpy as np
import pytest

from pytme_b200 import filters as F
from tests.golden.filter_cases import FILTER_CASES, build_filter_case


@pytest.mark.parametrize("i", range(len(FILTER_CASES)))
def test_host_filters_bit_exact(golden, i):
    g = golden("filters.npz")[f"case{i}"]
    got = np.asarray(build_filter_case(FILTER_CASES[i], F.CTFReconstructed,
                                       F.WedgeReconstructed, F.Compose))
    assert got.dtype == np.float32 and got.shape == g.shape
    assert np.array_equal(got, g)


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(FILTER_CASES)))
def test_device_filters_match_reference(golden, i):
    """Bit-exact except where CUDA's and the host's double-precision sine differ in the
    last bit and the float32 rounding of the CTF lands on the other side (at most one
    float32 ulp, at a few voxels in a million)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    g = golden("filters.npz")[f"case{i}"]
    shape, comps, rfft = FILTER_CASES[i]
    objs = [F.CTFReconstructed(**kw) if kind == "ctf" else
            F.WedgeReconstructed(create_continuous_wedge=True, **kw) for kind, kw in comps]
    got = F.device_filter(F.Compose(objs), shape, return_real_fourier=rfft).cpu().numpy()
    assert got.shape == g.shape
    diff = got != g
    ulp = np.abs(got.view(np.int32).astype(np.int64) - g.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1
    assert diff.mean() <= 1e-5 or diff.sum() <= 2


@pytest.mark.gpu
def test_device_filters_config4_time():
    """Config-4 filter set (12 targets up to 320 x 320 x 160, 3 templates, per-tomogram
    defocus and wedge) built on the device and on the host; the device must agree and be
    faster."""
    import time

    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(4)
    shapes = [(128, 128, 128), (320, 320, 160), (256, 256, 128), (192, 192, 96)] * 3
    tshapes = [(24,) * 3, (32,) * 3, (40,) * 3]
    jobs = []
    for s in shapes:
        df = float(rng.uniform(15000, 45000))
        w = float(rng.uniform(50, 65))
        for t in tshapes:
            jobs.append((s, t, df, w))
    def filters(j):
        s, t, df, w = j
        tf = F.Compose([F.CTFReconstructed(defocus_x=df, sampling_rate=6.8),
                        F.WedgeReconstructed(angles=(w, w), opening_axis=2, tilt_axis=0)])
        gf = F.Compose([F.WedgeReconstructed(angles=(w, w), opening_axis=2, tilt_axis=0)])
        return (tf, t), (gf, s)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev = []
    for j in jobs:
        (tf, t), (gf, s) = filters(j)
        dev.append((F.device_filter(tf, t), F.device_filter(gf, s)))
    torch.cuda.synchronize()
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    for j, (a, b) in list(zip(jobs, dev))[:6]:
        (tf, t), (gf, s) = filters(j)
        ha = tf(shape=t, return_real_fourier=True)["data"]
        hb = gf(shape=s, return_real_fourier=True)["data"]
        assert np.array_equal(a.cpu().numpy(), ha) or \
            np.abs(a.cpu().numpy() - ha).max() <= 1e-6
        assert np.array_equal(b.cpu().numpy(), hb)
    t_host = (time.perf_counter() - t0) * len(jobs) / 6
    print(f"config-4 filters: device {t_dev * 1e3:.1f} ms, host {t_host * 1e3:.0f} ms "
          f"(extrapolated from 6 of {len(jobs)} pairs)")
    assert t_dev < t_host
