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


# ----------------------------------------------------------------------------- whitening
from tests.golden.filter_cases import WHITENING_CASES, whitening_data  # noqa: E402


@pytest.mark.parametrize("i", range(len(WHITENING_CASES)))
def test_host_whitening_bit_exact(golden, i):
    """The host restatement of LinearWhiteningFilter against the reference's arrays
    (tests/golden/whitening.npz), from the same complex64 spectrum."""
    g = golden("whitening.npz")[f"case{i}"]
    dshape, fshape, rfft, n_bins = WHITENING_CASES[i]
    _, spec = whitening_data(i, dshape)
    got = F.LinearWhiteningFilter()(shape=fshape, data_rfft=spec, n_bins=n_bins,
                                    return_real_fourier=rfft)["data"]
    assert got.shape == g.shape
    assert np.array_equal(got, g)


def test_whitening_through_filter_evaluation_on_host():
    """A whitening filter in the scan's filter evaluation gets the target spectrum (the
    reference hands data_rfft to every filter); without a GPU it is built on the host."""
    from pytme_b200.matching import _evaluate_filter

    _, spec = whitening_data(0, WHITENING_CASES[0][0])
    got = _evaluate_filter(F.Compose([F.LinearWhiteningFilter()]), WHITENING_CASES[0][1],
                           data_rfft=spec, weight_type=None)
    want = F.LinearWhiteningFilter()(shape=WHITENING_CASES[0][1], data_rfft=spec)["data"]
    assert np.array_equal(got, want.astype(np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(WHITENING_CASES)))
def test_device_whitening_matches_reference(golden, i):
    """tm_whitening_filter against the reference's arrays from the same spectrum: the
    per-bin float64 sums run in another order, so values may differ in the last float32
    bit."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    g = golden("whitening.npz")[f"case{i}"].astype(np.float32)
    dshape, fshape, rfft, n_bins = WHITENING_CASES[i]
    _, spec = whitening_data(i, dshape)
    got = F.device_filter(F.LinearWhiteningFilter(), fshape, return_real_fourier=rfft,
                          data_rfft=torch.from_numpy(spec).cuda(), n_bins=n_bins)
    got = got.cpu().numpy()
    assert got.shape == g.shape
    ulp = np.abs(got.view(np.int32).astype(np.int64) - g.view(np.int32).astype(np.int64))
    assert ulp.max() <= 1


@pytest.mark.gpu
@pytest.mark.parametrize("order", [(0, 1, 2), (1, 0, 2), (2, 1, 0)])
def test_device_whitening_composed_with_ctf_and_wedge(order):
    """Whitening x CTF x wedge in any order on the device equals the host Compose (float64
    product rounded once to float32) within one float32 ulp."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dshape = (24, 20, 16)
    _, spec = whitening_data(0, dshape)
    items = [F.LinearWhiteningFilter(),
             F.CTFReconstructed(defocus_x=30000.0, sampling_rate=6.8),
             F.WedgeReconstructed(angles=(60, 60), opening_axis=2, tilt_axis=0,
                                  create_continuous_wedge=True)]
    filt = F.Compose([items[j] for j in order])
    want = np.asarray(filt(shape=dshape, return_real_fourier=True, data_rfft=spec)["data"],
                      dtype=np.float32)
    got = F.device_filter(filt, dshape, return_real_fourier=True,
                          data_rfft=torch.from_numpy(spec).cuda()).cpu().numpy()
    # the device CTF itself may differ from the host's by one ulp at a few voxels
    ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert ulp.max() <= 2
