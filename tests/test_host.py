"""Host-side logic of the package (no GPU): shapes, padding, rotation matrices,
splits, analyzer merges, synthetic inputs."""
import numpy as np
import pytest

from oracle import tm_oracle as O
from pytme_b200 import matching as M
from pytme_b200 import synthetic as syn


@pytest.mark.parametrize("n", [1, 7, 11, 13, 17, 23, 48, 49, 97, 121, 143, 200, 1000, 2187])
def test_next_fast_len_matches_oracle(n):
    assert M.next_fast_len(n) == O.next_fast_len(n)


@pytest.mark.parametrize("tshape,mshape,pad", [
    ((64, 64, 64), (16, 16, 16), False), ((80, 80, 80), (41, 41, 35), False),
    ((80, 80, 80), (41, 41, 35), True), ((512, 512, 200), (48, 48, 48), False),
    ((10, 12, 14), (17, 5, 3), False)])
def test_fourier_padding(tshape, mshape, pad):
    with np.errstate(all="ignore"):
        import warnings

        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            assert M.fourier_padding(tshape, mshape, pad) == O.fourier_padding(tshape, mshape, pad)


def test_rigid_transform_matrices_match_reference_construction():
    rng = np.random.default_rng(7)
    rots = np.concatenate([syn.random_rotation_matrices(200, rng),
                           syn.super_fibonacci_rotations(100),
                           np.eye(3, dtype=np.float32)[None]])
    for shape in ((16, 16, 16), (48, 48, 48), (41, 41, 35)):
        c = np.divide(np.asarray(shape) - 1, 2)
        got = M.rigid_transform_matrices(rots, c)
        for i in range(rots.shape[0]):
            ref = O.rigid_transform_matrix(rots[i], c)
            # float32 construction; identical up to the last bit of the offset column
            assert np.array_equal(got[i, :3, :3], ref[:3, :3])
            np.testing.assert_allclose(got[i, :3, 3], ref[:3, 3], rtol=0, atol=4e-6)


def test_split_shape():
    s = M.split_shape((80, 80, 80), {0: 2})
    assert len(s) == 2
    assert s[0][0] == slice(0, 40) and s[1][0] == slice(40, 80)
    assert M.split_shape((81, 10, 10), {0: 2})[1][0] == slice(40, 81)


def test_subset_reflect_padding_uses_neighbours():
    t = np.arange(10 * 4 * 4, dtype=np.float32).reshape(10, 4, 4)
    md = M.MatchingData(t, np.ones((3, 3, 3), np.float32))
    sub, off = md.subset_by_slice(target_slice=(slice(5, 10), slice(0, 4), slice(0, 4)),
                                  target_pad=(2, 2, 2))
    assert off == (5, 0, 0)
    # left pad of 1 on axis 0 comes from the real neighbour row 4
    assert np.array_equal(sub.target[0, 1:5, 1:5], t[4])


def test_apply_convolution_mode():
    a = np.arange(20 * 20 * 20).reshape(20, 20, 20)
    assert M.apply_convolution_mode(a, "same", (16, 16, 16), (5, 5, 5)).shape == (16, 16, 16)
    assert M.apply_convolution_mode(a, "valid", (16, 16, 16), (5, 5, 5),
                                    convolution_shape=(20, 20, 20)).shape == (12, 12, 12)


def test_max_score_merge_follows_reference():
    from pytme_b200.analyzer import MaxScoreOverRotations

    r = np.eye(3, dtype=np.float32)
    r2 = np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    s1 = np.zeros((4, 4, 4), np.float32)
    s1[1, 1, 1] = 0.5
    s2 = np.zeros((4, 4, 4), np.float32)
    s2[1, 1, 1] = 0.7
    a = (s1, np.array([0, 0, 0]), np.where(s1 > 0, 0, -1).astype(np.int32), {0: r})
    b = (s2, np.array([2, 0, 0]), np.where(s2 > 0, 0, -1).astype(np.int32), {0: r2})
    out = MaxScoreOverRotations.merge([a, b])
    assert out[0].shape == (6, 4, 4)
    assert out[0][1, 1, 1] == np.float32(0.5) and out[0][3, 1, 1] == np.float32(0.7)
    assert out[2][3, 1, 1] == 1 and np.array_equal(out[3][1], r2)


def test_synthetic_generators():
    rng = np.random.default_rng(0)
    t = syn.blob_template(16, rng)
    assert t.shape == (16, 16, 16) and t.dtype == np.float32 and t.max() > 0.5
    m = syn.spherical_mask((16, 16, 16), 8, center=(7.5, 7.5, 7.5))
    assert m.sum() > 0 and set(np.unique(m)) <= {0.0, 1.0}
    R = syn.super_fibonacci_rotations(1000)
    np.testing.assert_allclose(R @ R.transpose(0, 2, 1), np.broadcast_to(np.eye(3), R.shape),
                               atol=1e-6)
    assert syn.rotation_count_for_angle(7) == 27672
    assert syn.rotation_count_for_angle(30) == 360


def test_subset_without_padding_is_the_slice():
    """Without padding the subset is the slice itself (no copy before the upload); with
    padding it is NumPy's reflect padding of the slice."""
    rng = np.random.default_rng(5)
    a = rng.normal(size=(9, 8, 7)).astype(np.float32)
    sl = (slice(1, 8), slice(0, 8), slice(2, 6))
    out = M.MatchingData._subset_array(a, sl, (0, 0, 0))
    assert np.shares_memory(out, a) and np.array_equal(out, a[sl])
    full = tuple(slice(0, n) for n in a.shape)
    out = M.MatchingData._subset_array(a, full, (2, 0, 3))
    assert np.array_equal(out, np.pad(a, ((1, 1), (0, 0), (2, 1)), mode="reflect"))


def test_filter_spectrum_need():
    """Only filters other than CTFs and wedges ask for the target spectrum."""
    from pytme_b200 import filters as F

    ctf = F.CTFReconstructed(defocus_x=20000.0)
    wedge = F.WedgeReconstructed(angles=(60, 60), opening_axis=2, tilt_axis=0)
    assert not F.needs_spectrum(ctf)
    assert not F.needs_spectrum(F.Compose([ctf, wedge]))
    assert F.needs_spectrum(F.LinearWhiteningFilter())
    assert F.needs_spectrum(F.Compose([wedge, F.LinearWhiteningFilter()]))


def test_download_host_tensor():
    """download() of a host tensor is a plain copy to NumPy."""
    import torch

    from pytme_b200.analyzer import download

    t = torch.arange(24, dtype=torch.float32).reshape(2, 3, 4)
    got = download(t)
    assert got.dtype == np.float32 and np.array_equal(got, t.numpy())


def test_split_shape_matches_reference(golden):
    """split_shape against the reference's slices (tests/golden/splits.npz)."""
    from pytme_b200.matching import split_shape
    from tests.golden.make_golden import SPLIT_CASES

    g = golden("splits.npz")
    for i, (shape, splits) in enumerate(SPLIT_CASES):
        for eq in (True, False):
            got = np.array([[(x.start, x.stop) for x in combo]
                            for combo in split_shape(shape, dict(splits), equal_shape=eq)],
                           dtype=np.int64)
            assert np.array_equal(got, g[f"case{i}_{int(eq)}"]), (shape, splits, eq)


def test_filter_bucket_matches_reference(golden):
    """The bucket rule peak calling uses above 1e5 candidate points, against the
    reference's _filter_bucket on random points with and without scores."""
    from pytme_b200.peaks import filter_bucket, filter_points_indices

    g = golden("splits.npz")
    for j in range(3):
        c, sc, md = g[f"bucket{j}_coords"], g[f"bucket{j}_scores"], int(g[f"bucket{j}_md"])
        assert np.array_equal(filter_bucket(c, md, sc), g[f"bucket{j}_idx"])
        assert np.array_equal(filter_bucket(c, md, None), g[f"bucket{j}_idx_noscore"])
        # the dispatch takes the bucket path above the cutoff
        assert np.array_equal(filter_points_indices(c, md, scores=sc, bucket_cutoff=len(c) - 1),
                              g[f"bucket{j}_idx"])


def test_reference_rotation_set_matches_golden(golden):
    """pytme_b200.rotations loads the reference's own quaternion set: the 30-degree set
    equals the rotations the reference's scan used for the config-1 goldens."""
    from pytme_b200 import rotations as R

    if R.quaternion_data_dir() is None:
        pytest.skip("the reference's quaternion data are not available")
    g = golden("c1_flcsm.npz")
    m = R.get_rotation_matrices(30).astype(np.float32)
    assert np.array_equal(m, g["rotations"])
    m7, desc = R.rotation_set(7.0)
    assert m7.shape == (27672, 3, 3) and "reference" in desc


def test_backend_pass_options():
    """Pass forms accepted by change_backend("b200", ...): every pass takes "auto", "fft"
    and "tensor"; the y pass also "tensor2" and "tensor-inplace"; anything else raises
    ValueError, as the reference's backends do for unknown options."""
    import importlib

    B = importlib.import_module("pytme_b200.backend")  # the module, not the manager
    try:
        for mode in ("auto", "fft", "tensor", "tensor2", "tensor-inplace"):
            B._set_options(ypass=mode)
            assert B.current_options()["ypass"] == mode
        for key in ("xpass", "zpass"):
            for mode in ("tensor2", "tensor-inplace"):
                with pytest.raises(ValueError):
                    B._set_options(**{key: mode})
        with pytest.raises(ValueError):
            B._set_options(ypass="inplace")
    finally:
        B._set_options()
    assert B.current_options()["ypass"] == "auto"
