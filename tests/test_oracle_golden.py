"""Pin the CPU oracle against golden vectors produced by running the reference itself
(tests/golden/make_golden.py). These run without a GPU."""
import numpy as np
import pytest

from oracle import tm_oracle as O


def test_flcsm_config1_fp32_bit_exact(golden):
    g = golden("c1_flcsm.npz")
    r = O.scan(g["target"], g["template"], g["rotations"], "FLCSphericalMask",
               template_mask=g["mask"])
    assert r["scores"].shape == g["scores32"].shape
    assert np.array_equal(r["scores"], g["scores32"])
    assert np.array_equal(r["rotations"], g["rot32"].astype(np.int32))


def test_flcsm_config1_fp64(golden):
    g = golden("c1_flcsm.npz")
    r = O.scan(g["target"], g["template"], g["rotations"], "FLCSphericalMask",
               template_mask=g["mask"], dtype=np.float64)
    # the fixture stores the FP64 map rounded to float32
    assert np.abs(r["scores"] - g["scores64"]).max() < 1e-7
    assert np.array_equal(r["rotations"], g["rot64"].astype(np.int32))


def test_peak_caller_maximum_filter(golden):
    g = golden("c1_flcsm.npz")
    pos, sc = O.peak_caller_maximum_filter(g["scores32"], int(g["peak_num"]),
                                           int(g["peak_min_distance"]))
    assert np.array_equal(pos, g["peak_pos"])
    assert np.array_equal(sc, g["peak_scores"])


@pytest.mark.parametrize("dtype,tag,tol", [(np.float32, "32", 0.0), (np.float64, "64", 1e-7)])
def test_flc_filtered(golden, dtype, tag, tol):
    g = golden("flc_filt.npz")
    r = O.scan(g["target"], g["template"], g["rotations"], "FLC", template_mask=g["mask"],
               template_filter=g["template_filter"], target_filter=g["target_filter"],
               dtype=dtype)
    assert np.abs(r["scores"] - g["scores" + tag]).max() <= tol
    assert np.array_equal(r["rotations"], g["rot" + tag].astype(np.int32))


def test_cc(golden):
    g = golden("cc_small.npz")
    r = O.scan(g["target"], g["template"], g["rotations"], "CC")
    assert np.array_equal(r["scores"], g["scores32"])
    assert np.array_equal(r["rotations"], g["rot32"].astype(np.int32))


def test_dc_offset_fp32(golden):
    g = golden("flcsm_dc.npz")
    r = O.scan(g["target"], g["template"], g["rotations"], "FLCSphericalMask",
               template_mask=g["mask"])
    assert np.array_equal(r["scores"], g["scores32"])
    # the reference's own FP32 path loses digits to E[x^2] - E[x]^2 at a +100 offset
    assert np.abs(g["scores32"] - g["scores64"]).max() > 1e-4


def test_find_candidate_indices(golden):
    g = golden("candidates.npz")
    for i in range(4):
        idx = O.find_candidate_indices(g[f"coords{i}"], int(g[f"md{i}"]))
        assert np.array_equal(idx, g[f"idx{i}"])


def test_rigid_transform(golden):
    g = golden("rigid.npz")
    data = g["data"]
    c = np.divide(np.asarray(data.shape) - 1, 2)
    for i, R in enumerate(g["rotations"]):
        m = O.rigid_transform_matrix(R, c)
        assert np.array_equal(m, g["matrices"][i])
        out = np.zeros_like(data)
        O.rotate_order1(data, m, out)
        assert np.array_equal(out, g["out"][i])


def test_kat_box_case_fp32(golden):
    g = golden("kat_exhaustive.npz")
    target = np.zeros((80, 80, 80))
    target[25:31, 22:28, 12:16] = 1
    template = np.zeros((41, 41, 35))
    template[20:26, 25:31, 17:21] = 1
    for score in ("CC", "FLCSphericalMask"):
        r = O.scan(target, template, np.eye(3)[None], score, template_mask=np.ones_like(template))
        m = r["scores"]
        assert tuple(np.unravel_index(np.argmax(m), m.shape)) == tuple(g[f"{score}_0_argmax"])
        assert abs(float(m.max()) - float(g[f"{score}_0_max"])) < 1e-5


def test_refine_score_matches_reference_flc_map(golden):
    """The real-space refinement score at the scan's own pose reproduces the reference's
    FP64 FLC map (filtered, arbitrary mask) at interior score-map voxels."""
    g = golden("flc_filt.npz")
    tgt, tmpl, mask = g["target"], g["template"], g["mask"]
    _, fast, _, _ = O.fourier_padding(tgt.shape, tmpl.shape)
    tg = O.apply_target_filter(tgt.astype(np.float64), fast,
                               g["target_filter"].astype(np.float64))
    t = np.asarray(tmpl.shape)
    rng = np.random.default_rng(0)
    checked = 0
    for _ in range(40):
        x = np.array([rng.integers(t[i] // 2 + 1, tgt.shape[i] - t[i] // 2 - 1)
                      for i in range(3)])
        r = int(g["rot64"][tuple(x)])
        if r < 0:
            continue
        k = O.score_box_corner(x, tgt.shape, tmpl.shape)
        s = O.refine_flc_score(tg, tmpl, mask, k, g["rotations"][r].astype(np.float64),
                               template_filter=g["template_filter"])
        assert abs(s - float(g["scores64"][tuple(x)])) < 1e-6
        checked += 1
    assert checked >= 20


@pytest.mark.parametrize("score", ["FLCSphericalMask", "FLC", "CC"])
def test_cubic_scan(golden, score):
    """interpolation_order=3 (the reference's default): prefiltered cubic B-spline
    rotation of the template, unprefiltered of the mask."""
    g = golden("cubic.npz")
    mask = {"FLCSphericalMask": g["smask"], "FLC": g["mask"], "CC": None}[score]
    r = O.scan(g["target"], g["template"], g["rotations"], score, template_mask=mask,
               interpolation_order=3)
    assert np.array_equal(r["scores"], g[f"{score}_scores32"])
    assert np.array_equal(r["rotations"], g[f"{score}_rot32"].astype(np.int32))
    r = O.scan(g["target"], g["template"], g["rotations"], score, template_mask=mask,
               interpolation_order=3, dtype=np.float64)
    # the fixture stores the FP64 map rounded to float32 (CC maps are not normalised)
    ref64 = g[f"{score}_scores64"]
    assert np.abs(r["scores"] - ref64).max() < 1e-7 * max(1.0, float(np.abs(ref64).max()))


def test_cubic_rigid_transform(golden):
    g = golden("cubic.npz")
    data, mask = g["rigid_data"], g["rigid_mask"]
    m = O.rigid_transform_matrix(g["rotations"][0], (np.asarray(data.shape) - 1) / 2)
    out = np.zeros((16, 16, 16), np.float32)
    outm = np.zeros((16, 16, 16), np.float32)
    O.rotate(data, m, out, order=3, prefilter=True)
    O.rotate(mask, m, outm, order=3, prefilter=False)
    assert np.array_equal(out, g["rigid_out"])
    assert np.array_equal(outm, g["rigid_out_mask"])
