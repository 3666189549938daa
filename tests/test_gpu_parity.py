"""GPU parity: the CUDA path against the oracle and the reference's golden vectors.

Tolerances: scores within 1e-4 absolute of the reference FP32 map and of the FP64
map. Rotation indices must agree except at near-ties: with
both maps within 1e-4, a different argmax means two rotations score within 2e-4,
and such voxels must stay rare (<= 1e-4 of the map)."""
import numpy as np
import pytest

from oracle import tm_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4


def mixed_tol(ref_scores) -> float:
    """Error bound of the mixed-precision path: half2 storage of the product spectra
    (11-bit significands) gives absolute errors proportional to the RMS of the score
    map. Where the map is dominated by noise (the benchmark geometries) this is well
    below 1e-4; the FP32 path is always held to 1e-4."""
    return max(TOL, 2e-3 * float(np.sqrt(np.mean(np.square(ref_scores, dtype=np.float64)))))


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _scan(score, target, template, mask, rotations, precision="fp32", plain=False, batch=16,
          template_filter=None, target_filter=None, pad=False, splits=None, callback=None,
          callback_args=None, order=1, xpass="auto", zpass="auto", ypass="auto"):
    import pytme_b200 as P
    from pytme_b200.analyzer import MaxScoreOverRotations

    P.backend.change_backend("b200", precision=precision, rotation_batch=batch, plain=plain,
                             xpass=xpass, ypass=ypass, zpass=zpass)
    md = P.MatchingData(target.copy(), template.copy())
    if mask is not None:
        md.template_mask = mask.copy()
    md.rotations = rotations
    md.template_filter = template_filter
    md.target_filter = target_filter
    setup, scoring = P.MATCHING_EXHAUSTIVE_REGISTER[score]
    return P.scan_subsets(md, matching_score=scoring, matching_setup=setup,
                          callback_class=callback or MaxScoreOverRotations,
                          callback_class_args=callback_args or {"score_threshold": 0},
                          job_schedule=(1, 1), interpolation_order=order,
                          pad_target_edges=pad, target_splits=splits or {})


def _assert_argmax_ties(g, rot, score="FLCSphericalMask"):
    """Every voxel whose rotation index differs from the reference's is a documented
    tie: the oracle's score for the GPU's rotation there is within 2*TOL of the
    reference's best score (or, where the reference kept no rotation, the GPU's pick
    scores at most 2*TOL above the zero threshold)."""
    ref_rot = g["rot32"].astype(np.int32)
    mism = np.argwhere(rot != ref_rot)
    if len(mism) == 0:
        return
    picks = rot[tuple(mism.T)]
    best = g["scores32"][tuple(mism.T)]
    for j in np.unique(picks):
        sel = picks == j
        if j < 0:
            assert np.all(best[sel] <= 2 * TOL)
            continue
        r = O.scan(g["target"], g["template"], g["rotations"][j:j + 1], score,
                   template_mask=g["mask"], score_threshold=-np.inf)
        sj = r["scores"][tuple(mism[sel].T)]
        gap = best[sel] - sj
        assert np.all(gap <= 2 * TOL), (int(j), float(gap.max()))


@pytest.mark.parametrize("precision,plain", [("fp32", True), ("fp32", False), ("mixed", False)])
def test_flcsm_config1_matches_reference(torch_cuda, golden, precision, plain):
    g = golden("c1_flcsm.npz")
    r = _scan("FLCSphericalMask", g["target"], g["template"], g["mask"], g["rotations"],
              precision=precision, plain=plain)
    s, rot = r[0], r[2]
    assert s.shape == g["scores32"].shape
    err32 = np.abs(s - g["scores32"]).max()
    err64 = np.abs(s - g["scores64"]).max()
    assert err32 <= TOL, err32
    assert err64 <= TOL, err64
    _assert_argmax_ties(g, rot)
    # rotation mapping covers every rotation in order
    assert len(r[3]) == g["rotations"].shape[0]
    assert np.array_equal(r[3][5], g["rotations"][5])


def test_cc_matches_reference(torch_cuda, golden):
    g = golden("cc_small.npz")
    for plain in (True, False):
        r = _scan("CC", g["target"], g["template"], None, g["rotations"], plain=plain)
        # CC scores are raw correlations (order 10-100): relative tolerance
        scale = np.abs(g["scores32"]).max()
        assert np.abs(r[0] - g["scores32"]).max() <= TOL * scale
        assert np.count_nonzero(r[2] != g["rot32"]) <= 5


def test_flc_filtered_matches_reference(torch_cuda, golden):
    g = golden("flc_filt.npz")
    r = _scan("FLC", g["target"], g["template"], g["mask"], g["rotations"], plain=True,
              template_filter=g["template_filter"], target_filter=g["target_filter"])
    assert np.abs(r[0] - g["scores32"]).max() <= TOL
    assert np.abs(r[0] - g["scores64"]).max() <= TOL
    assert np.count_nonzero(r[2] != g["rot64"]) <= 5


@pytest.mark.parametrize("precision,plain", [("fp32", True), ("mixed", False)])
def test_dc_offset_tracks_fp64(torch_cuda, golden, precision, plain):
    g = golden("flcsm_dc.npz")
    r = _scan("FLCSphericalMask", g["target"], g["template"], g["mask"], g["rotations"],
              precision=precision, plain=plain)
    # FP64 denominator and a centred target keep the error far below the reference's
    # own FP32 error at this offset
    err64 = np.abs(r[0] - g["scores64"]).max()
    ref_err = np.abs(g["scores32"] - g["scores64"]).max()
    assert err64 <= TOL, err64
    assert err64 < ref_err


@pytest.mark.parametrize("score", ["CC", "FLC", "FLCSphericalMask"])
@pytest.mark.parametrize("pad", [False, True])
def test_reference_box_kat(torch_cuda, golden, score, pad):
    """tests/test_matching_exhaustive.py of the reference: exact peak [25, 17, 12]."""
    from pytme_b200.analyzer import PeakCallerSort

    g = golden("kat_exhaustive.npz")
    target = np.zeros((80, 80, 80))
    target[25:31, 22:28, 12:16] = 1
    template = np.zeros((41, 41, 35))
    template[20:26, 25:31, 17:21] = 1
    mask = np.ones_like(template)
    r = _scan(score, target, template, mask, np.eye(3, dtype=np.float32)[None], plain=True,
              pad=pad, splits={0: 2}, callback=PeakCallerSort, callback_args={})
    peak, sc = r[0][0], r[2][0]
    assert np.array_equal(peak, [25, 17, 12])
    assert np.array_equal(peak, g[f"{score}_{int(pad)}_peak"])
    assert abs(float(sc) - float(g[f"{score}_{int(pad)}_score"])) <= 1e-3 * max(1, abs(float(sc)))
    r = _scan(score, target, template, mask, np.eye(3, dtype=np.float32)[None], plain=True,
              pad=pad)
    m = r[0]
    assert tuple(m.shape) == tuple(g[f"{score}_{int(pad)}_shape"])
    assert tuple(np.unravel_index(np.argmax(m), m.shape)) == tuple(g[f"{score}_{int(pad)}_argmax"])


def test_rigid_transform_matches_reference(torch_cuda, golden):
    import pytme_b200 as P

    g = golden("rigid.npz")
    be = P.backend
    be.change_backend("b200")
    data = torch_cuda.as_tensor(g["data"], device="cuda")
    for i in range(g["rotations"].shape[0]):
        out, _ = be.rigid_transform(arr=data, rotation_matrix=torch_cuda.as_tensor(
            g["matrices"][i], device="cuda"), order=1, out=torch_cuda.zeros_like(data))
        np.testing.assert_allclose(out.cpu().numpy(), g["out"][i], rtol=0, atol=2e-6)
        big = torch_cuda.zeros((16, 16, 16), device="cuda")
        bigm = torch_cuda.zeros((16, 16, 16), device="cuda")
        o2, om = be.rigid_transform(arr=data, arr_mask=torch_cuda.as_tensor(g["mask"], device="cuda"),
                                    rotation_matrix=torch_cuda.as_tensor(g["rotations"][i], device="cuda"),
                                    out=big, out_mask=bigm, use_geometric_center=True, order=1)
        np.testing.assert_allclose(o2.cpu().numpy(), g["out_pad"][i][0], rtol=0, atol=2e-6)
        np.testing.assert_allclose(om.cpu().numpy(), g["out_pad"][i][1], rtol=0, atol=2e-6)


@pytest.mark.parametrize("n", [8, 16, 50, 64, 100, 128, 160, 200, 256, 320, 384, 512, 1000])
def test_line_fft_matches_numpy(torch_cuda, n):
    from pytme_b200 import _native as N

    lines = max(1, min(8, 4096 // n))
    rng = np.random.default_rng(n)
    x = (rng.normal(size=(lines, n)) + 1j * rng.normal(size=(lines, n))).astype(np.complex64)
    xt = torch_cuda.as_tensor(x, device="cuda")
    for d in (-1, 1):
        yt = torch_cuda.empty_like(xt)
        N.check(N.lib.tm_line_fft_test(N.ptr(xt), N.ptr(yt), n, lines, d, N.stream_ptr()))
        ref = np.fft.fft(x.astype(np.complex128), axis=1) if d < 0 else \
            np.fft.ifft(x.astype(np.complex128), axis=1) * n
        err = np.abs(yt.cpu().numpy() - ref).max() / np.abs(ref).max()
        assert err < 2e-6, (n, d, err)


def test_norm_scores_and_max_update(torch_cuda):
    import pytme_b200 as P

    be = P.backend
    be.change_backend("b200")
    rng = np.random.default_rng(3)
    n = 4099
    arr = rng.normal(size=n).astype(np.float32)
    e2 = rng.uniform(1, 3, size=n).astype(np.float32) * 50
    e1 = rng.normal(size=n).astype(np.float32) * 5
    out = torch_cuda.empty(n, device="cuda")
    be.norm_scores(torch_cuda.as_tensor(arr, device="cuda"), torch_cuda.as_tensor(e2, device="cuda"),
                   torch_cuda.as_tensor(e1, device="cuda"), 50.0, 1.1920929e-07, out)
    ref = O.norm_scores(arr.astype(np.float64), e2.astype(np.float64), e1.astype(np.float64), 50.0,
                        1.1920929e-07, np.empty(n))
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-6, atol=1e-7)
    mx = torch_cuda.zeros(n, device="cuda")
    rt = torch_cuda.full((n,), -1, dtype=torch_cuda.int32, device="cuda")
    s1 = torch_cuda.as_tensor(arr, device="cuda")
    be.max_score_over_rotations(s1, mx, rt, 3)
    be.max_score_over_rotations(s1, mx, rt, 4)  # equal scores keep the first index
    h = arr > 0
    assert np.array_equal(rt.cpu().numpy(), np.where(h, 3, -1))
    assert np.array_equal(mx.cpu().numpy(), np.where(h, arr, 0))


def test_peak_calling_matches_reference(torch_cuda, golden):
    import pytme_b200 as P
    from pytme_b200.analyzer import PeakCallerMaximumFilter

    g = golden("c1_flcsm.npz")
    pc = PeakCallerMaximumFilter(shape=g["scores32"].shape, num_peaks=int(g["peak_num"]),
                                 min_distance=int(g["peak_min_distance"]))
    state = pc.init_state()
    state = pc(state, scores=torch_cuda.as_tensor(g["scores32"], device="cuda"),
               rotation_matrix=np.eye(3, dtype=np.float32))
    assert np.array_equal(state[0], g["peak_pos"])
    assert np.array_equal(state[2], g["peak_scores"])


def test_greedy_filter_matches_reference(torch_cuda, golden):
    from pytme_b200.peaks import find_candidate_indices

    g = golden("candidates.npz")
    for i in range(4):
        idx = find_candidate_indices(g[f"coords{i}"], int(g[f"md{i}"]))
        assert np.array_equal(idx, g[f"idx{i}"])
    # beyond the shared-memory capacity the workspace path is used
    rng = np.random.default_rng(11)
    c = rng.integers(0, 400, size=(5000, 3)).astype(np.int64)
    assert np.array_equal(find_candidate_indices(c, 9), O.find_candidate_indices(c, 9))
    # a negative minimum distance keeps every point (floor(sqrt(d2)) <= md never holds)
    assert np.array_equal(find_candidate_indices(c, -3), O.find_candidate_indices(c, -3))
    assert np.array_equal(find_candidate_indices(c[:100], -3), np.arange(100))


def _filters_ctf_wedge(shape_t, shape_target):
    from pytme_b200.filters import Compose, CTFReconstructed, WedgeReconstructed

    wedge = WedgeReconstructed(angles=(60, 60), opening_axis=2, tilt_axis=0)
    wedge_t = WedgeReconstructed(angles=(60, 60), opening_axis=2, tilt_axis=0)
    ctf = CTFReconstructed(defocus_x=30000, amplitude_contrast=0.07, spherical_aberration=2.7e7,
                           acceleration_voltage=300e3, sampling_rate=6.8)
    tf = Compose([wedge, ctf])(shape=shape_t, return_real_fourier=True)["data"]
    gf = Compose([wedge_t])(shape=shape_target, return_real_fourier=True)["data"]
    return tf, gf


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_flc_fused_matches_oracle(torch_cuda, precision):
    """Fused FLC (rotated mask, CTF x wedge template filter, wedge target filter) on
    power-of-two x/y lengths against the oracle in FP32 and FP64."""
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(21)
    tmpl = syn.blob_template(12, rng, radius=3.5, sigma=1.2)
    mask = syn.dilated_threshold_mask(tmpl, 0.1, 1)
    target, _, _ = syn.make_tomogram((64, 64, 48), tmpl, 4, rng, snr=0.5, mask=mask)
    rots = syn.random_rotation_matrices(20, rng)
    tf, gf = _filters_ctf_wedge(tmpl.shape, target.shape)
    r = _scan("FLC", target, tmpl, mask, rots, precision=precision, batch=8,
              template_filter=tf, target_filter=gf)
    ref = O.scan(target, tmpl, rots, "FLC", template_mask=mask, template_filter=tf,
                 target_filter=gf)
    ref64 = O.scan(target, tmpl, rots, "FLC", template_mask=mask, template_filter=tf,
                   target_filter=gf, dtype=np.float64)
    tol = TOL if precision == "fp32" else mixed_tol(ref64["scores"])
    assert np.abs(r[0] - ref["scores"]).max() <= tol
    assert np.abs(r[0] - ref64["scores"]).max() <= tol
    assert np.count_nonzero(r[2] != ref64["rotations"]) <= int(2e-3 * r[2].size)


def test_flc_config2_shape(torch_cuda):
    """Config-2 geometry (256x256x128 target, 32^3 template, FLC with CTF x wedge) on a
    few rotations: fused mixed precision within 1e-4 of the FP32 oracle."""
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(22)
    tmpl = syn.blob_template(32, rng, sigma=3.0, radius=10.0)
    mask = syn.dilated_threshold_mask(tmpl, 0.1, 2)
    target, _, _ = syn.make_tomogram((256, 256, 128), tmpl, 40, rng, snr=0.1, mask=mask)
    rots = syn.random_rotation_matrices(3, rng)
    tf, gf = _filters_ctf_wedge(tmpl.shape, target.shape)
    r = _scan("FLC", target, tmpl, mask, rots, precision="mixed", batch=4,
              template_filter=tf, target_filter=gf)
    ref = O.scan(target, tmpl, rots, "FLC", template_mask=mask, template_filter=tf,
                 target_filter=gf)
    assert np.abs(r[0] - ref["scores"]).max() <= TOL


def test_flcsm_config3_shape(torch_cuda):
    """The headline geometry (512x512x200 target, 48^3 template, spherical mask) on two
    rotations: fused mixed precision within 1e-4 of the FP32 oracle."""
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(23)
    tmpl = syn.blob_template(48, rng, sigma=4.5, radius=15.0)
    mask = syn.spherical_mask((48,) * 3, 24, center=(23.5,) * 3)
    target = rng.normal(size=(512, 512, 200)).astype(np.float32)
    rots = syn.random_rotation_matrices(2, rng)
    r = _scan("FLCSphericalMask", target, tmpl, mask, rots, precision="mixed", batch=2)
    ref = O.scan(target, tmpl, rots, "FLCSphericalMask", template_mask=mask)
    assert np.abs(r[0] - ref["scores"]).max() <= TOL


@pytest.mark.parametrize("n2", [64, 100, 128, 160, 199, 200, 256, 400, 512])
@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_zpass_lengths(torch_cuda, n2, precision):
    """Every z-axis length with a dedicated c2r kernel (and the generic fallback for the
    others) against the FP32 oracle on a small FLCSphericalMask scan."""
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(n2)
    tmpl = syn.blob_template(8, rng, radius=2.0, sigma=1.0)
    mask = syn.spherical_mask((8,) * 3, 4, center=(3.5,) * 3)
    target, _, _ = syn.make_tomogram((32, 32, n2), tmpl, 3, rng, scale=0.5)
    rots = syn.random_rotation_matrices(6, rng)
    r = _scan("FLCSphericalMask", target, tmpl, mask, rots, precision=precision, batch=4)
    ref = O.scan(target, tmpl, rots, "FLCSphericalMask", template_mask=mask)
    tol = TOL if precision == "fp32" else mixed_tol(ref["scores"])
    assert np.abs(r[0] - ref["scores"]).max() <= tol


@pytest.mark.parametrize("shape", [(128, 128, 24), (256, 64, 24), (64, 256, 20), (1024, 128, 16)])
def test_xy_lengths(torch_cuda, shape):
    """Register-resident column kernels for every power-of-two x/y length (and mixed
    x/y) against the FP32 oracle."""
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(sum(shape))
    tmpl = syn.blob_template(8, rng, radius=2.0, sigma=1.0)
    mask = syn.spherical_mask((8,) * 3, 4, center=(3.5,) * 3)
    target, _, _ = syn.make_tomogram(shape, tmpl, 3, rng, scale=0.5)
    rots = syn.random_rotation_matrices(5, rng)
    r = _scan("FLCSphericalMask", target, tmpl, mask, rots, precision="fp32", batch=3)
    ref = O.scan(target, tmpl, rots, "FLCSphericalMask", template_mask=mask)
    assert np.abs(r[0] - ref["scores"]).max() <= TOL


def test_scan_batch_uneven_jobs_and_graph_replay(torch_cuda, tmp_path, monkeypatch):
    """Uneven (tomogram, template) jobs through scan_batch with per-job CTF x wedge
    filters, autotuned batch and CUDA-graph replay, against per-job oracle scans; graph
    replay must give bit-identical maps to direct launches."""
    from pytme_b200 import synthetic as syn
    from pytme_b200.batch import MatchJob, scan_batch
    from pytme_b200.filters import Compose, CTFReconstructed, WedgeReconstructed

    monkeypatch.setenv("PYTME_B200_CACHE", str(tmp_path / "autotune.json"))
    rng = np.random.default_rng(31)
    jobs = []
    for shape, t, defocus, wedge in (((64, 64, 48), 12, 15000, 50), ((32, 64, 40), 8, 30000, 60),
                                     ((64, 64, 48), 12, 45000, 65)):
        tmpl = syn.blob_template(t, rng, radius=t / 4, sigma=1.2)
        mask = syn.spherical_mask((t,) * 3, t / 2, center=((t - 1) / 2,) * 3)
        target, _, _ = syn.make_tomogram(shape, tmpl, 3, rng, scale=0.5)
        w = WedgeReconstructed(angles=(wedge, wedge), opening_axis=2, tilt_axis=0)
        ctf = CTFReconstructed(defocus_x=defocus, sampling_rate=6.8)
        tf = Compose([w, ctf])(shape=tmpl.shape, return_real_fourier=True)["data"]
        jobs.append(MatchJob(target=target, template=tmpl, mask=mask,
                             rotations=syn.random_rotation_matrices(20, rng),
                             template_filter=tf))
    res = scan_batch(jobs, precision="fp32", rotation_batch="auto", use_graph=True)
    direct = scan_batch(jobs, precision="fp32", rotation_batch=8, use_graph=False)
    graph8 = scan_batch(jobs, precision="fp32", rotation_batch=8, use_graph=True)
    for job, (s, r), (s2, r2), (s3, r3) in zip(jobs, res, direct, graph8):
        ref = O.scan(job.target, job.template, job.rotations, "FLCSphericalMask",
                     template_mask=job.mask, template_filter=job.template_filter,
                     interpolation_order=job.interpolation_order)
        assert np.abs(s - ref["scores"]).max() <= TOL
        assert np.array_equal(s2, s3) and np.array_equal(r2, r3)


def test_cubic_rigid_transform_matches_reference(torch_cuda, golden):
    """Backend rigid_transform with order 3 (prefiltered data, unfiltered mask) against
    the reference's own output."""
    import pytme_b200 as P

    g = golden("cubic.npz")
    be = P.backend
    be.change_backend("b200")
    out = torch_cuda.zeros((16, 16, 16), device="cuda")
    outm = torch_cuda.zeros((16, 16, 16), device="cuda")
    o, om = be.rigid_transform(arr=g["rigid_data"], arr_mask=g["rigid_mask"],
                               rotation_matrix=g["rotations"][0], out=out, out_mask=outm,
                               use_geometric_center=True, order=3)
    assert np.abs(o.cpu().numpy() - g["rigid_out"]).max() < 1e-5
    assert np.abs(om.cpu().numpy() - g["rigid_out_mask"]).max() < 1e-5


@pytest.mark.parametrize("score", ["FLCSphericalMask", "FLC", "CC"])
@pytest.mark.parametrize("precision,plain", [("fp32", True), ("fp32", False), ("mixed", False)])
def test_cubic_scan_matches_reference(torch_cuda, golden, score, precision, plain):
    """interpolation_order=3, the reference's default, through scan_subsets."""
    g = golden("cubic.npz")
    mask = {"FLCSphericalMask": g["smask"], "FLC": g["mask"], "CC": None}[score]
    res = _scan(score, g["target"], g["template"], mask, g["rotations"], precision=precision,
                plain=plain, batch=8, order=3)
    scores, rot = np.asarray(res[0]), np.asarray(res[2])
    ref32, ref64 = g[f"{score}_scores32"], g[f"{score}_scores64"]
    # CC maps are not normalised: the bound is relative to the map's scale there
    scale = max(1.0, float(np.abs(ref64).max())) if score == "CC" else 1.0
    tol = TOL * scale if precision == "fp32" else max(TOL * scale, mixed_tol(ref32))
    assert np.abs(scores - ref32).max() <= tol
    assert np.abs(scores - ref64).max() <= tol
    mism = np.argwhere(rot != g[f"{score}_rot32"].astype(np.int32))
    assert len(mism) <= max(1, int(1e-3 * rot.size))


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_tensor_core_xpass_matches_reference(torch_cuda, golden, precision):
    """The tensor-core x pass in the fused FLCSphericalMask scan (config 1) against the
    reference's FP32 and FP64 maps, with the same bounds as the FFT x pass."""
    g = golden("c1_flcsm.npz")
    res = _scan("FLCSphericalMask", g["target"], g["template"], g["mask"], g["rotations"],
                precision=precision, batch=32, xpass="tensor")
    scores, rot = np.asarray(res[0]), np.asarray(res[2])
    tol = TOL if precision == "fp32" else mixed_tol(g["scores32"])
    assert np.abs(scores - g["scores32"]).max() <= tol
    assert np.abs(scores - g["scores64"]).max() <= tol
    _assert_argmax_ties(g, rot)


def test_tensor_core_xpass_cc_and_dc_offset(torch_cuda, golden):
    g = golden("cc_small.npz")
    res = _scan("CC", g["target"], g["template"], None, g["rotations"], batch=16,
                xpass="tensor")
    scale = max(1.0, float(np.abs(g["scores32"]).max()))
    assert np.abs(np.asarray(res[0]) - g["scores32"]).max() <= TOL * scale
    g = golden("flcsm_dc.npz")
    res = _scan("FLCSphericalMask", g["target"], g["template"], g["mask"], g["rotations"],
                batch=16, xpass="tensor")
    assert np.abs(np.asarray(res[0]) - g["scores64"]).max() <= TOL


@pytest.mark.parametrize("xpass,zpass", [("tensor", "tensor"), ("fft", "tensor"),
                                         ("tensor", "fft")])
def test_tensor_core_passes_mixed(torch_cuda, golden, xpass, zpass):
    """Every combination of tensor-core and FFT x / z passes in the mixed-precision
    FLCSphericalMask scan (config 1) against the reference's maps."""
    g = golden("c1_flcsm.npz")
    res = _scan("FLCSphericalMask", g["target"], g["template"], g["mask"], g["rotations"],
                precision="mixed", batch=32, xpass=xpass, zpass=zpass)
    scores, rot = np.asarray(res[0]), np.asarray(res[2])
    tol = mixed_tol(g["scores32"])
    assert np.abs(scores - g["scores32"]).max() <= tol
    assert np.abs(scores - g["scores64"]).max() <= tol
    _assert_argmax_ties(g, rot)


@pytest.mark.parametrize("shape,dtype", [((173, 211, 97), "float32"), ((300, 301, 89), "int32"),
                                         ((5, 7), "float32")])
def test_state_download_matches_cpu_copy(torch_cuda, shape, dtype):
    """The chunked download through pinned staging (used for the analyzer's result) is
    byte-identical to a plain device-to-host copy, for sizes that are not a multiple of
    the chunk, twice in a row (the staging buffer is reused)."""
    import torch
    from pytme_b200.analyzer import download

    for seed in (0, 1):
        g = torch.Generator(device="cuda").manual_seed(seed)
        if dtype == "float32":
            t = torch.randn(shape, generator=g, device="cuda")
        else:
            t = torch.randint(-2**31, 2**31 - 1, shape, generator=g, device="cuda",
                              dtype=torch.int32)
        got = download(t)
        want = t.cpu().numpy()
        assert got.shape == want.shape and got.dtype == want.dtype
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8))


@pytest.mark.parametrize("score", ["FLCSphericalMask", "FLC"])
def test_whitening_filters_in_scan(torch_cuda, score):
    """Whitening by the target's power spectrum as the target filter, and whitening x CTF
    x wedge as the template filter, passed to the scan as filter objects: the scan builds
    them on the device from the spectrum of the padded target, as the reference hands
    data_rfft to every filter (tme/matching_exhaustive.py:84-90). The oracle gets the
    arrays of the host restatement (pinned to the reference's whitening arrays) from a
    NumPy spectrum of the same target."""
    from pytme_b200 import synthetic as syn
    from pytme_b200.filters import (Compose, CTFReconstructed, LinearWhiteningFilter,
                                    WedgeReconstructed)

    rng = np.random.default_rng(37)
    tmpl = syn.blob_template(10, rng, radius=3.0, sigma=1.1)
    mask = syn.spherical_mask((10,) * 3, 5, center=(4.5,) * 3)
    target, _, _ = syn.make_tomogram((48, 40, 32), tmpl, 4, rng, snr=0.5, mask=mask)
    rots = syn.random_rotation_matrices(9, rng)
    ctf = CTFReconstructed(defocus_x=25000, sampling_rate=6.8)
    wedge = WedgeReconstructed(angles=(60, 60), opening_axis=2, tilt_axis=0,
                               create_continuous_wedge=True)
    tfilt = Compose([LinearWhiteningFilter(), ctf, wedge])
    gfilt = Compose([LinearWhiteningFilter()])
    r = _scan(score, target, tmpl, mask, rots, precision="fp32", batch=4,
              template_filter=tfilt, target_filter=gfilt)
    spec = np.fft.rfftn(target).astype(np.complex64)  # fast shape = target shape here
    tf = tfilt(shape=tmpl.shape, return_real_fourier=True, data_rfft=spec)["data"]
    gf = gfilt(shape=target.shape, return_real_fourier=True, data_rfft=spec)["data"]
    ref = O.scan(target, tmpl, rots, score, template_mask=mask,
                 template_filter=np.asarray(tf, np.float32),
                 target_filter=np.asarray(gf, np.float32))
    assert np.abs(r[0] - ref["scores"]).max() <= TOL


@pytest.mark.parametrize("score", ["FLCSphericalMask", "CC"])
def test_default_passes_odd_z_length(torch_cuda, score):
    """The default mixed-precision passes (persistent tensor-core x pass, register y pass,
    even/odd tensor-core z pass) on an odd z length, with a partial last launch group,
    against the oracle in FP32 and FP64."""
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(41)
    tmpl = syn.blob_template(12, rng, radius=3.5, sigma=1.2)
    mask = syn.spherical_mask((12,) * 3, 6, center=(5.5,) * 3) if score != "CC" else None
    target, _, _ = syn.make_tomogram((128, 64, 199), tmpl, 5, rng, scale=0.5)
    rots = syn.random_rotation_matrices(40, rng)
    r = _scan(score, target, tmpl, mask, rots, precision="mixed", batch=32)
    ref = O.scan(target, tmpl, rots, score, template_mask=mask)
    ref64 = O.scan(target, tmpl, rots, score, template_mask=mask, dtype=np.float64)
    tol = mixed_tol(ref64["scores"])
    assert np.abs(r[0] - ref["scores"]).max() <= tol
    assert np.abs(r[0] - ref64["scores"]).max() <= tol


@pytest.mark.parametrize("shape,score", [((128, 512, 40), "FLCSphericalMask"),
                                         ((48, 256, 33), "FLCSphericalMask"),
                                         ((128, 256, 24), "CC")])
def test_tensor_core_ypass(torch_cuda, shape, score):
    """The tensor-core y pass (radix-16 and radix-n1/16 FP16 GEMM stages with twiddles
    between them; "tensor": the radix-16 stage in FP32 registers, "tensor2": both stages on
    the tensor cores) for both supported y lengths, with a partial last launch
    group, against the oracle in FP32 and FP64 and against the CUDA-core y pass. The
    shapes with n0 = 128 run it behind the warp-specialised tensor-core x pass, as the
    default mixed-precision plans do: the x pass then writes the spectra x'-inner for it
    ("tensor"), which must give the same maps bit for bit as the in-place form on
    row-major spectra ("tensor-inplace")."""
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(sum(shape))
    tmpl = syn.blob_template(12, rng, radius=3.5, sigma=1.2)
    mask = syn.spherical_mask((12,) * 3, 6, center=(5.5,) * 3) if score != "CC" else None
    target, _, _ = syn.make_tomogram(shape, tmpl, 4, rng, scale=0.5)
    rots = syn.random_rotation_matrices(37, rng)
    r = _scan(score, target, tmpl, mask, rots, precision="mixed", batch=32, ypass="tensor")
    ip = _scan(score, target, tmpl, mask, rots, precision="mixed", batch=32,
               ypass="tensor-inplace")
    assert np.array_equal(r[0], ip[0]) and np.array_equal(r[2], ip[2])
    # behind the x'-inner hand-over the FFT z pass reads the y pass's second buffer
    # (interleaved rows) as it reads H otherwise
    zf = None
    if shape[0] % 128 == 0 and score == "FLCSphericalMask":
        zf = _scan(score, target, tmpl, mask, rots, precision="mixed", batch=32,
                   ypass="tensor", zpass="fft")
    c = _scan(score, target, tmpl, mask, rots, precision="mixed", batch=32, ypass="tensor2")
    f = _scan(score, target, tmpl, mask, rots, precision="mixed", batch=32, ypass="fft")
    ref = O.scan(target, tmpl, rots, score, template_mask=mask)
    ref64 = O.scan(target, tmpl, rots, score, template_mask=mask, dtype=np.float64)
    scale = max(1.0, float(np.abs(ref64["scores"]).max())) if score == "CC" else 1.0
    tol = max(TOL * scale, mixed_tol(ref64["scores"]))
    assert np.abs(r[0] - ref["scores"]).max() <= tol
    assert np.abs(r[0] - ref64["scores"]).max() <= tol
    assert np.abs(r[0] - f[0]).max() <= tol
    if zf is not None:
        assert np.abs(zf[0] - ref64["scores"]).max() <= tol
    assert np.abs(c[0] - ref64["scores"]).max() <= tol
    assert np.abs(c[0] - f[0]).max() <= tol
    # a blob template makes many rotations score alike: every voxel whose rotation differs
    # from the FP64 oracle's must be a tie within the path's error bound
    for rot in (r[2], c[2], f[2]):
        mism = np.argwhere(rot != ref64["rotations"])
        print(f"{shape} {score}: {len(mism)} argmax differences of {rot.size}")
        assert len(mism) <= 0.02 * rot.size
        if len(mism) == 0:
            continue
        probe = O.scan_parallel(target, tmpl, rots, score, template_mask=mask,
                                dtype=np.float64, n_workers=4, score_threshold=-np.inf,
                                probe=mism)["probe"]
        best = ref64["scores"][tuple(mism.T)]
        picks = rot[tuple(mism.T)]
        gaps = np.where(picks < 0, best, best - probe[np.maximum(picks, 0), np.arange(len(mism))])
        assert gaps.max() <= 2 * tol, float(gaps.max())
