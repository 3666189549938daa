"""GPU parity of the local-refinement kernels (score at one pose per peak and its
hand-written adjoint) against the FP64 oracle, the reference's FLC map, central finite
differences (h = 1e-3) and a plain PyTorch autograd composition.

Tolerances: scores within 1e-4 absolute (the scan's bound). Gradients: the kernels
sample with float32 coordinates and weights and sum in double, so they agree with the
float64 autograd composition to 1e-3 of the largest component; central differences of
the shift straddle kinks of the piecewise-linear interpolant for about 2h of the
samples and are held to 3e-2 of the largest shift component."""
import numpy as np
import pytest

from oracle import tm_oracle as O
from tests import refine_torch_ref as TR

pytestmark = pytest.mark.gpu

TOL = 1e-4
H = 1e-3


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _small_rotations(n, max_deg, rng):
    """Rotations by a uniform angle in [0, max_deg] about random axes."""
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    ang = np.deg2rad(rng.uniform(0, max_deg, n))
    k = np.zeros((n, 3, 3))
    k[:, 0, 1], k[:, 0, 2], k[:, 1, 2] = -axis[:, 2], axis[:, 1], -axis[:, 0]
    k = k - k.transpose(0, 2, 1)
    s, c = np.sin(ang)[:, None, None], np.cos(ang)[:, None, None]
    return np.eye(3) + s * k + (1 - c) * (k @ k)


def _wedge(t):
    from pytme_b200 import filters as F

    w = F.WedgeReconstructed(angles=(50, 50), opening_axis=2, tilt_axis=0,
                             create_continuous_wedge=True)
    return np.asarray(w(shape=(t, t, t), return_real_fourier=True, shape_is_real_fourier=False,
                        data_rfft=None, batch_dimension=None, weight_type=None)["data"],
                      np.float32)


def _case(filtered, t=12, shape=(40, 36, 30), n_copies=3, n_extra=5, seed=5):
    from pytme_b200 import refine as RF
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(seed)
    tm = syn.blob_template(t, rng, radius=t / 4, sigma=1.2)
    mk = syn.dilated_threshold_mask(tm, 0.1, 1)
    target, pos, rots = syn.make_tomogram(shape, tm, n_copies, rng, scale=1.0)
    filt = _wedge(t) if filtered else None
    pert = _small_rotations(n_copies, 5.0, rng) @ rots.astype(np.float64)
    ang = RF.euler_zyz_from_matrix(pert)
    # extra poses anywhere (partly outside the target) with arbitrary orientations
    extra_ang = np.stack([rng.uniform(-180, 180, n_extra), rng.uniform(5, 175, n_extra),
                          rng.uniform(-180, 180, n_extra)], -1)
    extra_cor = np.stack([rng.integers(-t // 2, n - t // 2, n_extra) for n in shape], -1)
    ang = np.concatenate([ang, extra_ang])
    cor = np.concatenate([pos, extra_cor]).astype(np.int64)
    sh = rng.uniform(-1.5, 1.5, (len(cor), 3))
    return target, tm, mk, filt, cor, ang, sh


def _oracle(target, tm, mk, filt, cor, ang, sh):
    return np.array([O.refine_flc_score(target.astype(np.float64), tm, mk, cor[i],
                                        O.euler_zyz_to_matrix(ang[i]), sh[i],
                                        template_filter=filt) for i in range(len(cor))])


def test_euler_kernel(torch_cuda):
    torch = torch_cuda
    from pytme_b200 import _native as N
    from pytme_b200 import refine as RF

    rng = np.random.default_rng(0)
    P = 300
    a = np.stack([rng.uniform(-180, 180, P), rng.uniform(0, 180, P),
                  rng.uniform(-180, 180, P)], -1).astype(np.float32)
    ang = torch.tensor(a, device="cuda")
    R = torch.empty((P, 9), device="cuda")
    dR = torch.empty((P, 27), device="cuda")
    N.check(N.lib.tm_euler_zyz(N.ptr(ang), P, N.ptr(R), N.ptr(dR), N.stream_ptr()))
    torch.cuda.synchronize()
    want = RF.euler_zyz_to_matrix(a.astype(np.float64)).reshape(P, 9)
    assert np.abs(R.cpu().numpy() - want).max() < 1e-6
    h = 1e-4
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        fd = (RF.euler_zyz_to_matrix(a + e) - RF.euler_zyz_to_matrix(a - e)) / (2 * h)
        got = dR.cpu().numpy()[:, 9 * k:9 * k + 9]
        assert np.abs(got - fd.reshape(P, 9)).max() < 1e-6


@pytest.mark.parametrize("filtered", [False, True])
def test_forward_matches_oracle(torch_cuda, filtered):
    from pytme_b200 import refine as RF

    target, tm, mk, filt, cor, ang, sh = _case(filtered)
    prob = RF.RefineProblem(target, tm, mk, template_filter=filt)
    got = RF.refine_score(prob, cor, ang, sh).detach().cpu().numpy()
    want = _oracle(target, tm, mk, filt, cor, ang, sh)
    assert np.abs(got - want).max() < TOL


def test_score_at_scan_pose_matches_reference_map(torch_cuda, golden):
    """At the scan's own pose (shift 0, rotation of the argmax) the refinement score of
    a score-map voxel is the reference's FP64 FLC map value there."""
    from pytme_b200 import refine as RF

    g = golden("flc_filt.npz")
    tgt, tmpl = g["target"], g["template"]
    t = np.asarray(tmpl.shape)
    rng = np.random.default_rng(0)
    xs = []
    while len(xs) < 60:
        x = tuple(int(rng.integers(t[i] // 2 + 1, tgt.shape[i] - t[i] // 2 - 1)) for i in range(3))
        if g["rot64"][x] >= 0:
            xs.append(x)
    xs = np.asarray(xs)
    rots = g["rotations"][g["rot64"][tuple(xs.T)].astype(np.int64)].astype(np.float64)
    prob = RF.RefineProblem(tgt, tmpl, g["mask"], template_filter=g["template_filter"],
                            target_filter=g["target_filter"])
    cor = RF.score_box_corner(xs, tgt.shape, tmpl.shape)
    got = RF.refine_score(prob, cor, RF.euler_zyz_from_matrix(rots)).detach().cpu().numpy()
    assert np.abs(got - g["scores64"][tuple(xs.T)]).max() < TOL


def _gpu_grads(torch, prob, cor, ang, sh, template=None):
    from pytme_b200 import refine as RF

    A = torch.tensor(ang, dtype=torch.float32, device="cuda", requires_grad=True)
    S = torch.tensor(sh, dtype=torch.float32, device="cuda", requires_grad=True)
    T = (prob.template if template is None else template).clone().requires_grad_(True)
    c = torch.tensor(cor, dtype=torch.int32, device="cuda")
    s = RF.FLCRefineFunction.apply(T, A, S, prob, c)
    w = torch.linspace(0.5, 1.5, s.shape[0], device="cuda")
    (s * w).sum().backward()
    return (s.detach().cpu().numpy(), A.grad.cpu().numpy().astype(np.float64),
            S.grad.cpu().numpy().astype(np.float64), T.grad.cpu().numpy().astype(np.float64))


@pytest.mark.parametrize("filtered,t", [(False, 12), (True, 12), (False, 40), (True, 40)])
def test_backward_matches_torch_autograd(torch_cuda, filtered, t):
    """t = 12 accumulates the template gradient in shared memory, t = 40 with global
    atomics."""
    torch = torch_cuda
    from pytme_b200 import refine as RF

    shape = (96, 90, 80) if t == 40 else (40, 36, 30)
    target, tm, mk, filt, cor, ang, sh = _case(filtered, t=t, shape=shape)
    prob = RF.RefineProblem(target, tm, mk, template_filter=filt)
    s, ga, gs, gt = _gpu_grads(torch, prob, cor, ang, sh)
    # the composition runs on the problem's (filtered) target with its mean restored
    A = torch.tensor(ang, dtype=torch.float64, device="cuda", requires_grad=True)
    S = torch.tensor(sh, dtype=torch.float64, device="cuda", requires_grad=True)
    T = torch.tensor(tm, dtype=torch.float64, device="cuda", requires_grad=True)
    ref = TR.flc_scores(prob.target.double() - prob.outside, T, prob.mask.double(),
                        torch.tensor(cor, device="cuda"), A, S,
                        None if filt is None else torch.tensor(filt, dtype=torch.float64,
                                                               device="cuda"))
    w = torch.linspace(0.5, 1.5, ref.shape[0], device="cuda", dtype=torch.float64)
    (ref * w).sum().backward()
    assert np.abs(s - ref.detach().cpu().numpy()).max() < TOL
    for got, want in ((ga, A.grad), (gs, S.grad), (gt, T.grad)):
        want = want.cpu().numpy()
        scale = np.abs(want).max()
        assert scale > 0
        assert np.abs(got - want).max() <= 1e-3 * scale


@pytest.mark.parametrize("filtered", [False, True])
def test_backward_matches_finite_differences(torch_cuda, filtered):
    torch = torch_cuda
    from pytme_b200 import refine as RF

    target, tm, mk, filt, cor, ang, sh = _case(filtered, n_extra=0)
    prob = RF.RefineProblem(target, tm, mk, template_filter=filt)
    _, ga, gs, gt = _gpu_grads(torch, prob, cor, ang, sh)
    w = np.linspace(0.5, 1.5, len(cor))
    tc = prob.target.double().cpu().numpy() - prob.outside

    def score(i, a, s, T=tm):
        return O.refine_flc_score(tc, T, mk, cor[i], O.euler_zyz_to_matrix(a), s,
                                  template_filter=filt)

    for i in range(len(cor)):
        for k in range(3):
            e = np.zeros(3)
            e[k] = H
            fa = w[i] * (score(i, ang[i] + e, sh[i]) - score(i, ang[i] - e, sh[i])) / (2 * H)
            fs = w[i] * (score(i, ang[i], sh[i] + e) - score(i, ang[i], sh[i] - e)) / (2 * H)
            assert abs(ga[i, k] - fa) <= 1e-3 * np.abs(ga[i]).max() + 1e-7
            assert abs(gs[i, k] - fs) <= 3e-2 * np.abs(gs[i]).max() + 1e-7
    for v in [(6, 6, 6), (5, 7, 6), (4, 6, 8), (7, 5, 5)]:
        fd = 0.0
        for i in range(len(cor)):
            tp = tm.astype(np.float64).copy()
            tp[v] += H
            tn = tm.astype(np.float64).copy()
            tn[v] -= H
            fd += w[i] * (score(i, ang[i], sh[i], tp) - score(i, ang[i], sh[i], tn)) / (2 * H)
        assert abs(gt[v] - fd) <= 1e-3 * np.abs(gt).max()


def test_chunked_problem_matches_single_chunk(torch_cuda):
    """Peaks split over several scratch chunks give the same scores and gradients."""
    torch = torch_cuda
    from pytme_b200 import refine as RF

    target, tm, mk, filt, cor, ang, sh = _case(True, n_copies=3, n_extra=9)
    one = RF.RefineProblem(target, tm, mk, template_filter=filt)
    many = RF.RefineProblem(target, tm, mk, template_filter=filt, max_work_bytes=5 * 30000)
    assert many.chunk < len(cor)
    a = _gpu_grads(torch, one, cor, ang, sh)
    b = _gpu_grads(torch, many, cor, ang, sh)
    for x, y in zip(a, b):
        assert np.abs(x - y).max() <= 1e-5 * max(np.abs(x).max(), 1e-12)


def test_refinement_recovers_perturbed_poses(torch_cuda):
    """Copies perturbed by up to 5 degrees and 1.5 voxels move back towards their true
    poses in 50 Adam steps, and no peak's score decreases. The copies are strong
    (amplitude 20 over unit noise): at low SNR the FLC maximum of a smooth blob
    template sits degrees away from the true orientation, fitted to the noise."""
    from pytme_b200 import refine as RF
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(11)
    t = 24
    tm = syn.blob_template(t, rng, n_blobs=10, radius=7.0, sigma=1.0)
    mk = syn.dilated_threshold_mask(tm, 0.1, 2)
    target, pos, rots = syn.make_tomogram((128, 128, 96), tm, 24, rng, scale=20.0)
    n = len(pos)
    true_r = rots.astype(np.float64)
    start_r = _small_rotations(n, 5.0, rng) @ true_r
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    sh0 = d * rng.uniform(0, 1.5, (n, 1))
    prob = RF.RefineProblem(target, tm, mk)
    res = RF.refine_peaks(prob, pos, RF.euler_zyz_from_matrix(start_r), sh0, steps=50)

    def ang_err(r):
        c = (np.trace(np.transpose(r, (0, 2, 1)) @ true_r, axis1=1, axis2=2) - 1) / 2
        return np.rad2deg(np.arccos(np.clip(c, -1, 1)))

    c = (t - 1) / 2
    true_pos = pos + c
    before_a, after_a = ang_err(start_r), ang_err(res.rotations)
    before_s = np.linalg.norm(sh0, axis=1)
    after_s = np.linalg.norm(res.positions - true_pos, axis=1)
    assert np.all(res.scores >= res.initial_scores - 1e-6)
    assert res.scores.mean() > res.initial_scores.mean() + 0.01
    assert np.median(after_a) < 0.5 * np.median(before_a)
    assert np.median(after_s) < 0.5 * np.median(before_s)


def test_refinement_config5_scale(torch_cuda):
    """2048 candidate peaks of a 256 x 256 x 128 tomogram (40 copies at SNR 0.1, the rest
    random poses), 32^3 template with a CTF x missing-wedge filter: 50 Adam steps keep
    every score finite and never below its start, and raise the copies' scores."""
    torch = torch_cuda
    from pytme_b200 import filters as F
    from pytme_b200 import refine as RF
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(2)
    t = 32
    tm = syn.blob_template(t, rng, n_blobs=8, radius=8.0, sigma=2.0)
    mk = syn.dilated_threshold_mask(tm, 0.1, 2)
    target, pos, rots = syn.make_tomogram((256, 256, 128), tm, 40, rng, snr=0.1, mask=mk)
    ctf = F.CTFReconstructed(defocus_x=30000.0, spherical_aberration=2.7e7,
                             amplitude_contrast=0.07, acceleration_voltage=300e3,
                             sampling_rate=6.8, flip_phase=True)
    wedge = F.WedgeReconstructed(angles=(60, 60), opening_axis=2, tilt_axis=0,
                                 create_continuous_wedge=True)
    comp = F.Compose([ctf, wedge])
    n_true, P = len(pos), 2048
    start_r = _small_rotations(n_true, 5.0, rng) @ rots.astype(np.float64)
    ang = np.concatenate([RF.euler_zyz_from_matrix(start_r),
                          np.stack([rng.uniform(-180, 180, P - n_true),
                                    rng.uniform(5, 175, P - n_true),
                                    rng.uniform(-180, 180, P - n_true)], -1)])
    cor = np.concatenate([pos, np.stack([rng.integers(0, n - t, P - n_true)
                                         for n in target.shape], -1)])
    sh = rng.uniform(-1.5, 1.5, (P, 3)) / np.sqrt(3)
    prob = RF.RefineProblem(target, tm, mk, template_filter=comp)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    res = RF.refine_peaks(prob, cor, ang, sh, steps=50)
    e1.record()
    torch.cuda.synchronize()
    print(f"refine 2048 peaks x 50 steps: {e0.elapsed_time(e1):.1f} ms")
    assert np.all(np.isfinite(res.scores))
    assert np.all(res.scores >= res.initial_scores - 1e-6)
    assert res.scores[:n_true].mean() > res.initial_scores[:n_true].mean()
