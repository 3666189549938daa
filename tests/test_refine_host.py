"""Local refinement, host side: Euler conversions, the box-corner mapping, and the plain
PyTorch autograd composition of the score checked against the FP64 oracle and against
central finite differences (h = 1e-3) of it. No GPU needed."""
import numpy as np
import pytest
import torch

from oracle import tm_oracle as O
from pytme_b200 import refine as RF
from pytme_b200 import synthetic as syn
from tests import refine_torch_ref as TR

H = 1e-3


def test_euler_zyz_matches_scipy_and_round_trips():
    from scipy.spatial.transform import Rotation

    rng = np.random.default_rng(0)
    a = np.stack([rng.uniform(-180, 180, 200), rng.uniform(0, 180, 200),
                  rng.uniform(-180, 180, 200)], -1)
    m = RF.euler_zyz_to_matrix(a)
    assert np.abs(m - Rotation.from_euler("zyz", a, degrees=True).as_matrix()).max() < 1e-12
    assert np.abs(m - O.euler_zyz_to_matrix(a)).max() < 1e-12
    r = Rotation.random(100, random_state=1).as_matrix()
    back = RF.euler_zyz_to_matrix(RF.euler_zyz_from_matrix(r))
    assert np.abs(back - r).max() < 1e-12
    # gimbal-locked inputs (b = 0 and b = 180)
    e = np.array([[30.0, 0.0, 20.0], [10.0, 180.0, 40.0]])
    me = RF.euler_zyz_to_matrix(e)
    assert np.abs(RF.euler_zyz_to_matrix(RF.euler_zyz_from_matrix(me)) - me).max() < 1e-12
    t = torch.tensor(a)
    assert np.abs(TR.euler_zyz(t).numpy() - m).max() < 1e-12


@pytest.mark.parametrize("shape,tshape", [((40, 36, 30), (12, 12, 12)),
                                          ((37, 33, 29), (10, 11, 9))])
def test_score_box_corner_matches_oracle(shape, tshape):
    rng = np.random.default_rng(1)
    pos = np.stack([rng.integers(0, n, 20) for n in shape], -1)
    assert np.array_equal(RF.score_box_corner(pos, shape, tshape),
                          O.score_box_corner(pos, shape, tshape))


def _problem(filtered: bool, seed: int = 5, t: int = 12):
    rng = np.random.default_rng(seed)
    tm = syn.blob_template(t, rng, radius=3.0, sigma=1.2)
    mk = syn.dilated_threshold_mask(tm, 0.1, 1)
    target, pos, rots = syn.make_tomogram((40, 36, 30), tm, 3, rng, scale=1.0)
    filt = None
    if filtered:
        from pytme_b200 import filters as F

        w = F.WedgeReconstructed(angles=(50, 50), opening_axis=2, tilt_axis=0,
                                 create_continuous_wedge=True)
        filt = np.asarray(w(shape=(t, t, t), return_real_fourier=True,
                            shape_is_real_fourier=False, data_rfft=None,
                            batch_dimension=None, weight_type=None)["data"], np.float64)
    ang = RF.euler_zyz_from_matrix(rots.astype(np.float64)) + rng.uniform(-3, 3, (3, 3))
    sh = rng.uniform(-1, 1, (3, 3))
    return target.astype(np.float64), tm, mk, filt, pos.astype(np.int64), ang, sh


@pytest.mark.parametrize("filtered", [False, True])
def test_torch_reference_matches_oracle_and_finite_differences(filtered):
    target, tm, mk, filt, cor, ang, sh = _problem(filtered)

    def oracle(i, a, s, T=tm):
        return O.refine_flc_score(target, T, mk, cor[i], O.euler_zyz_to_matrix(a), s,
                                  template_filter=filt)

    A = torch.tensor(ang, requires_grad=True)
    S = torch.tensor(sh, requires_grad=True)
    T = torch.tensor(tm, dtype=torch.float64, requires_grad=True)
    sc = TR.flc_scores(torch.tensor(target), T, torch.tensor(mk, dtype=torch.float64),
                       torch.tensor(cor), A, S, None if filt is None else torch.tensor(filt))
    want = np.array([oracle(i, ang[i], sh[i]) for i in range(len(cor))])
    assert np.abs(sc.detach().numpy() - want).max() < 1e-10
    sc.sum().backward()
    for i in range(len(cor)):
        for k in range(3):
            e = np.zeros(3)
            e[k] = H
            fd_a = (oracle(i, ang[i] + e, sh[i]) - oracle(i, ang[i] - e, sh[i])) / (2 * H)
            fd_s = (oracle(i, ang[i], sh[i] + e) - oracle(i, ang[i], sh[i] - e)) / (2 * H)
            # angle steps of 1e-3 degree move no sample across a trilinear kink
            assert abs(A.grad[i, k].item() - fd_a) <= 1e-6 * abs(fd_a) + 1e-9
            # a 1e-3 voxel shift moves every sample, and about 2h of them straddle a
            # kink of the piecewise-linear interpolant, so central differences differ
            # from the one-sided analytic derivative by O(h) relative
            gmax = np.abs(S.grad[i].numpy()).max()
            assert abs(S.grad[i, k].item() - fd_s) <= 3e-2 * gmax
    for v in [(6, 6, 6), (5, 7, 6), (4, 6, 8)]:
        fd = 0.0
        for i in range(len(cor)):
            tp = tm.astype(np.float64).copy()
            tp[v] += H
            tn = tm.astype(np.float64).copy()
            tn[v] -= H
            fd += (oracle(i, ang[i], sh[i], tp) - oracle(i, ang[i], sh[i], tn)) / (2 * H)
        assert abs(T.grad[v].item() - fd) <= 1e-6 * abs(fd) + 1e-9
