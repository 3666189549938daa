"""The drop-in boundary exercised by the reference's own driver.

tme's unchanged ``scan_subsets`` (tme/matching_exhaustive.py:298-465) runs with the
backend ``"b200"`` selected through ``be.change_backend`` and the ``*_b200`` scores from
its own registry, with its own ``MaxScoreOverRotations`` behind its own
``SharedAnalyzerProxy`` (tme/analyzer/proxy.py:92-123). The maps must match the
reference's golden maps, and the rotation chunk must run fused: one ``tm_scan_run`` per
chunk, not one per rotation. The reference's backend test suite
(tests/test_backends.py of pyTME) then runs with the B200 backend in its
``BACKENDS_TO_TEST``.

The reference package comes from ``baseline/_ref`` (``python oracle/build_ref.py
--baseline`` installs it there from a reference checkout), with its missing third-party
imports provided by ``tests/golden/refshim``; the tests skip when it is absent.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import tm_oracle as O
from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

TOL = 1e-4
SHIM = os.path.join(ROOT, "tests", "golden", "refshim")
REF_INSTALL = os.environ.get("PYTME_REFERENCE_INSTALL", os.path.join(ROOT, "baseline", "_ref"))


@pytest.fixture(scope="module")
def tme_b200():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.isdir(os.path.join(REF_INSTALL, "tme")):
        pytest.skip("reference package not installed in baseline/_ref")
    if SHIM not in sys.path:
        sys.path.insert(0, SHIM)
    if REF_INSTALL not in sys.path:
        sys.path.append(REF_INSTALL)
    import tme  # noqa: F401
    from tme.backends import backend as tme_be

    from pytme_b200.tme_plugin import register

    assert register(strict=True)
    yield tme_be
    tme_be.change_backend("numpyfftw")


@pytest.fixture
def run_counter(monkeypatch):
    """Counts tm_scan_run calls and the rotations each one scores."""
    from pytme_b200 import scores

    calls = []
    orig = scores.ScanPlan.run

    def run(self, matrices, first_index, max_scores, argmax, stream=None):
        calls.append(int(matrices.shape[0]))
        return orig(self, matrices, first_index, max_scores, argmax, stream)

    monkeypatch.setattr(scores.ScanPlan, "run", run)
    return calls


def _tme_scan(score, target, template, mask, rotations, template_filter=None,
              target_filter=None):
    from tme.analyzer import MaxScoreOverRotations
    from tme.matching_data import MatchingData
    from tme.matching_exhaustive import scan_subsets
    from tme.matching_scores import MATCHING_EXHAUSTIVE_REGISTER

    md = MatchingData(target.copy(), template.copy())
    if mask is not None:
        md.template_mask = mask.copy()
    md.rotations = rotations
    if template_filter is not None:
        md.template_filter = template_filter
    if target_filter is not None:
        md.target_filter = target_filter
    setup, scoring = MATCHING_EXHAUSTIVE_REGISTER[f"{score}_b200"]
    return scan_subsets(md, matching_score=scoring, matching_setup=setup,
                        callback_class=MaxScoreOverRotations,
                        callback_class_args={"score_threshold": 0}, job_schedule=(1, 1),
                        interpolation_order=1, pad_target_edges=False,
                        pad_template_filter=False)


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_tme_scan_subsets_flcsm(tme_b200, golden, run_counter, precision):
    g = golden("c1_flcsm.npz")
    tme_b200.change_backend("b200", precision=precision, rotation_batch=32)
    res = _tme_scan("FLCSphericalMask", g["target"], g["template"], g["mask"], g["rotations"])
    scores, rot = np.asarray(res[0]), np.asarray(res[2])
    n = g["rotations"].shape[0]
    assert run_counter == [n], run_counter  # the whole chunk in one fused call
    tol = TOL if precision == "fp32" else max(TOL, 2e-3 * float(np.sqrt(np.mean(
        np.square(g["scores64"], dtype=np.float64)))))
    assert np.abs(scores - g["scores32"]).max() <= tol
    assert np.abs(scores - g["scores64"]).max() <= tol
    ref_rot = g["rot32"].astype(np.int32)
    mism = np.argwhere(rot != ref_rot)
    if len(mism):
        probe = O.scan_parallel(g["target"], g["template"], g["rotations"], "FLCSphericalMask",
                                template_mask=g["mask"], dtype=np.float64,
                                score_threshold=-np.inf, probe=mism)["probe"]
        best = g["scores64"][tuple(mism.T)]
        for j, (v, p) in enumerate(zip(mism, rot[tuple(mism.T)])):
            if p < 0:  # no rotation above the zero threshold here: the best is a tie with it
                assert best[j] <= 2 * TOL, (v, best[j])
            else:
                assert best[j] - probe[p, j] <= 2 * TOL, (v, p)
    # tme's result() inverts the mapping: index -> the rotation matrix scored under it
    rmap = res[3]
    assert len(rmap) == n
    for i in (0, 7, n - 1):
        assert np.array_equal(np.asarray(rmap[i], np.float32), g["rotations"][i])


def test_tme_scan_subsets_flc_with_tme_filters(tme_b200, golden, run_counter):
    """FLC with an arbitrary mask and tme's own Compose filters (CTF x wedge on the
    template, wedge on the target), which tme evaluates through the backend's methods."""
    from tme.filters import Compose, CTFReconstructed, WedgeReconstructed

    g = golden("flc_filt.npz")
    tme_b200.change_backend("b200", precision="fp32", rotation_batch=8)
    wedge = WedgeReconstructed(angles=(60, 60), create_continuous_wedge=True,
                               weight_wedge=False, opening_axis=2, tilt_axis=0)
    wedge_t = WedgeReconstructed(angles=(60, 60), create_continuous_wedge=True,
                                 weight_wedge=False, opening_axis=2, tilt_axis=0)
    ctf = CTFReconstructed(defocus_x=30000, amplitude_contrast=0.07,
                           spherical_aberration=2.7e7, acceleration_voltage=300e3)
    ctf.flip_phase = True
    for f in (wedge, wedge_t, ctf):
        f.sampling_rate = 6.8
    res = _tme_scan("FLC", g["target"], g["template"], g["mask"], g["rotations"],
                    template_filter=Compose([wedge, ctf]), target_filter=Compose([wedge_t]))
    assert run_counter == [g["rotations"].shape[0]], run_counter
    scores = np.asarray(res[0])
    assert np.abs(scores - g["scores32"]).max() <= TOL
    assert np.abs(scores - g["scores64"]).max() <= TOL
    assert np.count_nonzero(np.asarray(res[2]) != g["rot64"]) <= 5


def test_tme_scan_subsets_cc(tme_b200, golden, run_counter):
    g = golden("cc_small.npz")
    tme_b200.change_backend("b200", precision="fp32", rotation_batch=16)
    res = _tme_scan("CC", g["target"], g["template"], None, g["rotations"])
    assert run_counter == [g["rotations"].shape[0]], run_counter
    scale = np.abs(g["scores32"]).max()
    assert np.abs(np.asarray(res[0]) - g["scores32"]).max() <= TOL * scale
    assert np.count_nonzero(np.asarray(res[2]) != g["rot32"]) <= 5


def test_reference_backend_suite_with_b200(tme_b200):
    """tests/test_backends.py of the reference with the B200 backend appended to its
    BACKENDS_TO_TEST (``tests/ref_backend_suite.py`` does the appending), in a fresh
    process. Every test parametrised with the B200 backend must pass."""
    suite = os.path.join(REF_INSTALL, "tests", "test_backends.py")
    if not os.path.exists(suite):
        pytest.skip("the reference's test suite is not installed")
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([SHIM, os.path.join(ROOT, "tests"), ROOT, REF_INSTALL,
                                         env.get("PYTHONPATH", "")])
    out = subprocess.run(
        [sys.executable, "-m", "pytest", "-q", "-p", "ref_backend_suite", "-p", "no:cacheprovider",
         "--import-mode=importlib",
         "--confcutdir", os.path.dirname(suite), "--rootdir", os.path.dirname(suite),
         suite, "-rf"],
        env=env, capture_output=True, text=True, timeout=1200, cwd=os.path.dirname(suite))
    tail = out.stdout[-6000:] + out.stderr[-2000:]
    print(tail)
    assert "passed" in out.stdout, tail
    assert out.returncode == 0, tail
