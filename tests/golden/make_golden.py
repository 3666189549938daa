"""Generate the golden vectors in this directory by running the reference itself.

Usage (in a container that has the reference checkout; nothing else reads it):

    python tests/golden/make_golden.py [--reference /path/to/pyTME]

The reference package ``tme`` is copied to a temporary directory, its pybind11
extension (``tme/external/bindings.cpp``) is compiled there, and it is imported
with the stand-in modules in ``refshim/`` (pyFFTW -> scipy.fft; empty h5py /
mrcfile; scikit-image stubs). Its own public API then produces:

* ``c1_flcsm.npz``   FLCSphericalMask scan of the 64^3 / 16^3 blob case over the 360
                     rotations of its 30-degree set, FP32 and FP64 backends, plus
                     PeakCallerMaximumFilter on the FP32 map.
* ``flc_filt.npz``   FLC scan with an arbitrary (rotated) mask, a CTF x wedge
                     template filter and a wedge target filter, FP32 and FP64.
* ``cc_small.npz``   CC scan, FP32.
* ``flcsm_dc.npz``   FLCSphericalMask on a target with a +100 DC offset, FP32 and FP64.
* ``kat_exhaustive.npz``  the reference test's box case (tests/test_matching_exhaustive.py)
                     for every score and both ``pad_target_edges`` settings.
* ``rigid.npz``      order-1 rigid transforms of random data (both matrix forms).
* ``candidates.npz`` ``find_candidate_indices`` on random integer coordinates.
* ``filters.npz``    CTF, continuous wedge and Compose arrays for ``FILTER_CASES``.
* ``cubic.npz``      FLCSphericalMask, FLC and CC scans with ``interpolation_order=3``
                     (FP32 and FP64), and one order-3 rigid transform of data and mask.
* ``splits.npz``     ``split_shape`` slices and the bucket filter of peak calling
                     (``--only splits``).

Inputs are stored next to the outputs so the tests never need the reference.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import sysconfig
import tempfile
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _import_reference(ref: str):
    tmp = tempfile.mkdtemp(prefix="pytme_ref_")
    shutil.copytree(os.path.join(ref, "tme"), os.path.join(tmp, "tme"))
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    inc = subprocess.check_output([sys.executable, "-m", "pybind11", "--includes"],
                                  text=True).split()
    src = os.path.join(tmp, "tme", "external", "bindings.cpp")
    out = os.path.join(tmp, "tme", "extensions" + suffix)
    subprocess.check_call(["c++", "-O3", "-std=c++14", "-shared", "-fPIC", *inc, src,
                           "-o", out])
    sys.path[:0] = [os.path.join(HERE, "refshim"), tmp]
    import tme  # noqa: F401

    return tmp


def _scan(be, score, target, template, mask, rotations, dtype64=False,
          template_filter=None, target_filter=None, pad_edges=False, splits=None,
          callback=None, callback_args=None, job_schedule=(1, 1), order=1):
    from tme.matching_data import MatchingData
    from tme.matching_exhaustive import scan_subsets, MATCHING_EXHAUSTIVE_REGISTER
    from tme.analyzer import MaxScoreOverRotations

    kw = {}
    if dtype64:
        kw = dict(float_dtype=np.float64, complex_dtype=np.complex128,
                  overflow_safe_dtype=np.float64)
    be.change_backend("numpyfftw", **kw)
    md = MatchingData(target.copy(), template.copy())
    if mask is not None:
        md.template_mask = mask.copy()
    md.rotations = rotations
    if template_filter is not None:
        md.template_filter = template_filter
    if target_filter is not None:
        md.target_filter = target_filter
    setup, scoring = MATCHING_EXHAUSTIVE_REGISTER[score]
    return scan_subsets(
        md, matching_score=scoring, matching_setup=setup,
        callback_class=callback or MaxScoreOverRotations,
        callback_class_args=callback_args or {"score_threshold": 0},
        job_schedule=job_schedule, interpolation_order=order, pad_target_edges=pad_edges,
        pad_template_filter=False, target_splits=splits or {},
        backend_name="numpyfftw", backend_args=kw)


def _cubic(be, create_mask, syn):
    """Scans and one rigid transform with interpolation_order=3."""
    rng = np.random.default_rng(6)
    tmpl = syn.blob_template(12, rng, radius=3.5, sigma=1.2)
    target, _, _ = syn.make_tomogram((36, 32, 30), tmpl, 3, rng, scale=1.0)
    mask = syn.dilated_threshold_mask(tmpl, 0.1, 1)
    smask = create_mask("ellipse", shape=(12, 12, 12), radius=6,
                        center=(5.5, 5.5, 5.5)).astype(np.float32)
    rotations = syn.random_rotation_matrices(12, rng)
    cubic = {"target": target, "template": tmpl, "mask": mask, "smask": smask,
             "rotations": rotations}
    for score, m in (("FLCSphericalMask", smask), ("FLC", mask), ("CC", None)):
        r32 = _scan(be, score, target, tmpl, m, rotations, order=3)
        r64 = _scan(be, score, target, tmpl, m, rotations, dtype64=True, order=3)
        cubic[f"{score}_scores32"] = np.asarray(r32[0], np.float32)
        cubic[f"{score}_rot32"] = np.asarray(r32[2]).astype(np.int16)
        cubic[f"{score}_scores64"] = np.asarray(r64[0]).astype(np.float32)
        cubic[f"{score}_rot64"] = np.asarray(r64[2]).astype(np.int16)
    be.change_backend("numpyfftw")
    data = rng.normal(size=(13, 11, 9)).astype(np.float32)
    dmask = (rng.uniform(size=data.shape) > 0.3).astype(np.float32)
    big = np.zeros((16, 16, 16), np.float32)
    bigm = np.zeros((16, 16, 16), np.float32)
    o3, om3 = be.rigid_transform(arr=data, arr_mask=dmask, rotation_matrix=rotations[0],
                                 out=big, out_mask=bigm, use_geometric_center=True, order=3)
    cubic.update(rigid_data=data, rigid_mask=dmask, rigid_out=np.asarray(o3),
                 rigid_out_mask=np.asarray(om3))
    np.savez_compressed(os.path.join(HERE, "cubic.npz"), **cubic)



def _filters():
    """CTF / wedge / Compose arrays of FILTER_CASES from the reference."""
    from tme.filters import Compose, CTFReconstructed, WedgeReconstructed
    from filter_cases import FILTER_CASES, build_filter_case

    out = {}
    for i, case in enumerate(FILTER_CASES):
        out[f"case{i}"] = np.asarray(build_filter_case(case, CTFReconstructed,
                                                       WedgeReconstructed, Compose))
    np.savez_compressed(os.path.join(HERE, "filters.npz"), **out)


def _whitening():
    """LinearWhiteningFilter arrays of WHITENING_CASES from the reference, given the
    complex64 spectrum of the case's seeded data."""
    from tme.filters import LinearWhiteningFilter
    from filter_cases import WHITENING_CASES, whitening_data

    out = {}
    for i, (dshape, fshape, rfft, n_bins) in enumerate(WHITENING_CASES):
        _, data_rfft = whitening_data(i, dshape)
        ret = LinearWhiteningFilter()(shape=fshape, data_rfft=data_rfft, n_bins=n_bins,
                                      return_real_fourier=rfft)["data"]
        out[f"case{i}"] = np.asarray(ret)
    np.savez_compressed(os.path.join(HERE, "whitening.npz"), **out)


SPLIT_CASES = (((80, 80, 80), {0: 2}), ((81, 64, 33), {0: 3, 2: 2}), ((7, 5, 3), {0: 4, 1: 5}),
               ((3, 9, 10), {1: 4, 2: 3}), ((100,), {0: 7}), ((64, 64), {}),
               ((10, 11, 12), {0: 1, 1: 2, 2: 5}))


def _splits():
    """``split_shape`` slices for SPLIT_CASES (both equal_shape settings) and the
    reference's bucket filter (``_filter_bucket``, used by filter_points_indices above its
    point cutoff) on random points with and without scores."""
    from tme.analyzer.peaks import _filter_bucket
    from tme.matching_utils import split_shape

    out = {}
    for i, (shape, splits) in enumerate(SPLIT_CASES):
        for eq in (True, False):
            sl = split_shape(shape, dict(splits), equal_shape=eq)
            out[f"case{i}_{int(eq)}"] = np.array(
                [[(x.start, x.stop) for x in combo] for combo in sl], dtype=np.int64)
    rng = np.random.default_rng(12)
    for j, (n, md) in enumerate(((5000, 6), (20000, 10), (3000, 1))):
        c = rng.integers(0, 200, size=(n, 3)).astype(np.int64)
        sc = rng.normal(size=n).astype(np.float32)
        out[f"bucket{j}_coords"] = c
        out[f"bucket{j}_scores"] = sc
        out[f"bucket{j}_md"] = np.int64(md)
        out[f"bucket{j}_idx"] = np.asarray(_filter_bucket(c, md, sc))
        out[f"bucket{j}_idx_noscore"] = np.asarray(_filter_bucket(c, md, None))
    np.savez_compressed(os.path.join(HERE, "splits.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PYTME_REFERENCE",
                                                          "/root/reference"))
    ap.add_argument("--only", default=None,
                    help="write only this fixture (e.g. cubic) and leave the others")
    args = ap.parse_args()
    warnings.simplefilter("ignore")
    _import_reference(args.reference)
    sys.path.insert(0, REPO)

    from tme.backends import backend as be
    from tme.rotations import get_rotation_matrices
    from tme.matching_utils import create_mask
    from tme.analyzer import PeakCallerMaximumFilter, PeakCallerSort
    from tme.filters import Compose, CTFReconstructed, WedgeReconstructed
    from tme.extensions import find_candidate_indices
    from pytme_b200 import synthetic as syn

    if args.only == "cubic":
        _cubic(be, create_mask, syn)
        print("golden vectors written to", HERE)
        return
    if args.only == "whitening":
        _whitening()
        print("golden vectors written to", HERE)
        return
    if args.only == "filters":
        _filters()
        print("golden vectors written to", HERE)
        return
    if args.only == "splits":
        _splits()
        print("golden vectors written to", HERE)
        return

    # ---- config 1: 64^3 target, 16^3 blob template, spherical mask r=8, 30 deg set
    rng = np.random.default_rng(0)
    tmpl = syn.blob_template(16, rng)
    target, pos, rots_in = syn.make_tomogram((64, 64, 64), tmpl, 5, rng, scale=0.5)
    mask = create_mask("ellipse", shape=(16, 16, 16), radius=8,
                       center=(7.5, 7.5, 7.5)).astype(np.float32)
    rotations = get_rotation_matrices(30, dim=3).astype(np.float32)
    r32 = _scan(be, "FLCSphericalMask", target, tmpl, mask, rotations)
    r64 = _scan(be, "FLCSphericalMask", target, tmpl, mask, rotations, dtype64=True)
    be.change_backend("numpyfftw")
    pc = PeakCallerMaximumFilter(shape=r32[0].shape, num_peaks=16, min_distance=6)
    state = pc.init_state()
    state = pc(state, scores=np.asarray(r32[0]), rotation_matrix=np.eye(3, dtype=np.float32))
    np.savez_compressed(
        os.path.join(HERE, "c1_flcsm.npz"), target=target, template=tmpl, mask=mask,
        rotations=rotations, scores32=np.asarray(r32[0], np.float32),
        rot32=np.asarray(r32[2]).astype(np.int16),
        scores64=np.asarray(r64[0]).astype(np.float32),
        rot64=np.asarray(r64[2]).astype(np.int16),
        peak_pos=np.asarray(state[0]), peak_scores=np.asarray(state[2]),
        peak_num=16, peak_min_distance=6)

    # ---- FLC with arbitrary mask and CTF x wedge template filter, wedge target filter
    rng = np.random.default_rng(1)
    tmpl = syn.blob_template(12, rng, radius=3.5, sigma=1.2)
    mask = syn.dilated_threshold_mask(tmpl, 0.1, 1)
    target, _, _ = syn.make_tomogram((40, 36, 30), tmpl, 4, rng, snr=0.5, mask=mask)
    rotations = syn.random_rotation_matrices(24, rng)
    wedge = WedgeReconstructed(angles=(60, 60), create_continuous_wedge=True,
                               weight_wedge=False, opening_axis=2, tilt_axis=0)
    wedge_t = WedgeReconstructed(angles=(60, 60), create_continuous_wedge=True,
                                 weight_wedge=False, opening_axis=2, tilt_axis=0)
    ctf = CTFReconstructed(defocus_x=30000, amplitude_contrast=0.07,
                           spherical_aberration=2.7e7, acceleration_voltage=300e3)
    ctf.flip_phase = True
    for f in (wedge, wedge_t, ctf):
        f.sampling_rate = 6.8
    out = {}
    for tag, d64 in (("32", False), ("64", True)):
        r = _scan(be, "FLC", target, tmpl, mask, rotations, dtype64=d64,
                  template_filter=Compose([wedge, ctf]), target_filter=Compose([wedge_t]))
        out["scores" + tag] = np.asarray(r[0]).astype(np.float32)
        out["rot" + tag] = np.asarray(r[2]).astype(np.int16)
    # the filter arrays the reference multiplies in (template rfft shape, target rfft shape)
    be.change_backend("numpyfftw")
    import scipy.fft as sfft
    t_ft = sfft.rfftn(np.zeros((40, 36, 30), np.float32))
    tf = Compose([wedge, ctf])(shape=tmpl.shape, return_real_fourier=True,
                               shape_is_real_fourier=False, data_rfft=t_ft,
                               batch_dimension=None)["data"]
    gf = Compose([wedge_t])(shape=(40, 36, 30), return_real_fourier=True,
                            shape_is_real_fourier=False, data_rfft=t_ft,
                            batch_dimension=None, weight_type=None)["data"]
    np.savez_compressed(os.path.join(HERE, "flc_filt.npz"), target=target, template=tmpl,
                        mask=mask, rotations=rotations, template_filter=np.asarray(tf),
                        target_filter=np.asarray(gf), **out)

    # ---- CC
    rng = np.random.default_rng(2)
    tmpl = syn.blob_template(10, rng, radius=3.0, sigma=1.2)
    target, _, _ = syn.make_tomogram((36, 32, 30), tmpl, 3, rng, scale=1.0)
    rotations = syn.random_rotation_matrices(16, rng)
    r = _scan(be, "CC", target, tmpl, None, rotations)
    np.savez_compressed(os.path.join(HERE, "cc_small.npz"), target=target, template=tmpl,
                        rotations=rotations, scores32=np.asarray(r[0], np.float32),
                        rot32=np.asarray(r[2]).astype(np.int16))

    # ---- DC offset variant: E[x^2] - E[x]^2 cancellation in the denominator
    rng = np.random.default_rng(3)
    tmpl = syn.blob_template(12, rng, radius=3.5, sigma=1.2)
    target, _, _ = syn.make_tomogram((32, 32, 32), tmpl, 3, rng, scale=0.5)
    target = target + np.float32(100.0)
    mask = syn.spherical_mask((12, 12, 12), 6, center=(5.5, 5.5, 5.5))
    rotations = syn.random_rotation_matrices(16, rng)
    r32 = _scan(be, "FLCSphericalMask", target, tmpl, mask, rotations)
    r64 = _scan(be, "FLCSphericalMask", target, tmpl, mask, rotations, dtype64=True)
    np.savez_compressed(os.path.join(HERE, "flcsm_dc.npz"), target=target, template=tmpl,
                        mask=mask, rotations=rotations,
                        scores32=np.asarray(r32[0], np.float32),
                        rot32=np.asarray(r32[2]).astype(np.int16),
                        scores64=np.asarray(r64[0]).astype(np.float32),
                        rot64=np.asarray(r64[2]).astype(np.int16))

    # ---- the reference's known-answer box case (tests/test_matching_exhaustive.py:18-97)
    target = np.zeros((80, 80, 80))
    target[25:31, 22:28, 12:16] = 1
    template = np.zeros((41, 41, 35))
    template[20:26, 25:31, 17:21] = 1
    tmask = np.ones_like(template)
    kat = {}
    for score in ("CC", "FLC", "FLCSphericalMask"):
        for pad in (False, True):
            r = _scan(be, score, target, template, tmask, np.eye(3)[None].astype(np.float32),
                      pad_edges=pad, splits={0: 2}, callback=PeakCallerSort,
                      callback_args={}, job_schedule=(2, 1))
            kat[f"{score}_{int(pad)}_peak"] = np.asarray(r[0][0])
            kat[f"{score}_{int(pad)}_score"] = np.asarray(r[2][0])
            r = _scan(be, score, target, template, tmask, np.eye(3)[None].astype(np.float32),
                      pad_edges=pad)
            m = np.asarray(r[0], np.float32)
            kat[f"{score}_{int(pad)}_shape"] = np.asarray(m.shape)
            kat[f"{score}_{int(pad)}_argmax"] = np.asarray(np.unravel_index(np.argmax(m),
                                                                            m.shape))
            kat[f"{score}_{int(pad)}_max"] = m.max()
    np.savez_compressed(os.path.join(HERE, "kat_exhaustive.npz"), **kat)

    _cubic(be, create_mask, syn)
    _filters()
    _whitening()

    # ---- rigid transforms (order 1, constant mode), both matrix forms
    be.change_backend("numpyfftw")
    rng = np.random.default_rng(4)
    data = rng.normal(size=(13, 11, 9)).astype(np.float32)
    dmask = (rng.uniform(size=data.shape) > 0.3).astype(np.float32)
    rots = syn.random_rotation_matrices(6, rng)
    rots[0] = np.eye(3, dtype=np.float32)
    rots[1] = np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    outs, outs_m, mats = [], [], []
    center = np.divide(np.asarray(data.shape) - 1, 2)
    for R in rots:
        m = be._rigid_transform_matrix(rotation_matrix=R, center=center)
        mats.append(m)
        o, _ = be.rigid_transform(arr=data, rotation_matrix=m, order=1,
                                  out=np.zeros_like(data))
        outs.append(o)
        big = np.zeros((16, 16, 16), np.float32)
        bigm = np.zeros((16, 16, 16), np.float32)
        o2, om = be.rigid_transform(arr=data, arr_mask=dmask, rotation_matrix=R, out=big,
                                    out_mask=bigm, use_geometric_center=True, order=1)
        outs_m.append(np.stack([o2, om]))
    np.savez_compressed(os.path.join(HERE, "rigid.npz"), data=data, mask=dmask,
                        rotations=rots, matrices=np.stack(mats), out=np.stack(outs),
                        out_pad=np.stack(outs_m))

    # ---- greedy min-distance filter
    rng = np.random.default_rng(5)
    cand = {}
    for i, (n, md) in enumerate(((50, 3), (400, 6), (1000, 24), (1, 5))):
        coords = rng.integers(0, 100, size=(n, 3)).astype(np.int64)
        cand[f"coords{i}"] = coords
        cand[f"md{i}"] = md
        cand[f"idx{i}"] = np.asarray(find_candidate_indices(coords, md))
    np.savez_compressed(os.path.join(HERE, "candidates.npz"), **cand)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
