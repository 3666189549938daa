#!/usr/bin/env python
"""Benchmark of the exhaustive FLCSphericalMask rotation scan.

Workload (the configuration the headline metric is quoted on): a 512x512x200
float32 tomogram (N(0,1) noise plus 300 rotated copies of the template at SNR 0.05),
a 48^3 Gaussian-blob template with a spherical mask of radius 24, and the 7-degree
rotation set (27,672 rotations, super-Fibonacci sampling of the same size as the
reference's set). All inputs are seeded synthetic data.

A step scores ``--step-rotations`` rotations (a contiguous slice of the set; a rank
takes a different slice per step) over the whole tomogram, with the target spectrum,
denominator and running (max, argmax) state resident in HBM; ``value`` is rotations
per second of the whole job. The spectra and the state (>= 210 MB each) are larger
than the 126 MB L2, so consecutive steps do not hit in L2.

``--impl reference`` times the CPU oracle (the reference algorithm restated in
NumPy/SciPy) on the host cores instead and prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "FLC rotations/s, 512x512x200 tomo, 48³ template, err≤1e-4 vs FP64, vs plain"
SHAPE = (512, 512, 200)
TSIZE = 48
ANGLE = 7.0
WORKLOAD = ("FLCSphericalMask scan, 512x512x200 float32 tomogram (noise + 300 copies, "
            "SNR 0.05), 48^3 blob template, spherical mask r=24, 7-degree set "
            "(27672 rotations), MaxScoreOverRotations")


def parse():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--step-rotations", type=int, default=1024)
    ap.add_argument("--precision", choices=("fp32", "mixed"), default="mixed")
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--zpass", choices=("auto", "tensor", "fft"), default="auto",
                    help="z pass on the tensor cores, as CUDA-core FFTs, or the plan default")
    ap.add_argument("--ypass", choices=("auto", "tensor", "tensor-inplace", "tensor2", "fft"),
                    default="auto",
                    help="y pass on the tensor cores, as CUDA-core FFTs, or the plan default")
    ap.add_argument("--xpass", choices=("auto", "tensor", "fft"), default="auto",
                    help="x pass on the tensor cores, as CUDA-core FFTs, or the plan default "
                         "(tensor cores for mixed precision)")
    ap.add_argument("--plain-rotations", type=int, default=12)
    ap.add_argument("--e2e-rotations", type=int, default=0,
                    help="rotations per end-to-end call (0: the whole set)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the config-2 (filtered FLC) and config-4 (uneven batch) legs")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="scoring-loop seconds of the cpu_baseline leg of this arm")
    ap.add_argument("--ref-seconds", type=float, default=60.0,
                    help="scoring-loop seconds of --impl reference (at least)")
    ap.add_argument("--err-rotations", type=int, default=32,
                    help="rotations of the measured error against the FP64 oracle (0: skip)")
    ap.add_argument("--small", action="store_true", help="128x128x64 / 24^3 quick check")
    ap.add_argument("--profile-case", default=None, metavar="N0,N1,N2",
                    help="run --groups launch groups of the fused scan on a target of this "
                         "shape and exit (a small case for ncu captures; no timing, no JSON)")
    ap.add_argument("--groups", type=int, default=2)
    ap.add_argument("--profile-score", choices=("FLCSphericalMask", "FLC", "CC"),
                    default="FLCSphericalMask", help="score of --profile-case")
    ap.add_argument("--profile-template", type=int, default=None,
                    help="template edge of --profile-case (default: the bench's 48)")
    return ap.parse_args()


def _synthetic():
    """pytme_b200/synthetic.py loaded by file path: the input generators are plain NumPy,
    and loading them this way keeps the reference arm from importing the package (and
    its CUDA library)."""
    return _load_by_path("_pytme_b200_synthetic", os.path.join("pytme_b200", "synthetic.py"))


def _load_by_path(name, rel):
    import importlib.util

    mod = sys.modules.get(name)
    if mod is None:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, rel))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return mod


def rotation_set(angle):
    """(float32 matrices, description): the reference's own quaternion set for ``angle``
    when its data are available (pytme_b200/rotations.py finds them: an installed tme,
    baseline/_ref), else the super-Fibonacci stand-in of the same size. Loaded by file
    path so the reference arm does not import the package."""
    rot = _load_by_path("_pytme_b200_rotations", os.path.join("pytme_b200", "rotations.py"))
    try:
        m = rot.get_rotation_matrices(angle)
        return np.ascontiguousarray(m, dtype=np.float32), \
            f"the reference's quaternion set for {angle} degrees ({len(m)} rotations)"
    except FileNotFoundError:
        m = _synthetic().rotations_for_angle(angle)
        return m, f"super-Fibonacci stand-in of the reference set's size ({len(m)} rotations)"


def make_inputs(small=False):
    """The headline workload: a 512x512x200 tomogram (N(0,1) noise plus 300 rotated
    copies at SNR 0.05), a 48^3 blob template, its spherical mask (r = 24) and the
    7-degree rotation set."""
    syn = _synthetic()
    rng = np.random.default_rng(2024)
    shape = (128, 128, 64) if small else SHAPE
    t = 24 if small else TSIZE
    tmpl = syn.blob_template(t, rng, n_blobs=6, sigma=1.5 * t / 16, radius=5.0 * t / 16)
    c = (t - 1) / 2.0
    mask = syn.spherical_mask((t, t, t), t / 2, center=(c, c, c))
    target, _, _ = syn.make_tomogram(shape, tmpl, 20 if small else 300, rng, snr=0.05, mask=mask)
    rots, _ = rotation_set(ANGLE)
    return target, tmpl, mask, rots


CONFIG2_SHAPE = (256, 256, 128)
CONFIG2_ANGLE = 15.0


def make_config2_inputs():
    """The filtered-FLC workload: a 256x256x128 tomogram (N(0,1) noise plus 40 rotated
    copies at SNR 0.1), a 32^3 blob template, the mask (template > 0.1 max) dilated by 2
    voxels, and the 15-degree rotation set. Filter parameters: ``config2_filters``."""
    syn = _synthetic()
    rng = np.random.default_rng(2025)
    tmpl = syn.blob_template(32, rng, n_blobs=6, sigma=3.0, radius=10.0)
    mask = syn.dilated_threshold_mask(tmpl, 0.1, 2)
    target, _, _ = syn.make_tomogram(CONFIG2_SHAPE, tmpl, 40, rng, snr=0.1, mask=mask)
    rots, _ = rotation_set(CONFIG2_ANGLE)
    return target, tmpl, mask, rots


# CTF (300 kV, Cs 2.7 mm, amplitude contrast 0.07, defocus 3 um, 6.8 A pixels, phase
# flipped) and a continuous missing wedge of +-60 degrees (opening axis 2, tilt axis 0):
# the template gets CTF x wedge, the target the wedge.
CONFIG2_CTF = dict(defocus_x=30000, amplitude_contrast=0.07, spherical_aberration=2.7e7,
                   acceleration_voltage=300e3, sampling_rate=6.8, flip_phase=True)
CONFIG2_WEDGE = dict(angles=(60, 60), opening_axis=2, tilt_axis=0,
                     create_continuous_wedge=True)


def profile_traffic(stage, precision, batch, variant):
    """DRAM bytes (read + write) of one bench-size launch of ``stage`` from the committed
    ncu summaries: each holds a line ``bench-traffic: stage=... precision=... batch=...
    variant=... bytes=... <how the capture was scaled>``. Returns (bytes, source) or
    (None, None) when no summary covers the kernel the bench ran."""
    import glob
    import re

    pat = re.compile(r"^bench-traffic: stage=(\S+) precision=(\S+) batch=(\d+) variant=(\S+) "
                     r"bytes=(\S+)\s*(.*)$")
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                m = pat.match(line.strip())
                if m and m.group(1) == stage and m.group(2) == precision and \
                        int(m.group(3)) == batch and m.group(4) == variant:
                    return float(m.group(5)), f"{os.path.relpath(path, ROOT)}: {m.group(6)}"
    return None, None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for name, v in zip(names, s[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


CONFIG4_ANGLE = 12.0
# 12 tomograms of mixed sizes between 128^3 and 320x320x160
CONFIG4_SHAPES = ((128, 128, 128), (160, 160, 128), (192, 192, 128), (256, 256, 128),
                  (256, 256, 160), (320, 320, 128), (320, 320, 160), (128, 256, 160),
                  (192, 256, 128), (256, 192, 160), (160, 320, 128), (320, 256, 160))
CONFIG4_TEMPLATES = (24, 32, 40)


def make_config4_jobs(n_rotations=None, seed=2026):
    """The uneven-batch workload: 12 tomograms (N(0,1) noise plus 6 rotated copies of each
    of 3 blob templates, 24^3, 32^3 and 40^3, at SNR 0.1), every tomogram searched with
    every template (36 jobs) over the 12-degree set, with a per-tomogram CTF (defocus
    uniform in 1.5-4.5 um, 300 kV, Cs 2.7 mm, amplitude contrast 0.07, 6.8 A pixels, phase
    flipped) times a continuous wedge (half-angle uniform in 50-65 degrees) on the
    template and the wedge on the target. FLCSphericalMask with each template's spherical
    mask. Returns a list of (job keyword arguments, template size, target index)."""
    syn = _synthetic()
    rng = np.random.default_rng(seed)
    rots, _ = rotation_set(CONFIG4_ANGLE)
    if n_rotations is not None:
        rots = np.ascontiguousarray(rots[:: max(1, len(rots) // n_rotations)][:n_rotations])
    templates = []
    for t in CONFIG4_TEMPLATES:
        tmpl = syn.blob_template(t, rng, n_blobs=6, sigma=1.5 * t / 16, radius=5.0 * t / 16)
        mask = syn.spherical_mask((t,) * 3, t / 2, center=((t - 1) / 2,) * 3)
        templates.append((t, tmpl, mask))
    jobs = []
    for i, shape in enumerate(CONFIG4_SHAPES):
        target = rng.normal(size=shape).astype(np.float32)
        for t, tmpl, mask in templates:
            sel = tmpl[mask > 0]
            amp = float(np.sqrt(0.1 / max(float(sel.var()), 1e-30)))
            syn.insert_copies(target, tmpl, 6, amp, rng)
        defocus = float(rng.uniform(15000.0, 45000.0))
        wedge = float(rng.uniform(50.0, 65.0))
        for t, tmpl, mask in templates:
            jobs.append((dict(target=target, template=tmpl, mask=mask, rotations=rots,
                              score="FLCSphericalMask", interpolation_order=1,
                              meta={"defocus": defocus, "wedge": wedge}), t, i))
    return jobs


def config4_filters(meta):
    """Filter objects of a config-4 job (built on the GPU by scan_batch)."""
    from pytme_b200.filters import Compose, CTFReconstructed, WedgeReconstructed

    w = dict(angles=(meta["wedge"], meta["wedge"]), opening_axis=2, tilt_axis=0,
             create_continuous_wedge=True)
    ctf = dict(CONFIG2_CTF, defocus_x=meta["defocus"])
    return (Compose([WedgeReconstructed(**w), CTFReconstructed(**ctf)]),
            Compose([WedgeReconstructed(**w)]))


# ------------------------------------------------------------------ CPU arms
REF_INSTALL = os.path.join(ROOT, "baseline", "_ref")
REF_SHIM = os.path.join(ROOT, "tests", "golden", "refshim")


def _host_workers(gb_per_worker: float, cap: int = 64) -> int:
    import psutil

    avail = psutil.virtual_memory().available / 1024 ** 3
    return max(1, min(os.cpu_count() or 1, cap, int(avail // gb_per_worker)))


class TmeScanLoop:
    """The reference's own scan (tme/matching_exhaustive.py:144-295) on the host cores,
    split into steps: ``scan``'s set-up once (MatchingData padding, the target filter,
    ``flcSphericalMask_setup``, the SharedAnalyzerProxy instances), then every step runs
    ``scan``'s joblib ``Parallel(n_jobs)`` over ``corr_scoring`` with one rotation chunk per
    job, into the same analyzer state. NumpyFFTWBackend, FP32, interpolation order 1,
    ``job_schedule=(1, n_jobs)``; pyFFTW is replaced by scipy.fft (tests/golden/refshim).
    The package comes from baseline/_ref (oracle/build_ref.py --baseline)."""

    kind = "reference"

    def __init__(self, target, tmpl, mask, n_rotations, n_jobs):
        for p, front in ((REF_SHIM, True), (REF_INSTALL, False)):
            if p not in sys.path:
                sys.path.insert(0, p) if front else sys.path.append(p)
        from multiprocessing.managers import SharedMemoryManager

        from joblib import Parallel
        from tme.analyzer import MaxScoreOverRotations
        from tme.analyzer.proxy import SharedAnalyzerProxy
        from tme.backends import backend as be
        from tme.matching_data import MatchingData
        from tme.matching_exhaustive import (_setup_template_filter_apply_target_filter,
                                             _wrap_backend)
        from tme.matching_scores import MATCHING_EXHAUSTIVE_REGISTER

        t0 = time.perf_counter()
        be.change_backend("numpyfftw")
        self.be = be
        self.n_jobs = n_jobs
        self.smh = SharedMemoryManager()
        self.smh.start()
        md = MatchingData(target.copy(), tmpl.copy())
        md.template_mask = mask.copy()
        md.rotations = np.eye(3, dtype=np.float32)[None]
        md, offset = md.subset_by_slice(target_pad=md.target_padding(pad_target=False))
        md.to_backend()
        conv, fwd, inv, shift = md.fourier_padding(pad_target=False)
        tf = _setup_template_filter_apply_target_filter(md, fwd, inv, pad_template_filter=False)
        setup_fn, self.score_fn = MATCHING_EXHAUSTIVE_REGISTER["FLCSphericalMask"]
        args = {"shape": fwd, "offset": offset, "fourier_shift": shift, "fast_shape": fwd,
                "targetshape": md._output_shape, "templateshape": md.template.shape,
                "convolution_shape": conv, "thread_safe": n_jobs > 1,
                "convolution_mode": "same", "shm_handler": self.smh,
                "only_unique_rotations": True, "n_rotations": n_rotations,
                "aggregate_axis": md._batch_axis(md._batch_mask),
                "inversion_mapping": n_jobs == 1, "score_threshold": 0}
        self.setup = setup_fn(matching_data=md, template_filter=tf, fast_shape=fwd,
                              fast_ft_shape=inv, shm_handler=self.smh)
        self.setup["interpolation_order"] = 1
        self.setup["template_filter"] = be.to_sharedarr(tf, self.smh)
        self.callbacks = [SharedAnalyzerProxy(MaxScoreOverRotations, args,
                                              shm_handler=self.smh if n_jobs > 1 else None)
                          for _ in range(max(n_jobs // 8, 1))]
        self.wrapped = _wrap_backend(self.score_fn)
        self.parallel = Parallel(n_jobs=n_jobs)
        self.parallel.__enter__()  # keep the workers for every step
        self.setup_s = time.perf_counter() - t0

    def step(self, chunks):
        from joblib import delayed

        nc = len(self.callbacks)
        self.parallel(delayed(self.wrapped)(
            backend_name=self.be._backend_name, backend_args=self.be._backend_args,
            rotations=r, callback=self.callbacks[i % nc], **self.setup)
            for i, r in enumerate(chunks))

    def close(self):
        self.parallel.__exit__(None, None, None)
        self.smh.shutdown()


_PORT_STATE = {}


def _port_init(target, tmpl, mask):
    from oracle import tm_oracle as O

    t, t_rev, m_rev = O._prepare(target, tmpl, mask, False, None, np.float32)
    _, fast, _, _ = O.fourier_padding(t.shape, t_rev.shape)
    _PORT_STATE.update(O=O, t_rev=t_rev, m_rev=m_rev, fast=fast,
                       setup=O._setup("FLCSphericalMask", t, t_rev, m_rev, fast, np.float32,
                                      np.complex64),
                       ms=np.zeros(fast, np.float32), am=np.full(fast, -1, np.int32))


def _port_step(rots):
    st = _PORT_STATE
    st["O"]._loop("FLCSphericalMask", st["setup"], st["t_rev"], st["m_rev"], rots, st["fast"],
                  np.float32, np.complex64, None, 0, st["ms"], st["am"])
    return 0


class PortScanLoop:
    """The oracle (the reference's loop restated in NumPy/SciPy) with the same step
    structure as TmeScanLoop: spawned worker processes do the set-up once, then every
    step scores one rotation chunk per worker. Used when the reference package is not
    installed."""

    kind = "port"

    def __init__(self, target, tmpl, mask, n_rotations, n_jobs):
        import multiprocessing as mp

        t0 = time.perf_counter()
        self.n_jobs = n_jobs
        self.pool = mp.get_context("spawn").Pool(n_jobs, initializer=_port_init,
                                                 initargs=(target, tmpl, mask))
        self.pool.map(_port_step, [np.zeros((0, 3, 3), np.float32)] * n_jobs)
        self.setup_s = time.perf_counter() - t0

    def step(self, chunks):
        self.pool.map(_port_step, chunks, chunksize=1)

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_scan_loop(target, tmpl, mask, n_rotations, prefer_reference=True):
    """The reference's loop on the host cores: tme itself when baseline/_ref holds it,
    else the oracle port."""
    if prefer_reference and os.path.isdir(os.path.join(REF_INSTALL, "tme")):
        try:
            return TmeScanLoop(target, tmpl, mask, n_rotations, _host_workers(2.0))
        except ImportError:
            pass
    return PortScanLoop(target, tmpl, mask, n_rotations, _host_workers(3.0))


def time_cpu_loop(loop, rots, steps, warmup, min_seconds):
    """``warmup`` steps of one rotation per worker (the last of them, when there are two or
    more, of two), then ``steps`` timed steps of r rotations per worker, r sized from the
    warm-up's cost per added rotation so the timed loop lasts at least ``min_seconds``.
    Returns (rotations/s, ms per step, rotations timed, r)."""
    w = loop.n_jobs
    pos = 0

    def chunks(r):
        nonlocal pos
        out = []
        for _ in range(w):
            out.append(np.ascontiguousarray(rots[pos % len(rots):pos % len(rots) + r]))
            pos += r
        return out

    t_warm = []
    nw = max(1, warmup)
    for i in range(nw):
        t0 = time.perf_counter()
        loop.step(chunks(2 if (nw >= 2 and i == nw - 1) else 1))
        t_warm.append(time.perf_counter() - t0)
    # a step costs a fixed part (dispatch, analyzer merge) plus a part per rotation and
    # worker: the last two warm-up steps (one and two rotations per worker; the first ones
    # also plan the FFTs and fault in the workers' memory) give both; 15 % margin
    if nw >= 2:
        per_rot = max(t_warm[-1] - t_warm[-2], 0.25 * t_warm[-2])
        fixed = max(t_warm[-2] - per_rot, 0.0)
    else:
        per_rot, fixed = t_warm[-1], 0.0
    target = 1.15 * min_seconds / max(steps, 1)
    r = int(min(16, max(1, np.ceil((target - fixed) / per_rot))))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        loop.step(chunks(r))
        times.append(time.perf_counter() - t0)
    n = steps * w * r
    return n / sum(times), 1000.0 * float(np.mean(times)), n, r


def cpu_sample_desc(loop, n, r, steps, total_s):
    what = ("tme's own scan (NumpyFFTWBackend, scipy.fft for pyFFTW) via joblib"
            if loop.kind == "reference" else "the oracle port in spawned processes")
    return (f"{what}: {steps} steps x {loop.n_jobs} workers x {r} rotation(s) of the 7-degree "
            f"set on the full 512x512x200 map ({n} rotations, scoring loop {total_s:.1f} s); "
            f"set-up {loop.setup_s:.1f} s excluded")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    target, tmpl, mask, rots = make_inputs(args.small)
    loop = cpu_scan_loop(target, tmpl, mask, len(rots))
    try:
        value, ms, n, r = time_cpu_loop(loop, rots, max(1, args.steps), args.warmup,
                                        args.ref_seconds)
    finally:
        loop.close()
    total = n / value
    line = {
        "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": args.gpus,
        "steps": max(1, args.steps), "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference", "config": workload_config(args.small),
        "cpu_baseline": {"value": value, "unit": "rotations/s", "cores": loop.n_jobs,
                         "kind": loop.kind,
                         "sample": cpu_sample_desc(loop, n, r, max(1, args.steps), total),
                         "setup_s": loop.setup_s},
        "e2e": {"value": value, "unit": "rotations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(small=False):
    """The workload both arms report (identical keys and values)."""
    shape = (128, 128, 64) if small else SHAPE
    t = 24 if small else TSIZE
    return {"workload": WORKLOAD + (" [small]" if small else ""), "target_shape": list(shape),
            "template_shape": [t] * 3, "rotations": 27672, "score": "FLCSphericalMask",
            "analyzer": "MaxScoreOverRotations", "interpolation_order": 1,
            "rotation_set": rotation_set(ANGLE)[1],
            "l2": "inputs larger than L2 (target spectrum 212 MB, state 420 MB)"}


def fp64_error(target, tmpl, mask, rots, gpu_map, n_workers):
    """Max |GPU map - FP64 oracle map| over the 'same'-mode map of a scan of ``rots``
    (the oracle on the host cores, spawned workers)."""
    from oracle import tm_oracle as O

    ref = O.scan_parallel(target, tmpl, rots, "FLCSphericalMask", template_mask=mask,
                          dtype=np.float64, n_workers=n_workers)
    return float(np.abs(np.asarray(gpu_map, np.float64) - ref["scores"]).max())


def run_ours(args):
    import torch
    import torch.distributed as dist

    import pytme_b200 as P
    from pytme_b200.distributed import merge_max_argmax, rotation_share
    from pytme_b200.matching import fourier_padding, rigid_transform_matrices
    from pytme_b200.scores import ScanPlan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    target, tmpl, mask, rots = make_inputs(args.small)
    conv, fast, fast_ft, shift = fourier_padding(target.shape, tmpl.shape)
    t_rev = np.ascontiguousarray(tmpl[::-1, ::-1, ::-1])
    m_rev = np.ascontiguousarray(mask[::-1, ::-1, ::-1])
    center = np.divide(np.asarray(tmpl.shape) - 1, 2)
    mats_all = torch.as_tensor(rigid_transform_matrices(rots, center), device=dev)
    n_rot = mats_all.shape[0]
    lo, hi = rotation_share(n_rot, rank, world)

    plan = ScanPlan("FLCSphericalMask", fast, tmpl.shape, precision=args.precision,
                    batch=args.batch)
    plan.set_xpass(args.xpass)
    plan.set_ypass(args.ypass)
    plan.set_zpass(args.zpass)
    plan.set_template(t_rev, m_rev)
    tpad = torch.zeros(fast, dtype=torch.float32, device=dev)
    tpad[tuple(slice(0, s) for s in target.shape)] = torch.as_tensor(target, device=dev)
    plan.set_target(tpad)
    del tpad
    smax = torch.zeros(fast, dtype=torch.float32, device=dev)
    sarg = torch.full(fast, -1, dtype=torch.int32, device=dev)
    R = args.step_rotations
    span = max(1, hi - lo - R)

    def step(i):
        s = lo + (i * R) % span
        plan.run(mats_all[s:s + R], s, smax, sarg)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(args.steps):
            step(args.warmup + i)
        if world > 1:
            merge_max_argmax(smax, sarg)
        e1.record(stream)
        torch.cuda.synchronize()
    plan.check()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_rot = world * args.steps * R
    value = total_rot / (ms / 1000.0)
    groups = -(-R // args.batch)
    launches = args.steps * groups * 8

    result = None
    if rank == 0:
        # per-stage timing (events around each stage on the launching stream)
        plan.set_timing(True)
        step(0)
        timing = plan.get_timing()
        plan.set_timing(False)
        stage_ms = {k: v[0] for k, v in timing.items()}
        dom = max(("template", "xpass", "ypass", "zpass"), key=lambda k: stage_ms[k])
        n_launch = timing[dom][1]
        avg_ms = stage_ms[dom] / max(n_launch, 1)
        alg = plan.stage_bytes(dom, args.batch)
        peak, peak_kind = measured_peaks()
        achieved = alg / (avg_ms / 1000.0) / 1e9
        stages = {k: {"ms": round(v[0], 3), "launches": v[1],
                      "gbs": round(plan.stage_bytes(k, args.batch) / (v[0] / max(v[1], 1) / 1000)
                                   / 1e9, 1) if v[1] and k != "prepare" else None}
                  for k, v in timing.items()}
        # plain FP32 one-rotation-at-a-time path on the same GPU
        plain = ScanPlan("FLCSphericalMask", fast, tmpl.shape, precision="fp32", plain=True)
        plain.set_template(t_rev, m_rev)
        tpad = torch.zeros(fast, dtype=torch.float32, device=dev)
        tpad[tuple(slice(0, s) for s in target.shape)] = torch.as_tensor(target, device=dev)
        plain.set_target(tpad)
        del tpad
        pm = torch.zeros(fast, dtype=torch.float32, device=dev)
        pa = torch.full(fast, -1, dtype=torch.int32, device=dev)
        plain.run(mats_all[:2], 0, pm, pa)
        torch.cuda.synchronize()
        pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        pe0.record(stream)
        plain.run(mats_all[:args.plain_rotations], 0, pm, pa)
        pe1.record(stream)
        torch.cuda.synchronize()
        plain_rate = args.plain_rotations / (pe0.elapsed_time(pe1) / 1000.0)
        plain.close()
        del pm, pa

        variant = {"xpass": plan.xpass, "zpass": plan.zpass, "ypass": plan.ypass}.get(dom, "fft")
        traffic, traffic_src = (None, None) if args.small else profile_traffic(
            dom, args.precision, args.batch, variant)
        result = {
            "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f32 (f16 spectra, f64 denominator)",
            "data": "synthetic",
            "config": workload_config(args.small),
            "impl_config": {"step_rotations": R, "rotation_batch": args.batch,
                            "precision": args.precision, "xpass": plan.xpass,
                            "ypass": plan.ypass, "zpass": plan.zpass, "fast_shape": list(fast)},
            "voxel_rotations_per_s": value * float(np.prod(fast)),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": traffic_src,
                         "alg_bytes_per_launch": alg,
                         "avg_launch_ms": avg_ms},
            "stages": stages,
            "plain": {"value": plain_rate, "unit": "rotations/s", "rotations": args.plain_rotations,
                      "path": "fp32, one rotation at a time, full cuFFT r2c/c2r"},
            "vs_plain": value / world / plain_rate,
            "model_roofline": model_roofline(fast, args.precision, args.batch, value,
                                             measured_peaks()),
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
    if rank == 0:
        result["peak_calling"] = time_peak_calling(smax)
    # end-to-end through the public API with host arrays (rank 0)
    if rank == 0 and not args.no_e2e:
        n_e2e = args.e2e_rotations or n_rot
        P.backend.change_backend("b200", precision=args.precision, rotation_batch=args.batch,
                                 xpass=args.xpass, ypass=args.ypass, zpass=args.zpass)
        setup, scoring = P.MATCHING_EXHAUSTIVE_REGISTER["FLCSphericalMask"]
        del plan, smax, sarg
        torch.cuda.empty_cache()

        def e2e():
            md = P.MatchingData(target, tmpl)
            md.template_mask = mask
            md.rotations = rots[:n_e2e]
            res = P.scan_subsets(md, matching_score=scoring, matching_setup=setup,
                                 callback_class=P.MaxScoreOverRotations,
                                 callback_class_args={"score_threshold": 0},
                                 interpolation_order=1)
            return res

        e2e()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = e2e()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        h2d = target.nbytes + tmpl.nbytes + mask.nbytes + n_e2e * 64
        d2h = res[0].nbytes + res[2].nbytes
        result["e2e"] = {"value": n_e2e / dt, "unit": "rotations/s", "h2d_bytes_per_step": h2d,
                         "d2h_bytes_per_step": d2h, "rotations_per_step": n_e2e,
                         "seconds_per_step": dt,
                         "call": "pytme_b200.scan_subsets on host NumPy arrays"}
    if rank == 0 and world == 1 and not args.no_legs:
        torch.cuda.empty_cache()
        # config 4 runs in FP32: its filtered maps exceed 1e-4 in mixed precision
        result["legs"] = {"config2": leg_config2(args.precision, cpu=not args.no_cpu),
                          "config4": leg_config4("fp32", cpu=not args.no_cpu)}
        torch.cuda.empty_cache()
    if rank == 0 and args.err_rotations > 0:
        # measured score error of the GPU map against the FP64 oracle on a rotation subset
        # spread over the set (the public API on the GPU, the oracle on the host cores)
        stride = max(1, n_rot // args.err_rotations)
        sub = np.ascontiguousarray(rots[::stride][:args.err_rotations])
        P.backend.change_backend("b200", precision=args.precision, rotation_batch=args.batch,
                                 xpass=args.xpass, ypass=args.ypass, zpass=args.zpass)
        setup, scoring = P.MATCHING_EXHAUSTIVE_REGISTER["FLCSphericalMask"]
        md = P.MatchingData(target, tmpl)
        md.template_mask = mask
        md.rotations = sub
        gmap = P.scan_subsets(md, matching_score=scoring, matching_setup=setup,
                              callback_class=P.MaxScoreOverRotations,
                              callback_class_args={"score_threshold": 0},
                              interpolation_order=1)[0]
        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        err = fp64_error(target, tmpl, mask, sub, gmap, _host_workers(6.0, cap=32))
        result["error_vs_fp64"] = {
            "max_abs": err, "bound": 1e-4, "rotations": int(sub.shape[0]),
            "what": "max |score - FP64 oracle| over the 'same'-mode map, rotations spread "
                    "over the 7-degree set", "oracle_s": time.perf_counter() - t0}
    if rank == 0 and not args.no_cpu:
        loop = cpu_scan_loop(target, tmpl, mask, n_rot)
        try:
            rate, cms, n, r = time_cpu_loop(loop, rots, 3, 1, args.cpu_seconds)
        finally:
            loop.close()
        result["cpu_baseline"] = {"value": rate, "unit": "rotations/s", "cores": loop.n_jobs,
                                  "kind": loop.kind,
                                  "sample": cpu_sample_desc(loop, n, r, 3, n / rate),
                                  "setup_s": loop.setup_s}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def model_roofline(fast, precision, batch, rate, peak):
    """Whole-scan HBM fraction by the FFT I/O model of the fused FLCSphericalMask / CC path:
    per rotation 7 passes over the S-element product spectrum of e bytes per value (two HBM
    passes per full-size FFT, elementwise stages fused, the target spectrum read once)
    plus the per-voxel state (max, argmax, the d-byte denominator and the state write) once
    per launch group of B rotations: 7 S e + (d + 16) N / B bytes."""
    n0, n1, n2 = (int(x) for x in fast)
    N = n0 * n1 * n2
    S = n0 * n1 * (n2 // 2 + 1)
    e = 4 if precision == "mixed" else 8
    d = 4  # the inverse denominator is stored as float32
    per_rot = 7 * S * e + (d + 16) * N / batch
    gbs = per_rot * rate / 1e9
    return {"bytes_per_rotation": per_rot, "achieved": gbs, "peak": peak[0],
            "peak_kind": peak[1], "unit": "GB/s", "frac": gbs / peak[0],
            "model": "7 S e + (d + 16) N / B bytes per rotation (two HBM passes per "
                     "full-size FFT, fused elementwise stages, state once per launch group)"}


def time_peak_calling(scores, num_peaks=1000, min_distance=24, reps=3):
    """PeakCallerMaximumFilter (the reference's defaults for the analysis: 1,000 peaks,
    minimum distance 24) on a device score map, timed from the call to the peaks on the
    host (maximum filter, candidate gather and greedy distance filter on the device)."""
    import torch

    from pytme_b200.analyzer import PeakCallerMaximumFilter

    pc = PeakCallerMaximumFilter(shape=tuple(scores.shape), num_peaks=num_peaks,
                                 min_distance=min_distance)
    eye = np.eye(3, dtype=np.float32)
    st = pc(pc.init_state(), scores=scores, rotation_matrix=eye)  # warm-up
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        st = pc(pc.init_state(), scores=scores, rotation_matrix=eye)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    found = int(np.count_nonzero(np.asarray(st[0])[:, 0] >= 0))
    return {"ms": 1000.0 * min(times), "num_peaks": num_peaks, "min_distance": min_distance,
            "peaks_found": found, "map": list(scores.shape),
            "what": "PeakCallerMaximumFilter on the device score map after the timed steps, "
                    "best of %d calls" % reps}


def oracle_sample_rate(target, tmpl, score, mask, rots, tf=None, gf=None, seconds=10.0):
    """The oracle (the reference's loop restated on the host cores) on a bounded sample of
    a workload: spawned workers, one pool call of about ``seconds``; rotations/s."""
    from oracle import tm_oracle as O

    w = _host_workers(3.0)
    t0 = time.perf_counter()
    O.scan_parallel(target, tmpl, rots[:w], score, template_mask=mask, template_filter=tf,
                    target_filter=gf, n_workers=w)
    per = time.perf_counter() - t0
    n = int(min(len(rots), max(w, w * int(seconds / max(per, 1e-3)))))
    t0 = time.perf_counter()
    O.scan_parallel(target, tmpl, rots[:n], score, template_mask=mask, template_filter=tf,
                    target_filter=gf, n_workers=w)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "rotations/s", "cores": w, "kind": "port",
            "sample": f"the oracle over {n} rotations in {w} spawned workers ({dt:.1f} s)"}


def leg_config2(precision="mixed", batch=64, cpu=True):
    """Filtered FLC at its workload (256x256x128, 32^3 template, CTF x wedge, the
    1,992-rotation 15-degree set, 64 rotations per launch group), device-timed, with the
    dominant stage's roofline."""
    import torch

    from pytme_b200.filters import Compose, CTFReconstructed, WedgeReconstructed
    from pytme_b200.matching import fourier_padding, rigid_transform_matrices
    from pytme_b200.scores import ScanPlan, _prepare_target

    target, tmpl, mask, rots = make_config2_inputs()
    tf = np.asarray(Compose([WedgeReconstructed(**CONFIG2_WEDGE), CTFReconstructed(
        **CONFIG2_CTF)])(shape=tmpl.shape, return_real_fourier=True)["data"], np.float32)
    gf = np.asarray(Compose([WedgeReconstructed(**CONFIG2_WEDGE)])(
        shape=target.shape, return_real_fourier=True)["data"], np.float32)
    conv, fast, _, _ = fourier_padding(target.shape, tmpl.shape)
    plan = ScanPlan("FLC", fast, tmpl.shape, precision=precision, batch=batch)
    plan.set_template(np.ascontiguousarray(tmpl[::-1, ::-1, ::-1]),
                      np.ascontiguousarray(mask[::-1, ::-1, ::-1]), tf)
    plan.set_target(_prepare_target(target, tuple(fast), gf))
    mats = torch.as_tensor(rigid_transform_matrices(rots, (np.asarray(tmpl.shape) - 1) / 2),
                           device="cuda")
    smax = torch.zeros(fast, dtype=torch.float32, device="cuda")
    sarg = torch.full(fast, -1, dtype=torch.int32, device="cuda")
    for _ in range(3):
        plan.run(mats[:batch], 0, smax, sarg)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    plan.run(mats, 0, smax, sarg)
    e1.record()
    torch.cuda.synchronize()
    plan.check()
    ms = e0.elapsed_time(e1)
    plan.set_timing(True)
    plan.run(mats[:4 * batch], 0, smax, sarg)
    timing = plan.get_timing()
    plan.set_timing(False)
    stages = {k: v for k, v in timing.items() if k != "prepare"}
    dom = max(stages, key=lambda k: stages[k][0])
    avg = stages[dom][0] / max(stages[dom][1], 1)
    alg = plan.stage_bytes(dom, batch)
    peak, peak_kind = measured_peaks()
    plan.close()
    del smax, sarg
    torch.cuda.empty_cache()
    extra = {}
    if cpu:
        extra["cpu_baseline"] = oracle_sample_rate(target, tmpl, "FLC", mask, rots, tf, gf)
    return {**extra, "workload": "FLC, 256x256x128 (40 copies, SNR 0.1), 32^3 template, dilated "
                        "threshold mask, CTF x wedge template filter, wedge target filter, "
                        "15-degree set (1992 rotations)",
            "value": len(rots) / (ms / 1000.0), "unit": "rotations/s", "rotations": len(rots),
            "rotation_batch": batch, "precision": precision,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": alg / (avg / 1000) / 1e9,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": alg / (avg / 1000) / 1e9 / peak, "alg_bytes_per_launch": alg,
                         "avg_launch_ms": avg},
            "stages_ms_per_group": {k: round(v[0] / max(v[1], 1), 3) for k, v in stages.items()}}


def _stage_roofline(plan, mats, batch, groups=2):
    """Roofline of a plan's dominant stage: per-stage CUDA-event timing of ``groups``
    launch groups after one warm-up group."""
    import torch

    shape = plan.fast_shape
    smax = torch.zeros(shape, dtype=torch.float32, device="cuda")
    sarg = torch.full(shape, -1, dtype=torch.int32, device="cuda")
    plan.run(mats[:batch], 0, smax, sarg)
    plan.set_timing(True)
    plan.run(mats[batch:(groups + 1) * batch], batch, smax, sarg)
    timing = plan.get_timing()
    plan.set_timing(False)
    stages = {k: v for k, v in timing.items() if k != "prepare"}
    dom = max(stages, key=lambda k: stages[k][0])
    avg = stages[dom][0] / max(stages[dom][1], 1)
    alg = plan.stage_bytes(dom, batch)
    peak, peak_kind = measured_peaks()
    return {"bound": "hbm", "kernel": dom, "achieved": alg / (avg / 1000) / 1e9, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": alg / (avg / 1000) / 1e9 / peak,
            "alg_bytes_per_launch": alg, "avg_launch_ms": avg}


def leg_config4(precision="mixed", cpu=True):
    """The uneven batch (make_config4_jobs: 36 (tomogram, template) jobs, 12-degree set)
    through scan_batch with the autotuned rotation batch and CUDA-graph replay; the timed
    call includes every job's upload, target set-up, filters and result download."""
    import torch

    from pytme_b200.batch import MatchJob, autotune_batch, scan_batch

    jobs = []
    for kw, t, i in make_config4_jobs():
        tfilt, gfilt = config4_filters(kw["meta"])
        jobs.append(MatchJob(template_filter=tfilt, target_filter=gfilt, **kw))
    t0 = time.perf_counter()
    batches = {}
    for job in jobs:
        batches[(job.target.shape, job.template.shape)] = autotune_batch(job, precision)
    tune_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = scan_batch(jobs, precision=precision, rotation_batch="auto", use_graph=True)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    n = sum(int(j.rotations.shape[0]) for j in jobs)
    assert len(out) == len(jobs)
    del out
    # roofline and CPU baseline on the largest job (320x320x160 with the 40^3 template)
    from pytme_b200.matching import fourier_padding, rigid_transform_matrices
    from pytme_b200.scores import ScanPlan, _prepare_target

    big = max(jobs, key=lambda j: j.target.size * j.template.size)
    tf = np.asarray(big.template_filter(shape=big.template.shape,
                                        return_real_fourier=True)["data"], np.float32)
    gf = np.asarray(big.target_filter(shape=big.target.shape,
                                      return_real_fourier=True)["data"], np.float32)
    _, fast, _, _ = fourier_padding(big.target.shape, big.template.shape)
    b = batches[(big.target.shape, big.template.shape)]
    plan = ScanPlan(big.score, fast, big.template.shape, precision=precision, batch=b)
    try:
        plan.set_template(np.ascontiguousarray(big.template[::-1, ::-1, ::-1]),
                          np.ascontiguousarray(big.mask[::-1, ::-1, ::-1]), tf)
        plan.set_target(_prepare_target(big.target, tuple(fast), gf))
        mats = torch.as_tensor(rigid_transform_matrices(
            big.rotations, (np.asarray(big.template.shape) - 1) / 2), device="cuda")
        roof = _stage_roofline(plan, mats, b)
    finally:
        plan.close()
    torch.cuda.empty_cache()
    extra = {"roofline": dict(roof, job=f"{'x'.join(map(str, big.target.shape))} target, "
                                        f"{big.template.shape[0]}^3 template")}
    if cpu:
        c = oracle_sample_rate(big.target, big.template, big.score, big.mask, big.rotations,
                               tf, gf)
        c["unit"] = "job-rotations/s"
        c["sample"] += " of the largest job"
        extra["cpu_baseline"] = c
    return {**extra, "workload": "36 jobs: 12 tomograms 128^3..320x320x160 x templates 24^3/32^3/40^3, "
                        "per-tomogram CTF (1.5-4.5 um) x wedge (50-65 deg), 12-degree set "
                        "(4344 rotations), FLCSphericalMask",
            "value": n / dt, "unit": "job-rotations/s", "job_rotations": n, "seconds": dt,
            "autotune_s": tune_s, "precision": precision,
            "rotation_batches": sorted({int(b) for b in batches.values()}),
            "timed": "scan_batch on host arrays: uploads, set-up, filters, graph replay, "
                     "downloads"}


def run_profile_case(args):
    """A fixed amount of fused-scan work for profilers: --profile-score (FLCSphericalMask
    by default) with a blob template (48^3 by default) and its spherical mask on an N(0,1)
    target of the given shape, --groups groups of --batch rotations."""
    import torch

    from pytme_b200 import synthetic as syn
    from pytme_b200.matching import rigid_transform_matrices
    from pytme_b200.scores import ScanPlan

    shape = tuple(int(x) for x in args.profile_case.split(","))
    t = args.profile_template or TSIZE
    rng = np.random.default_rng(0)
    tmpl = syn.blob_template(t, rng, sigma=1.5 * t / 16, radius=5.0 * t / 16)
    mask = syn.spherical_mask((t,) * 3, t / 2, center=((t - 1) / 2,) * 3)
    target = rng.normal(size=shape).astype(np.float32)
    plan = ScanPlan(args.profile_score, shape, (t,) * 3, precision=args.precision,
                    batch=args.batch)
    if args.profile_score != "FLC":
        plan.set_xpass(args.xpass)
        plan.set_ypass(args.ypass)
        plan.set_zpass(args.zpass)
    plan.set_template(tmpl[::-1, ::-1, ::-1].copy(),
                      None if args.profile_score == "CC" else mask[::-1, ::-1, ::-1].copy())
    plan.set_target(torch.as_tensor(target, device="cuda"))
    rots = syn.super_fibonacci_rotations(args.batch * args.groups)
    m = torch.as_tensor(rigid_transform_matrices(rots, ((t - 1) / 2,) * 3), device="cuda")
    smax = torch.zeros(shape, device="cuda")
    sarg = torch.full(shape, -1, dtype=torch.int32, device="cuda")
    for g in range(args.groups):
        plan.run(m[g * args.batch:(g + 1) * args.batch], g * args.batch, smax, sarg)
    torch.cuda.synchronize()
    print("profile case done", shape, float(smax.max()))
    return 0


def main():
    args = parse()
    if args.profile_case:
        return run_profile_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
