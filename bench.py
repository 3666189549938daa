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
    ap.add_argument("--xpass", choices=("auto", "tensor", "fft"), default="auto",
                    help="x pass on the tensor cores, as CUDA-core FFTs, or the plan default "
                         "(tensor cores for mixed precision)")
    ap.add_argument("--plain-rotations", type=int, default=12)
    ap.add_argument("--e2e-rotations", type=int, default=0,
                    help="rotations per end-to-end call (0: the whole set)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--small", action="store_true", help="128x128x64 / 24^3 quick check")
    ap.add_argument("--profile-case", default=None, metavar="N0,N1,N2",
                    help="run --groups launch groups of the fused scan on a target of this "
                         "shape and exit (a small case for ncu captures; no timing, no JSON)")
    ap.add_argument("--groups", type=int, default=2)
    return ap.parse_args()


def make_inputs(small=False):
    from pytme_b200 import synthetic as syn

    rng = np.random.default_rng(2024)
    shape = (128, 128, 64) if small else SHAPE
    t = 24 if small else TSIZE
    tmpl = syn.blob_template(t, rng, n_blobs=6, sigma=1.5 * t / 16, radius=5.0 * t / 16)
    c = (t - 1) / 2.0
    mask = syn.spherical_mask((t, t, t), t / 2, center=(c, c, c))
    target, _, _ = syn.make_tomogram(shape, tmpl, 20 if small else 300, rng, snr=0.05, mask=mask)
    rots = syn.rotations_for_angle(ANGLE)
    return target, tmpl, mask, rots


# DRAM bytes (read + write) of one launch of a pass of the benchmark configuration
# (512x512x200, 48^3 template, mixed precision, 32 rotations per group) from ncu captures
# of smaller launches of the same kernels, scaled to it: x and y passes from 512x512x48
# targets (by columns, rotations and row pitch), the z pass from a 256x256x200 target (by
# rows). Keyed by (pass, precision, rotations per group, variant of the pass).
NCU_TRAFFIC = {("xpass", "mixed", 32, "fft"): 3.91e9, ("xpass", "mixed", 32, "tensor"): 4.18e9,
               ("ypass", "mixed", 32, "fft"): 6.81e9, ("zpass", "mixed", 32, "tensor"): 4.23e9}


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


def cpu_oracle_rate(target, tmpl, mask, rots, seconds, cores=None):
    """The oracle scan on host cores (spawned workers over rotation chunks); returns
    (rotations/s of the scoring loop, cores, sample description)."""
    import multiprocessing as mp

    import psutil

    cores = cores or os.cpu_count() or 1
    # each process holds about 3 GB of full-size arrays during setup
    by_mem = int(psutil.virtual_memory().available // (3 * 1024 ** 3))
    cores = max(1, min(cores, 32, by_mem))
    # per-rotation cost ~2.3 s on one core at this size; size the sample for `seconds`
    per_worker = max(1, int(round(seconds / 2.5)))
    n = cores * per_worker
    sample = np.ascontiguousarray(rots[:n])
    from oracle import tm_oracle as O

    ctx = mp.get_context("spawn")
    chunks = [(target, tmpl, mask, sample[i * per_worker:(i + 1) * per_worker])
              for i in range(cores)]
    with ctx.Pool(cores) as pool:
        outs = pool.map(_cpu_chunk, chunks)
    loop = max(o[1] for o in outs)
    setup = max(o[0] for o in outs)
    desc = (f"{n} rotations of the 7-degree set on the full 512x512x200 map, {cores} "
            f"processes x {per_worker} rotations; scoring loop {loop:.1f} s, per-process "
            f"setup {setup:.1f} s excluded")
    return n / loop, cores, desc


def _cpu_chunk(args):
    target, tmpl, mask, rots = args
    from oracle import tm_oracle as O

    t0 = time.perf_counter()
    O.scan(target, tmpl, rots[:0], "FLCSphericalMask", template_mask=mask)
    t1 = time.perf_counter()
    O.scan(target, tmpl, rots, "FLCSphericalMask", template_mask=mask)
    t2 = time.perf_counter()
    return t1 - t0, (t2 - t1) - (t1 - t0)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    target, tmpl, mask, rots = make_inputs(args.small)
    steps = max(1, args.steps)
    rates = []
    cores = None
    desc = ""
    secs = max(5.0, min(args.cpu_seconds, 120.0 / (steps + args.warmup)))
    for i in range(args.warmup + steps):
        r, cores, desc = cpu_oracle_rate(target, tmpl, mask, rots[i * 7 % 1000:], secs)
        if i >= args.warmup:
            rates.append(r)
    value = float(np.median(rates))
    line = {
        "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "step": "one rotation per step (rate of the sample)"},
        "cpu_baseline": {"value": value, "unit": "rotations/s", "cores": cores,
                         "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "rotations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


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

        result = {
            "metric": METRIC, "value": value, "unit": "rotations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f32 (f16 spectra, f64 denominator)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD + ("" if not args.small else " [small]"),
                       "step_rotations": R, "rotation_batch": args.batch,
                       "precision": args.precision, "xpass": plan.xpass,
                       "zpass": plan.zpass,
                       "l2": "inputs larger than L2 (target spectrum 212 MB, state 420 MB)",
                       "fast_shape": list(fast), "template": [TSIZE] * 3},
            "voxel_rotations_per_s": value * float(np.prod(fast)),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": NCU_TRAFFIC.get((dom, args.precision, args.batch,
                                                     {"xpass": plan.xpass, "zpass": plan.zpass}
                                                     .get(dom, "fft")))
                         if not args.small else None,
                         "alg_bytes_per_launch": alg,
                         "avg_launch_ms": avg_ms},
            "stages": stages,
            "plain": {"value": plain_rate, "unit": "rotations/s", "rotations": args.plain_rotations,
                      "path": "fp32, one rotation at a time, full cuFFT r2c/c2r"},
            "vs_plain": value / world / plain_rate,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
    # end-to-end through the public API with host arrays (rank 0)
    if rank == 0 and not args.no_e2e:
        n_e2e = args.e2e_rotations or n_rot
        P.backend.change_backend("b200", precision=args.precision, rotation_batch=args.batch,
                                 xpass=args.xpass, zpass=args.zpass)
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
    if rank == 0 and not args.no_cpu:
        r, cores, desc = cpu_oracle_rate(target, tmpl, mask, rots, args.cpu_seconds)
        result["cpu_baseline"] = {"value": r, "unit": "rotations/s", "cores": cores,
                                  "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_profile_case(args):
    """A fixed amount of fused-scan work for profilers: FLCSphericalMask with a 48^3
    blob template on an N(0,1) target of the given shape, --groups groups of --batch
    rotations."""
    import torch

    from pytme_b200 import synthetic as syn
    from pytme_b200.matching import rigid_transform_matrices
    from pytme_b200.scores import ScanPlan

    shape = tuple(int(x) for x in args.profile_case.split(","))
    t = TSIZE
    rng = np.random.default_rng(0)
    tmpl = syn.blob_template(t, rng, sigma=1.5 * t / 16, radius=5.0 * t / 16)
    mask = syn.spherical_mask((t,) * 3, t / 2, center=((t - 1) / 2,) * 3)
    target = rng.normal(size=shape).astype(np.float32)
    plan = ScanPlan("FLCSphericalMask", shape, (t,) * 3, precision=args.precision,
                    batch=args.batch)
    plan.set_xpass(args.xpass)
    plan.set_zpass(args.zpass)
    plan.set_template(tmpl[::-1, ::-1, ::-1].copy(), mask[::-1, ::-1, ::-1].copy())
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
