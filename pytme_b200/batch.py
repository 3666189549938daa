"""Many (tomogram, template) jobs of different sizes, and the rotation-batch autotuner.

``scan_batch`` runs a list of jobs, each a target with its own template, mask,
filters and rotation set. Jobs that share a score, transform shape and template shape
reuse one ``ScanPlan`` (its spectra, scratch and cuFFT plans); each job only uploads
its target and template. Full launch groups replay one captured CUDA graph per plan.
Results come back per job in the reference's ``MaxScoreOverRotations.result``
layout.

``autotune_plan`` times the plan's configurations on the real target: candidate
rotations-per-launch-group values, and for each the form of every pass (tensor cores or
FFTs for the x, y and z passes, a coordinate search from the plan's default), and caches
the fastest per (GPU, score, shapes, precision) in a JSON file (``$PYTME_B200_CACHE`` or
``~/.cache/pytme_b200/autotune.json``). ``autotune_batch`` returns its rotation batch.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .matching import (TargetSpectrum, _evaluate_filter, apply_convolution_mode,
                       fourier_padding, rigid_transform_matrices)
from .scores import ScanPlan, _prepare_target

__all__ = ["MatchJob", "scan_batch", "autotune_batch", "autotune_plan"]

_PASSES = ("xpass", "ypass", "zpass")


@dataclass
class MatchJob:
    """One exhaustive search: target, template (as given, not reversed), optional
    mask, rotations (n, 3, 3), optional filters (arrays at the template's and the
    transform's rfft shapes, or filter objects; CTFs and continuous wedges are then
    built on the GPU) and the template rotation order (3, the reference's default, or
    1)."""

    target: np.ndarray
    template: np.ndarray
    rotations: np.ndarray
    mask: Optional[np.ndarray] = None
    score: str = "FLCSphericalMask"
    template_filter: Optional[object] = None
    target_filter: Optional[object] = None
    score_threshold: float = 0.0
    interpolation_order: int = 3
    meta: Dict = field(default_factory=dict)


def _cache_path() -> str:
    return os.environ.get("PYTME_B200_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "pytme_b200",
                                       "autotune.json"))


def _cache_load() -> Dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _cache_store(data: Dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    except OSError:
        pass


def _key(score, fast, tshape, precision) -> str:
    name = torch.cuda.get_device_name(torch.cuda.current_device())
    return f"{name}|{score}|{'x'.join(map(str, fast))}|{'x'.join(map(str, tshape))}|{precision}"


def _time_groups(plan, mats, b, groups, smax, sarg) -> float:
    """Rotations per second of ``groups`` launch groups after one warm-up group."""
    n = b * (groups + 1)
    plan.run(mats[:b], 0, smax, sarg)  # warm-up group
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    plan.run(mats[b:n], b, smax, sarg)
    e1.record()
    torch.cuda.synchronize()
    return (n - b) / (e0.elapsed_time(e1) / 1000.0)


def _apply_passes(plan, config: Dict) -> None:
    for name in _PASSES:
        getattr(plan, "set_" + name)(config.get(name, "auto"))


def autotune_plan(job: MatchJob, precision: str = "mixed",
                  candidates: Sequence[int] = (8, 16, 32, 64), groups: int = 2,
                  use_cache: bool = True) -> Dict:
    """Fastest plan configuration for this job's shapes (device-timed): the rotation
    batch and, per batch, the x, y and z pass forms found by a coordinate search from the
    plan's defaults (each pass's other form is kept when it is faster). Returns
    ``{"batch": B, "xpass": ..., "ypass": ..., "zpass": ..., "rate": rotations/s}``."""
    conv, fast, fast_ft, shift = fourier_padding(job.target.shape, job.template.shape)
    key = _key(job.score, fast, job.template.shape, precision)
    cache = _cache_load() if use_cache else {}
    hit = cache.get(key)
    if isinstance(hit, dict) and "batch" in hit:
        return dict(hit)
    t_rev = np.ascontiguousarray(job.template[::-1, ::-1, ::-1], dtype=np.float32)
    m_rev = None if job.mask is None else np.ascontiguousarray(job.mask[::-1, ::-1, ::-1],
                                                                   dtype=np.float32)
    spec = TargetSpectrum(job.target, tuple(fast))
    tf = _evaluate_filter(job.template_filter, job.template.shape, data_rfft=spec)
    gf = _evaluate_filter(job.target_filter, tuple(fast), data_rfft=spec, weight_type=None)
    del spec
    target = _prepare_target(job.target, tuple(fast), gf)
    center = np.divide(np.asarray(job.template.shape) - 1, 2)
    dev = target.device
    best: Optional[Dict] = None
    for b in candidates:
        try:
            plan = ScanPlan(job.score, fast, job.template.shape, precision=precision, batch=b)
        except MemoryError:
            continue
        try:
            if plan.plain:
                return {"batch": int(candidates[0]), "rate": 0.0}
            plan.set_template(t_rev, m_rev, tf)
            plan.set_interpolation(job.interpolation_order)
            plan.set_target(target)
            n = b * (groups + 1)
            rots = np.resize(np.asarray(job.rotations, dtype=np.float32).reshape(-1, 3, 3),
                             (n, 3, 3))
            mats = torch.as_tensor(rigid_transform_matrices(rots, center), device=dev)
            smax = torch.zeros(tuple(fast), dtype=torch.float32, device=dev)
            sarg = torch.full(tuple(fast), -1, dtype=torch.int32, device=dev)
            config = {name: getattr(plan, name) for name in _PASSES}
            rate = _time_groups(plan, mats, b, groups, smax, sarg)
            for name in _PASSES:
                other = "fft" if config[name] == "tensor" else "tensor"
                trial = dict(config, **{name: other})
                try:
                    _apply_passes(plan, trial)
                except (NotImplementedError, ValueError):
                    _apply_passes(plan, config)
                    continue
                r = _time_groups(plan, mats, b, groups, smax, sarg)
                if r > rate:
                    config, rate = trial, r
                _apply_passes(plan, config)
            del smax, sarg
        finally:
            plan.close()
        if best is None or rate > best["rate"]:
            best = dict(config, batch=int(b), rate=float(rate))
    if best is None:
        best = {"batch": int(candidates[0]), "rate": 0.0}
    if use_cache:
        cache = _cache_load()
        cache[key] = best
        _cache_store(cache)
    return dict(best)


def autotune_batch(job: MatchJob, precision: str = "mixed",
                   candidates: Sequence[int] = (8, 16, 32, 64), groups: int = 2,
                   use_cache: bool = True) -> int:
    """Fastest rotations-per-launch-group for this job's shapes (``autotune_plan``)."""
    return int(autotune_plan(job, precision, candidates, groups, use_cache)["batch"])


def scan_batch(jobs: List[MatchJob], precision: str = "mixed", rotation_batch="auto",
               use_graph: bool = True) -> List[Tuple[np.ndarray, np.ndarray]]:
    """Run every job; returns [(scores, rotation_index)] in the reference's ``result``
    layout (rolled by the Fourier shift and cropped to the target, "same" mode)."""
    plans: Dict[Tuple, ScanPlan] = {}
    out = []
    try:
        for job in jobs:
            tmpl = np.asarray(job.template, dtype=np.float32)
            conv, fast, fast_ft, shift = fourier_padding(job.target.shape, tmpl.shape)
            has_filter = job.template_filter is not None
            key = (job.score, tuple(fast), tmpl.shape, has_filter)
            plan = plans.get(key)
            if plan is None:
                b, config = rotation_batch, {}
                if b == "auto":
                    config = autotune_plan(job, precision=precision)
                    b = config["batch"]
                plan = ScanPlan(job.score, fast, tmpl.shape, precision=precision, batch=int(b))
                if not plan.plain:
                    _apply_passes(plan, config)
                if use_graph:
                    plan.set_graph(True)
                plans[key] = plan
            t_rev = np.ascontiguousarray(tmpl[::-1, ::-1, ::-1])
            m_rev = None if job.mask is None else np.ascontiguousarray(
                np.asarray(job.mask, dtype=np.float32)[::-1, ::-1, ::-1])
            spec = TargetSpectrum(job.target, tuple(fast))
            plan.set_template(t_rev, m_rev, _evaluate_filter(job.template_filter, tmpl.shape,
                                                             data_rfft=spec))
            plan.set_interpolation(job.interpolation_order)
            gf = _evaluate_filter(job.target_filter, tuple(fast), data_rfft=spec,
                                  weight_type=None)
            del spec
            target = _prepare_target(job.target, tuple(fast), gf)
            plan.set_target(target)
            dev = target.device
            smax = torch.full(tuple(fast), float(job.score_threshold), dtype=torch.float32,
                              device=dev)
            sarg = torch.full(tuple(fast), -1, dtype=torch.int32, device=dev)
            center = np.divide(np.asarray(tmpl.shape) - 1, 2)
            mats = torch.as_tensor(rigid_transform_matrices(job.rotations, center), device=dev)
            plan.run(mats, 0, smax, sarg)
            axis = tuple(range(3))
            s = torch.roll(smax, shifts=shift, dims=axis)
            r = torch.roll(sarg, shifts=shift, dims=axis)
            s = apply_convolution_mode(s, "same", job.target.shape, tmpl.shape, conv)
            r = apply_convolution_mode(r, "same", job.target.shape, tmpl.shape, conv)
            out.append((s.contiguous().cpu().numpy(), r.contiguous().cpu().numpy()))
    finally:
        for p in plans.values():
            p.close()
    return out
