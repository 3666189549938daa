"""Local refinement of candidate peaks by gradient ascent on the FLC score.

The reference refines one pose at a time with derivative-free SciPy optimisers
(``optimize_match``, tme/matching_optimization.py:1143-1312, over the score classes of
:54-277 and :488-548). Here the objective is the exhaustive FLC of ``flc_scoring``
(tme/matching_scores.py:629-759) evaluated at one pose per peak, so that at the
starting pose it equals the score-map value the scan reported for that peak. Its
gradient with respect to three zyz Euler angles, three shifts and the template
density comes from hand-written CUDA adjoint kernels (``csrc/refine.cu``) behind
``FLCRefineFunction``, a ``torch.autograd.Function``; many peaks are refined at once.

Pose of peak p:

* ``corners[p]`` -- target voxel of template voxel 0 (``score_box_corner`` maps a
  score-map voxel of a "same"-mode result to it);
* ``angles[p]`` -- (a, b, g) in degrees, R = Rz(g) Ry(b) Rz(a), the reference's
  ``euler_to_rotationmatrix`` (tme/rotations.py:171-196);
* ``shifts[p]`` -- sub-voxel translation in the target frame.

Template voxel o samples the template and mask at R^T (o - c - s) + c with
c = (t - 1)/2, the rotation centre of the scan. The particle centre in the target is
``corners + c + shifts``.

The rotated templates are checkpointed: the forward pass keeps only six sums per peak
and the backward pass recomputes the rotation (and the template filter) instead of
reading stored copies.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _native as N
from .matching import TargetSpectrum, _evaluate_filter, fourier_padding
from .scores import _prepare_target, _to_device

__all__ = [
    "EPS",
    "euler_zyz_from_matrix",
    "euler_zyz_to_matrix",
    "score_box_corner",
    "RefineProblem",
    "FLCRefineFunction",
    "refine_score",
    "RefineResult",
    "refine_peaks",
]

EPS = float(np.finfo(np.float32).eps)


# ----------------------------------------------------------------------------- poses
def euler_zyz_to_matrix(angles) -> np.ndarray:
    """R = Rz(g) Ry(b) Rz(a) for (a, b, g) in degrees, float64, shape (..., 3, 3)."""
    a = np.deg2rad(np.asarray(angles, dtype=np.float64))
    ca, sa = np.cos(a[..., 0]), np.sin(a[..., 0])
    cb, sb = np.cos(a[..., 1]), np.sin(a[..., 1])
    cg, sg = np.cos(a[..., 2]), np.sin(a[..., 2])
    r = np.empty(a.shape[:-1] + (3, 3), dtype=np.float64)
    r[..., 0, 0] = cg * cb * ca - sg * sa
    r[..., 0, 1] = -cg * cb * sa - sg * ca
    r[..., 0, 2] = cg * sb
    r[..., 1, 0] = sg * cb * ca + cg * sa
    r[..., 1, 1] = -sg * cb * sa + cg * ca
    r[..., 1, 2] = sg * sb
    r[..., 2, 0] = -sb * ca
    r[..., 2, 1] = sb * sa
    r[..., 2, 2] = cb
    return r


def euler_zyz_from_matrix(rotations) -> np.ndarray:
    """Inverse of ``euler_zyz_to_matrix``: b in [0, 180]; at b = 0 or 180 the first
    angle is set to 0."""
    r = np.asarray(rotations, dtype=np.float64).reshape(-1, 3, 3)
    b = np.arccos(np.clip(r[:, 2, 2], -1.0, 1.0))
    sb = np.sin(b)
    a = np.arctan2(r[:, 2, 1], -r[:, 2, 0])
    g = np.arctan2(r[:, 1, 2], r[:, 0, 2])
    lock = sb < 1e-6
    up = lock & (r[:, 2, 2] > 0)
    down = lock & (r[:, 2, 2] <= 0)
    a = np.where(lock, 0.0, a)
    g = np.where(up, np.arctan2(r[:, 1, 0], r[:, 0, 0]), g)
    g = np.where(down, np.arctan2(-r[:, 0, 1], -r[:, 0, 0]), g)
    out = np.rad2deg(np.stack([a, b, g], axis=-1))
    return out.reshape(np.asarray(rotations).shape[:-2] + (3,))


def score_box_corner(position, target_shape, template_shape) -> np.ndarray:
    """Box corner (target voxel of template voxel 0) of the score-map voxel
    ``position`` of a "same"-mode ``MaxScoreOverRotations.result`` with the target at
    least as large as the template. The scan correlates with the reversed template and
    the result is rolled by ``1 - t//2 - t%2`` (tme/matching_data.py:510-512) and
    cropped from (min(conv, fast) - T) // 2 (tme/matching_utils.py:469-524), which
    puts the box at position + crop start - t//2."""
    conv, fast, _, _ = fourier_padding(target_shape, template_shape)
    start = np.asarray([(min(c, f) - n) // 2 for c, f, n in zip(conv, fast, target_shape)])
    return np.asarray(position, dtype=np.int64) + start - np.asarray(template_shape) // 2


# ----------------------------------------------------------------------------- problem
class _FilterPlan:
    """Batched single-precision cuFFT plan at template shape for ``tm_fft_filter``."""

    def __init__(self, shape, batch: int):
        self.shape = tuple(int(x) for x in shape)
        self.batch = int(batch)
        arr = (N.c_int * 3)(*self.shape)
        h = N.c_void_p()
        N.check(N.lib.tm_fft_plan_create(3, arr, self.batch, 0, N.ctypes.byref(h)),
                "tm_fft_plan_create")
        self._h = h
        self.n_ft = self.shape[0] * self.shape[1] * (self.shape[2] // 2 + 1)

    def apply(self, x: torch.Tensor, spectrum: torch.Tensor, filt: torch.Tensor) -> None:
        N.check(N.lib.tm_fft_filter(self._h, N.ptr(x), N.ptr(spectrum), N.ptr(filt),
                                    N.stream_ptr()), "tm_fft_filter")

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.lib.tm_fft_plan_destroy(self._h)
                self._h = None
        except Exception:
            pass


class RefineProblem:
    """Target, mask and template filter resident on the current GPU.

    ``target`` is filtered once with ``target_filter`` (an array at the rfft shape of
    the scan's transform, or a filter object) exactly as the scan does, and its mean
    is subtracted (the FLC is invariant to an offset of the target; removing it keeps
    the local variance free of cancellation). Boxes that reach past the target see
    the raw target's zero there (minus the mean in the centred frame). ``template_filter`` (array at the
    template's rfft shape, or a filter object) is applied to every rotated template
    at template shape, like the scan with ``pad_template_filter=False``.
    ``max_work_bytes`` bounds the per-call scratch (rotated templates, their
    gradients and spectra); more peaks are processed in chunks.
    """

    def __init__(self, target, template, mask, template_filter=None, target_filter=None,
                 eps: float = EPS, max_work_bytes: int = 2 << 30):
        template = np.asarray(template.detach().cpu() if isinstance(template, torch.Tensor)
                              else template, dtype=np.float32)
        if template.ndim != 3 or tuple(mask.shape) != template.shape:
            raise ValueError("template and mask must be 3D arrays of the same shape")
        tshape = tuple(int(x) for x in target.shape)
        if len(tshape) != 3:
            raise ValueError("target must be a 3D array")
        self.template_shape = tuple(int(x) for x in template.shape)
        self.target_shape = tshape
        _, fast, _, _ = fourier_padding(tshape, self.template_shape)
        spec = TargetSpectrum(target, fast)
        tf = _evaluate_filter(target_filter, fast, data_rfft=spec, weight_type=None)
        padded = _prepare_target(target, tuple(fast), tf)
        tgt = padded[tuple(slice(0, n) for n in tshape)].contiguous()
        mean = tgt.double().mean().float()
        tgt -= mean
        self.target = tgt
        # boxes reaching past the target see the raw target's zero there
        self.outside = -float(mean)
        self.template = _to_device(template)
        self.mask = _to_device(mask)
        self.eps = float(eps)
        filt = _evaluate_filter(template_filter, self.template_shape, data_rfft=spec)
        del spec
        self.template_filter = None if filt is None else _to_device(filt)
        if self.template_filter is not None:
            ft = self.template_shape[:2] + (self.template_shape[2] // 2 + 1,)
            if tuple(self.template_filter.shape) != ft:
                raise ValueError(f"template filter shape {tuple(self.template_filter.shape)} "
                                 f"is not the template's rfft shape {ft}")
        nv = int(np.prod(self.template_shape))
        n_ft = self.template_shape[0] * self.template_shape[1] * (self.template_shape[2] // 2 + 1)
        per_peak = (2 * nv * 4 + n_ft * 8) if self.template_filter is not None else 0
        self.chunk = max(1, int(max_work_bytes // per_peak)) if per_peak else 1 << 30
        self._plans: Dict[int, _FilterPlan] = {}

    @property
    def filtered(self) -> bool:
        return self.template_filter is not None

    @property
    def center(self) -> np.ndarray:
        return (np.asarray(self.template_shape) - 1) / 2.0

    def plan(self, batch: int) -> _FilterPlan:
        p = self._plans.get(batch)
        if p is None:
            p = _FilterPlan(self.template_shape, batch)
            self._plans[batch] = p
        return p

    def desc(self, template: torch.Tensor, rot: torch.Tensor, shifts: torch.Tensor,
             corners: torch.Tensor, lo: int, hi: int) -> N.RefineDesc:
        d = N.RefineDesc()
        d.tmpl = template.data_ptr()
        d.mask = self.mask.data_ptr()
        d.template_shape = (N.c_int * 3)(*self.template_shape)
        d.target = self.target.data_ptr()
        d.target_shape = (N.c_int * 3)(*self.target_shape)
        d.target_outside = self.outside
        d.rot = rot.data_ptr() + lo * 9 * 4
        d.shifts = shifts.data_ptr() + lo * 3 * 4
        d.corners = corners.data_ptr() + lo * 3 * 4
        d.n_peaks = hi - lo
        d.eps = self.eps
        return d

    def chunks(self, P: int):
        for lo in range(0, P, self.chunk):
            yield lo, min(P, lo + self.chunk)


def _filtered_templates(problem: RefineProblem, d, n: int, buf: torch.Tensor,
                        spec: torch.Tensor) -> None:
    """buf[:n] = template filter of the rotated templates of the chunk in ``d``."""
    N.check(N.lib.tm_refine_rotate(N.ctypes.byref(d), N.ptr(buf), N.stream_ptr()),
            "tm_refine_rotate")
    problem.plan(n).apply(buf, spec, problem.template_filter)


def _work(problem: RefineProblem, n: int, dev) -> Tuple[torch.Tensor, torch.Tensor]:
    nv = int(np.prod(problem.template_shape))
    n_ft = problem.plan(n).n_ft
    return (torch.empty((n, nv), dtype=torch.float32, device=dev),
            torch.empty((n, n_ft), dtype=torch.complex64, device=dev))


def _as_f32(x: torch.Tensor, shape) -> torch.Tensor:
    return x.detach().to(dtype=torch.float32).contiguous().reshape(shape)


class FLCRefineFunction(torch.autograd.Function):
    """scores[p] = FLC of peak p at (angles[p], shifts[p]) with template density
    ``template``; backward gives d/d(template), d/d(angles) (per degree) and
    d/d(shifts) (per voxel). ``problem`` and ``corners`` (int32, (P, 3)) are
    constants."""

    @staticmethod
    def forward(ctx, template, angles, shifts, problem: RefineProblem, corners):
        P = int(angles.shape[0])
        dev = problem.target.device
        tmpl = _as_f32(template, (-1,))
        ang = _as_f32(angles, (P, 3))
        sh = _as_f32(shifts, (P, 3))
        cor = corners.to(device=dev, dtype=torch.int32).contiguous()
        rot = torch.empty((P, 9), dtype=torch.float32, device=dev)
        drot = torch.empty((P, 27), dtype=torch.float32, device=dev)
        st = N.stream_ptr()
        N.check(N.lib.tm_euler_zyz(N.ptr(ang), P, N.ptr(rot), N.ptr(drot), st), "tm_euler_zyz")
        sums = torch.empty((P, 6), dtype=torch.float64, device=dev)
        scores = torch.empty((P,), dtype=torch.float32, device=dev)
        for lo, hi in problem.chunks(P):
            d = problem.desc(tmpl, rot, sh, cor, lo, hi)
            tf = None
            if problem.filtered:
                tf, spec = _work(problem, hi - lo, dev)
                _filtered_templates(problem, d, hi - lo, tf, spec)
            N.check(N.lib.tm_refine_forward(N.ctypes.byref(d), N.ptr(tf), N.ptr(sums[lo:hi]),
                                            N.ptr(scores[lo:hi]), st), "tm_refine_forward")
        ctx.problem = problem
        ctx.save_for_backward(tmpl, sh, cor, rot, drot, sums)
        ctx.template_shape = tuple(template.shape)
        return scores

    @staticmethod
    def backward(ctx, grad_scores):
        problem: RefineProblem = ctx.problem
        tmpl, sh, cor, rot, drot, sums = ctx.saved_tensors
        P = int(sums.shape[0])
        dev = sums.device
        g = grad_scores.detach().to(dtype=torch.float32).contiguous()
        g_ang = torch.zeros((P, 3), dtype=torch.float64, device=dev)
        g_sh = torch.zeros((P, 3), dtype=torch.float64, device=dev)
        g_t = torch.zeros(tmpl.shape, dtype=torch.float32, device=dev) \
            if ctx.needs_input_grad[0] else None
        st = N.stream_ptr()
        for lo, hi in problem.chunks(P):
            d = problem.desc(tmpl, rot, sh, cor, lo, hi)
            tf = gbuf = None
            if problem.filtered:
                tf, spec = _work(problem, hi - lo, dev)
                _filtered_templates(problem, d, hi - lo, tf, spec)
                gbuf = torch.empty_like(tf)
                N.check(N.lib.tm_refine_grad_filtered(N.ctypes.byref(d), N.ptr(tf),
                                                      N.ptr(sums[lo:hi]), N.ptr(g[lo:hi]),
                                                      N.ptr(gbuf), st),
                        "tm_refine_grad_filtered")
                problem.plan(hi - lo).apply(gbuf, spec, problem.template_filter)
            N.check(N.lib.tm_refine_backward(N.ctypes.byref(d), N.ptr(tf), N.ptr(gbuf),
                                             N.ptr(sums[lo:hi]), N.ptr(g[lo:hi]),
                                             N.ptr(drot[lo:hi]), None, N.ptr(g_sh[lo:hi]),
                                             N.ptr(g_ang[lo:hi]), N.ptr(g_t), st),
                    "tm_refine_backward")
        gt = None if g_t is None else g_t.reshape(ctx.template_shape)
        return gt, g_ang.to(torch.float32), g_sh.to(torch.float32), None, None


def refine_score(problem: RefineProblem, corners, angles, shifts=None,
                 template: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Differentiable FLC scores (P,) of the given poses."""
    dev = problem.target.device
    angles = torch.as_tensor(angles, dtype=torch.float32, device=dev)
    if shifts is None:
        shifts = torch.zeros_like(angles)
    shifts = torch.as_tensor(shifts, dtype=torch.float32, device=dev)
    corners = torch.as_tensor(np.asarray(corners) if not isinstance(corners, torch.Tensor)
                              else corners, dtype=torch.int32, device=dev)
    tmpl = problem.template if template is None else template
    return FLCRefineFunction.apply(tmpl, angles, shifts, problem, corners)


@dataclass
class RefineResult:
    """Best pose per peak over the optimisation (scores at the returned poses)."""

    corners: np.ndarray        # (P, 3) int
    angles: np.ndarray         # (P, 3) degrees, zyz
    shifts: np.ndarray         # (P, 3) voxels
    scores: np.ndarray         # (P,)
    initial_scores: np.ndarray  # (P,)
    positions: np.ndarray      # (P, 3) particle centres in the target: corner + c + shift
    rotations: np.ndarray      # (P, 3, 3)
    steps: int


def refine_peaks(problem: RefineProblem, corners, angles, shifts=None, steps: int = 50,
                 lr_angle: float = 0.5, lr_shift: float = 0.1, recenter: bool = True,
                 template: Optional[torch.Tensor] = None) -> RefineResult:
    """Maximise every peak's FLC with ``steps`` Adam steps on (angles, shifts).

    Angles are in degrees and shifts in voxels; the learning rates are Adam step
    sizes in those units, decayed by a cosine from 1 to 0.1 over the steps. With ``recenter`` the integer part of a shift moves into
    the box corner after each step, so the box follows the particle. The best pose
    seen for each peak is returned (a step may overshoot).
    """
    dev = problem.target.device
    ang = torch.tensor(np.asarray(angles, dtype=np.float32).reshape(-1, 3), device=dev,
                       requires_grad=True)
    P = int(ang.shape[0])
    sh0 = np.zeros((P, 3), np.float32) if shifts is None else np.asarray(shifts, np.float32)
    sh = torch.tensor(sh0.reshape(P, 3), device=dev, requires_grad=True)
    cor = torch.as_tensor(np.asarray(corners).reshape(P, 3), dtype=torch.int32,
                          device=dev).clone()
    tmpl = problem.template if template is None else template
    opt = torch.optim.Adam([{"params": [ang], "lr": lr_angle},
                            {"params": [sh], "lr": lr_shift}])
    base = (lr_angle, lr_shift)
    best = torch.full((P,), -math.inf, dtype=torch.float32, device=dev)
    best_ang = ang.detach().clone()
    best_sh = sh.detach().clone()
    best_cor = cor.clone()
    initial = None
    for it in range(steps + 1):
        opt.zero_grad(set_to_none=True)
        s = FLCRefineFunction.apply(tmpl, ang, sh, problem, cor)
        with torch.no_grad():
            if initial is None:
                initial = s.detach().clone()
            better = s > best
            best = torch.where(better, s, best)
            best_ang[better] = ang[better]
            best_sh[better] = sh[better]
            best_cor[better] = cor[better]
        if it == steps:
            break
        (-s.sum()).backward()
        decay = 0.1 + 0.45 * (1.0 + math.cos(math.pi * it / max(steps, 1)))
        for grp, lr in zip(opt.param_groups, base):
            grp["lr"] = lr * decay
        opt.step()
        if recenter:
            with torch.no_grad():
                r = torch.round(sh)
                cor += r.to(torch.int32)
                sh -= r
    c = problem.center
    out_ang = best_ang.cpu().numpy().astype(np.float64)
    out_sh = best_sh.cpu().numpy().astype(np.float64)
    out_cor = best_cor.cpu().numpy().astype(np.int64)
    return RefineResult(corners=out_cor, angles=out_ang, shifts=out_sh,
                        scores=best.cpu().numpy(), initial_scores=initial.cpu().numpy(),
                        positions=out_cor + c + out_sh,
                        rotations=euler_zyz_to_matrix(out_ang), steps=steps)
