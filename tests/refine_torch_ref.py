"""Plain PyTorch autograd composition of the local-refinement FLC score (test helper).

The same objective as ``pytme_b200.refine`` written with differentiable torch ops in
float64: zyz Euler angles to a rotation matrix, order-1 sampling of the template and
mask at R^T (o - c - s) + c (zero unless every coordinate is inside [0, t - 1]), the
template filter as rfftn -> multiply -> irfftn at template shape, masked
normalisation (tme/matching_utils.py:61-99) and ``norm_scores``
(tme/backends/npfftw_backend.py:537-587). Autograd through this composition is the
reference the CUDA adjoint is checked against.
"""
from __future__ import annotations

import math

import torch

EPS = 1.1920928955078125e-07


def euler_zyz(angles: torch.Tensor) -> torch.Tensor:
    a = angles * (math.pi / 180.0)
    ca, sa = torch.cos(a[:, 0]), torch.sin(a[:, 0])
    cb, sb = torch.cos(a[:, 1]), torch.sin(a[:, 1])
    cg, sg = torch.cos(a[:, 2]), torch.sin(a[:, 2])
    rows = [
        torch.stack([cg * cb * ca - sg * sa, -cg * cb * sa - sg * ca, cg * sb], -1),
        torch.stack([sg * cb * ca + cg * sa, -sg * cb * sa + cg * ca, sg * sb], -1),
        torch.stack([-sb * ca, sb * sa, cb], -1),
    ]
    return torch.stack(rows, -2)


def flc_scores(target, template, mask, corners, angles, shifts, template_filter=None,
               eps: float = EPS) -> torch.Tensor:
    """(P,) scores; all tensors float64 on one device, corners int64 (P, 3)."""
    dev = template.device
    t = torch.tensor(template.shape, device=dev)
    tshape = tuple(template.shape)
    c = (t.double() - 1) / 2
    grid = torch.stack(torch.meshgrid(*[torch.arange(n, device=dev) for n in tshape],
                                      indexing="ij"), -1).reshape(-1, 3)
    R = euler_zyz(angles)
    d = grid[None].double() - c - shifts[:, None, :]
    u = torch.einsum("pji,pvj->pvi", R, d) + c
    inside = ((u >= 0) & (u <= (t - 1).double())).all(-1)
    lo = torch.floor(u).detach()
    f = u - lo
    lo = lo.long().clamp(min=0)
    lo = torch.minimum(lo, t - 1)
    hi = torch.minimum(lo + 1, t - 1)
    tflat, mflat = template.reshape(-1), mask.reshape(-1)
    tr = torch.zeros(u.shape[:2], dtype=torch.float64, device=dev)
    mr = torch.zeros_like(tr)
    for q in range(8):
        b = [(q >> 2) & 1, (q >> 1) & 1, q & 1]
        idx = [hi[..., a] if b[a] else lo[..., a] for a in range(3)]
        w = 1.0
        for a in range(3):
            w = w * (f[..., a] if b[a] else 1 - f[..., a])
        lin = (idx[0] * tshape[1] + idx[1]) * tshape[2] + idx[2]
        tr = tr + w * tflat[lin]
        mr = mr + w * mflat[lin]
    tr = tr * inside
    mr = mr * inside
    P = tr.shape[0]
    if template_filter is not None:
        spec = torch.fft.rfftn(tr.reshape((P,) + tshape), dim=(1, 2, 3))
        tr = torch.fft.irfftn(spec * template_filter, s=tshape, dim=(1, 2, 3)).reshape(P, -1)
    pos = corners[:, None, :] + grid[None]
    n = torch.tensor(target.shape, device=dev)
    ok = ((pos >= 0) & (pos < n)).all(-1)
    posc = torch.minimum(pos.clamp(min=0), n - 1)
    fbox = target[posc[..., 0], posc[..., 1], posc[..., 2]] * ok
    n_obs = mr.sum(1)
    mean = (tr * mr).sum(1) / n_obs
    var_t = torch.clamp((tr * tr * mr).sum(1) / n_obs - mean * mean, min=0)
    tn = (tr - mean[:, None]) / torch.sqrt(var_t)[:, None] * mr
    numerator = (tn * fbox).sum(1)
    e1 = (fbox * mr).sum(1) / n_obs
    e2 = (fbox * fbox * mr).sum(1) / n_obs
    sd = torch.sqrt(torch.clamp(e2 - e1 * e1, min=0))
    sd = torch.where(sd < eps, torch.ones_like(sd), sd)
    return numerator / (sd * n_obs)
