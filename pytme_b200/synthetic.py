"""Seeded synthetic tomograms, templates, masks and rotation sets.

No public dataset is named for the exhaustive-matching benchmarks, so these
generators stand in for tomograms: Gaussian noise with rotated copies of a
blob template inserted at random integer positions, at a stated amplitude or
signal-to-noise ratio. Everything is driven by ``numpy.random.default_rng(seed)``
so tests, fixtures and the benchmark see identical inputs.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

__all__ = [
    "blob_template",
    "spherical_mask",
    "dilated_threshold_mask",
    "random_rotation_matrices",
    "super_fibonacci_rotations",
    "rotation_count_for_angle",
    "rotations_for_angle",
    "insert_copies",
    "make_tomogram",
]


def blob_template(n: int, rng: np.random.Generator, n_blobs: int = 6,
                  sigma: float = 1.5, radius: float = 5.0) -> np.ndarray:
    """Sum of isotropic Gaussians whose centres lie within ``radius`` of the cube centre."""
    grid = np.indices((n, n, n), dtype=np.float64)
    centre = (n - 1) / 2.0
    out = np.zeros((n, n, n), dtype=np.float64)
    for _ in range(n_blobs):
        v = rng.normal(size=3)
        v = v / np.linalg.norm(v) * rng.uniform(0, radius)
        p = centre + v
        d2 = ((grid - p[:, None, None, None]) ** 2).sum(0)
        out += np.exp(-d2 / (2 * sigma * sigma))
    return out.astype(np.float32)


def spherical_mask(shape: Tuple[int, ...], radius: float, center=None) -> np.ndarray:
    """Binary ball, ``|x - c| / r <= 1`` (the reference's elliptical mask with equal radii,
    ``tme/matching_utils.py:765-842``)."""
    shape = tuple(int(x) for x in shape)
    if center is None:
        center = tuple(x // 2 for x in shape)
    center = np.asarray(center, dtype=np.float32).reshape((-1,) + (1,) * len(shape))
    idx = np.indices(shape, dtype=np.float32) - center
    dist = np.linalg.norm(idx / np.float32(radius), axis=0)
    return (dist <= 1).astype(np.float32)


def dilated_threshold_mask(template: np.ndarray, threshold: float = 0.1,
                           dilation: int = 2) -> np.ndarray:
    """``template > threshold * max`` dilated by ``dilation`` voxels (6-connected steps)."""
    from scipy.ndimage import binary_dilation

    m = template > threshold * template.max()
    if dilation > 0:
        m = binary_dilation(m, iterations=int(dilation))
    return m.astype(np.float32)


def _quat_to_matrix(q: np.ndarray) -> np.ndarray:
    q = q / np.linalg.norm(q, axis=-1, keepdims=True)
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    m = np.empty(q.shape[:-1] + (3, 3), dtype=np.float64)
    m[..., 0, 0] = 1 - 2 * (y * y + z * z)
    m[..., 0, 1] = 2 * (x * y - z * w)
    m[..., 0, 2] = 2 * (x * z + y * w)
    m[..., 1, 0] = 2 * (x * y + z * w)
    m[..., 1, 1] = 1 - 2 * (x * x + z * z)
    m[..., 1, 2] = 2 * (y * z - x * w)
    m[..., 2, 0] = 2 * (x * z - y * w)
    m[..., 2, 1] = 2 * (y * z + x * w)
    m[..., 2, 2] = 1 - 2 * (x * x + y * y)
    return m


def random_rotation_matrices(n: int, rng: np.random.Generator) -> np.ndarray:
    """Haar-uniform random rotations from normalised Gaussian quaternions (float32)."""
    q = rng.normal(size=(n, 4))
    return _quat_to_matrix(q).astype(np.float32)


def super_fibonacci_rotations(n: int) -> np.ndarray:
    """Deterministic near-uniform SO(3) sampling with ``n`` rotations (float32).

    Super-Fibonacci spirals (M. Alexa, "Super-Fibonacci Spirals: Fast, Low-Discrepancy
    Sampling of SO(3)", CVPR 2022): sample ``i`` is the unit quaternion
    ``(r sin a, r cos a, R sin b, R cos b)`` with ``s = i + 1/2``, ``r = sqrt(s/n)``,
    ``R = sqrt(1 - s/n)``, ``a = 2 pi s / phi``, ``b = 2 pi s / psi``, ``phi = sqrt(2)`` and
    ``psi`` the real root of ``psi^4 = psi + 4``.
    """
    phi = math.sqrt(2.0)
    psi = 1.533751168755204288118041
    s = np.arange(n, dtype=np.float64) + 0.5
    r = np.sqrt(s / n)
    rr = np.sqrt(1.0 - s / n)
    a = 2.0 * math.pi * s / phi
    b = 2.0 * math.pi * s / psi
    q = np.stack([r * np.sin(a), r * np.cos(a), rr * np.sin(b), rr * np.cos(b)], axis=-1)
    return _quat_to_matrix(q).astype(np.float32)


# (step in degrees, number of rotations) of the reference's precomputed quaternion
# sets, in the order of tme/data/metadata.yaml. The reference picks the set whose
# step is nearest to the request, the first listed on a tie
# (tme/rotations.py:266-299). Only the counts are reproduced here; the matrices
# themselves come from ``super_fibonacci_rotations``.
_REFERENCE_SET_SIZES = (
    (9.72, 7416), (8.17, 12648), (36.47, 216), (62.8, 24), (6.6, 27672),
    (6.48, 28824), (5.75, 39384), (12.29, 4344), (5.27, 53256), (20.83, 648),
    (4.71, 70728), (4.37, 89592), (4.0, 113976), (3.74, 141096), (3.53, 170664),
    (7.4, 19560), (16.29, 1992), (3.26, 207576), (44.48, 60), (27.78, 360),
)


def rotation_count_for_angle(angle: float) -> int:
    """Number of rotations the reference samples at an ``angle`` degree step."""
    best = min(_REFERENCE_SET_SIZES, key=lambda e: abs(angle - e[0]))
    return best[1]


def rotations_for_angle(angle: float) -> np.ndarray:
    return super_fibonacci_rotations(rotation_count_for_angle(angle))


def insert_copies(target: np.ndarray, template: np.ndarray, n_copies: int,
                  amplitude: float, rng: np.random.Generator):
    """Add ``n_copies`` randomly rotated copies of ``template`` times ``amplitude``.

    Copies are rotated about the template centre with order-1 interpolation and
    placed at uniform random integer corner positions that keep them inside the
    target. Returns the corner positions and rotation matrices.
    """
    from scipy.ndimage import affine_transform

    t = np.asarray(template.shape)
    c = (t - 1) / 2.0
    rots = random_rotation_matrices(n_copies, rng)
    hi = np.asarray(target.shape) - t
    pos = np.stack([rng.integers(0, max(int(h), 0) + 1, size=n_copies) for h in hi], axis=1)
    for i in range(n_copies):
        rinv = rots[i].T.astype(np.float64)
        offset = c - rinv @ c
        rotated = affine_transform(template.astype(np.float64), rinv, offset=offset,
                                   order=1, mode="constant")
        sl = tuple(slice(int(p), int(p) + int(s)) for p, s in zip(pos[i], t))
        target[sl] += (amplitude * rotated).astype(target.dtype)
    return pos, rots


def make_tomogram(shape, template: np.ndarray, n_copies: int, rng: np.random.Generator,
                  scale: float = None, snr: float = None, mask: np.ndarray = None):
    """N(0,1) noise plus ``n_copies`` rotated template copies.

    The copy amplitude is ``scale`` if given, else chosen so that the template's
    variance inside ``mask`` times amplitude^2 equals ``snr`` (noise variance 1).
    """
    target = rng.normal(size=tuple(shape)).astype(np.float32)
    if scale is None:
        m = np.ones_like(template) if mask is None else mask
        sel = template[m > 0]
        var = float(sel.var()) if sel.size else 1.0
        scale = math.sqrt(float(snr) / max(var, 1e-30))
    pos, rots = insert_copies(target, template, n_copies, scale, rng)
    return target, pos, rots
