"""Rotation sets of the exhaustive search.

The reference samples SO(3) with precomputed optimised quaternion sets shipped as package
data (``tme/data/*.npy`` with ``metadata.yaml``; tme/rotations.py:227-299): for a
requested angular step it loads the set whose step is nearest (the first listed on a
tie), takes the first four columns of the array as quaternions (x, y, z, w) and turns
them into matrices with ``scipy.spatial.transform.Rotation``. ``get_rotation_matrices``
here does the same from a directory holding those files, so the rotation indices of a
scan match the reference's exactly. The directory is found in this order:

* ``data_dir`` when given;
* ``$PYTME_ROTATION_DATA``;
* the data directory of an installed ``tme`` package (found without importing it);
* ``baseline/_ref/tme/data`` of this repository, where the offline reference install puts
  it.

Without any of them ``get_rotation_matrices`` raises FileNotFoundError, and
``rotation_set`` falls back to a super-Fibonacci sampling with the reference set's size
(``pytme_b200.synthetic``), saying so in its result.
"""
from __future__ import annotations

import importlib.util
import os
from typing import Optional, Tuple

import numpy as np

__all__ = ["quaternion_data_dir", "get_rotation_matrices", "rotation_set"]

_HERE = os.path.dirname(os.path.abspath(__file__))


def _tme_data_dir() -> Optional[str]:
    try:
        spec = importlib.util.find_spec("tme")
    except (ImportError, ValueError):
        spec = None
    for loc in (spec.submodule_search_locations or []) if spec else []:
        d = os.path.join(loc, "data")
        if os.path.exists(os.path.join(d, "metadata.yaml")):
            return d
    return None


def quaternion_data_dir(data_dir: Optional[str] = None) -> Optional[str]:
    """The first directory with the reference's quaternion sets (see module doc)."""
    cands = [data_dir, os.environ.get("PYTME_ROTATION_DATA"), _tme_data_dir(),
             os.path.join(os.path.dirname(_HERE), "baseline", "_ref", "tme", "data")]
    for d in cands:
        if d and os.path.exists(os.path.join(d, "metadata.yaml")):
            return d
    return None


def _nearest_set(metadata: dict, angle: float) -> str:
    """The set whose step is nearest to ``angle``; the first in file order on a tie
    (``min`` over the metadata's insertion order, tme/rotations.py:285-290)."""
    best, best_diff = None, None
    for name, (_, step, _) in metadata.items():
        diff = abs(angle - step)
        if best_diff is None or diff < best_diff:
            best, best_diff = name, diff
    return best


def get_rotation_matrices(angular_sampling: float, dim: int = 3,
                          data_dir: Optional[str] = None) -> np.ndarray:
    """The reference's optimised rotation set for ``angular_sampling`` degrees as
    (n, 3, 3) float64 matrices (tme/rotations.py:227-263 with use_optimized_set)."""
    if dim != 3:
        raise NotImplementedError("only 3D rotation sets are provided")
    d = quaternion_data_dir(data_dir)
    if d is None:
        raise FileNotFoundError("no directory with the reference's quaternion sets; pass "
                                "data_dir or set PYTME_ROTATION_DATA (tme/data of pyTME)")
    import yaml
    from scipy.spatial.transform import Rotation

    with open(os.path.join(d, "metadata.yaml")) as f:
        metadata = yaml.full_load(f)
    name = _nearest_set(metadata, float(angular_sampling))
    quat = np.load(os.path.join(d, name))[:, :4]
    return Rotation.from_quat(quat).as_matrix()


def rotation_set(angular_sampling: float, data_dir: Optional[str] = None
                 ) -> Tuple[np.ndarray, str]:
    """(float32 matrices, description): the reference's set when its data are found,
    else the super-Fibonacci stand-in of the same size."""
    try:
        m = get_rotation_matrices(angular_sampling, data_dir=data_dir)
        return np.ascontiguousarray(m, dtype=np.float32), \
            f"reference quaternion set for {angular_sampling} degrees ({len(m)} rotations)"
    except FileNotFoundError:
        from .synthetic import rotations_for_angle

        m = rotations_for_angle(angular_sampling)
        return m, (f"super-Fibonacci stand-in with the reference set's size "
                   f"({len(m)} rotations); the reference's quaternion data were not found")
