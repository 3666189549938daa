"""pytme_b200: pyTME's exhaustive template-matching hot path on NVIDIA B200.

The package mirrors the reference's plugin surfaces for this path:

* ``backend`` / ``B200Backend`` — the ``MatchingBackend`` method surface
  (``backend.change_backend("b200", precision=..., rotation_batch=...)``);
* ``MATCHING_EXHAUSTIVE_REGISTER`` / ``register_matching_exhaustive`` — the score
  registry with "CC", "FLC" and "FLCSphericalMask";
* ``MatchingData``, ``scan``, ``scan_subsets`` — the exhaustive driver;
* ``MaxScoreOverRotations``, ``PeakCallerMaximumFilter``, ``PeakCallerSort`` — the
  analyzer/callback API.

All compute runs in ``libpytme_b200.so`` (CUDA, sm_100a); importing the package
fails if that library is missing. When the reference package ``tme`` is
importable, ``pytme_b200.tme_plugin.register()`` adds the backend and the
``*_b200`` scores to it.
"""
from ._native import lib as _lib  # noqa: F401  (fails loudly without the CUDA library)
from .backend import B200Backend, backend
from .matching import MatchingData, fourier_padding, rigid_transform_matrices, scan, scan_subsets
from .scores import MATCHING_EXHAUSTIVE_REGISTER, ScanPlan, register_matching_exhaustive
from . import filters  # noqa: F401
from .analyzer import (MaxScoreOverRotations, PeakCaller, PeakCallerMaximumFilter,
                       PeakCallerSort, SharedAnalyzerProxy)

__version__ = "0.1.0"

__all__ = [
    "B200Backend", "backend", "MatchingData", "fourier_padding", "rigid_transform_matrices",
    "scan", "scan_subsets", "MATCHING_EXHAUSTIVE_REGISTER", "ScanPlan",
    "register_matching_exhaustive", "MaxScoreOverRotations", "PeakCaller",
    "PeakCallerMaximumFilter", "PeakCallerSort", "SharedAnalyzerProxy",
]
