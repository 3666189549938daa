"""Registration into the reference package when it is importable.

``register()`` adds

* the backend ``"b200"`` to tme's BackendManager
  (``tme.backends.backend.add_backend``, tme/backends/__init__.py:82-107), as a class
  that derives from both ``B200Backend`` and tme's ``MatchingBackend`` ABC, so
  ``be.change_backend("b200", precision=..., rotation_batch=...)`` selects it;
* the scores ``"CC_b200"``, ``"FLC_b200"`` and ``"FLCSphericalMask_b200"`` through
  ``tme.matching_exhaustive.register_matching_exhaustive`` (:468-501) with the
  reference's memory classes.

tme's own ``scan`` then drives them unchanged: it applies the target filter
through the backend's cuFFT ``rfftn``/``irfftn``, calls the setup function with its
MatchingData (already on the device), and calls the scoring function with its
``SharedAnalyzerProxy``. With ``MaxScoreOverRotations`` and ``job_schedule=(1, 1)``
the rotation chunk runs fused on the GPU; other analyzers get one map per rotation.
"""
from __future__ import annotations

from .backend import B200Backend
from . import scores as _scores

__all__ = ["register", "SCORE_NAMES"]

SCORE_NAMES = {"CC": "CC_b200", "FLC": "FLC_b200", "FLCSphericalMask": "FLCSphericalMask_b200"}
_MEMORY_CLASSES = {"CC": "CCMemoryUsage", "FLC": "FLCMemoryUsage",
                   "FLCSphericalMask": "FLCSphericalMaskMemoryUsage"}


def _setup_from_tme(score):
    def setup(matching_data, fast_shape, fast_ft_shape=None, shm_handler=None,
              template_filter=None, **kwargs):
        # tme's scan already multiplied the target filter into matching_data.target
        return _scores._setup(score, matching_data, fast_shape, template_filter=template_filter,
                              target_filter=None)

    setup.__name__ = f"{score}_b200_setup"
    return setup


def register(strict: bool = False) -> bool:
    """Register with tme if it is importable; returns whether it did."""
    try:
        from tme.backends import backend as tme_be
        from tme.backends.matching_backend import MatchingBackend
        from tme.matching_exhaustive import register_matching_exhaustive
        from tme.matching_scores import MATCHING_EXHAUSTIVE_REGISTER
        import tme.memory as tme_memory
    except ImportError:
        if strict:
            raise
        return False
    cls = type("B200Backend", (B200Backend, MatchingBackend), {"__module__": __name__})
    if "b200" not in getattr(tme_be, "_BACKEND_REGISTRY", {}):
        tme_be.add_backend("b200", cls)
    for score, name in SCORE_NAMES.items():
        if name in MATCHING_EXHAUSTIVE_REGISTER:
            continue
        memory = getattr(tme_memory, _MEMORY_CLASSES[score])
        scoring = _scores.MATCHING_EXHAUSTIVE_REGISTER[score][1]
        register_matching_exhaustive(name, _setup_from_tme(score), scoring, memory)
    return True
