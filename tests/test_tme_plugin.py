"""Registration into the reference package (CPU): the backend satisfies tme's
MatchingBackend ABC and the *_b200 scores enter tme's registry. Runs only where the
reference checkout is present (it is not needed anywhere else)."""
import os
import sys

import pytest

REF = os.environ.get("PYTME_REFERENCE", "/root/reference")
SHIM = os.path.join(os.path.dirname(__file__), "golden", "refshim")


@pytest.fixture(scope="module")
def tme_mod():
    if not os.path.isdir(os.path.join(REF, "tme")):
        pytest.skip("reference checkout not present")
    sys.dont_write_bytecode = True
    for p in (SHIM, REF):
        if p not in sys.path:
            sys.path.insert(0, p)
    import tme  # noqa: F401

    return tme


def test_register_adds_backend_and_scores(tme_mod):
    from tme.backends import backend as tme_be
    from tme.backends.matching_backend import MatchingBackend
    from tme.matching_scores import MATCHING_EXHAUSTIVE_REGISTER

    from pytme_b200.tme_plugin import SCORE_NAMES, register

    assert register(strict=True)
    assert register(strict=True)  # idempotent
    cls = tme_be._BACKEND_REGISTRY["b200"]
    assert issubclass(cls, MatchingBackend)
    assert not getattr(cls, "__abstractmethods__", frozenset())
    for name in SCORE_NAMES.values():
        setup, scoring = MATCHING_EXHAUSTIVE_REGISTER[name]
        assert callable(setup) and callable(scoring)
