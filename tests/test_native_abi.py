"""The C-ABI library loads and exports every entry point the public header declares;
argument checks run before any device work, so they are testable without a GPU."""
import ctypes
import os
import re

import pytest

from tests.conftest import ROOT


def _header_functions():
    src = open(os.path.join(ROOT, "include", "pytme_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:int|int64_t)\s+(tm_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from pytme_b200 import _native as N

    lib = ctypes.CDLL(N.LIB_PATH)
    names = _header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/pytme_b200.h but not exported"
    assert set(N.EXPORTED) == set(names)
    # the test-only diagnostics are exported too, but declared outside the public header
    for name in N.DIAGNOSTICS:
        assert hasattr(lib, name) and name not in names


def test_version_and_error_buffer():
    from pytme_b200 import _native as N

    assert N.lib.tm_version() >= 100
    assert isinstance(N.last_error(), str)


def test_scan_create_rejects_bad_descriptors_without_gpu():
    from pytme_b200 import _native as N

    desc = N.ScanDesc()
    desc.score = 9
    h = ctypes.c_void_p()
    assert N.lib.tm_scan_create(ctypes.byref(desc), ctypes.byref(h)) == N.TM_E_INVALID
    assert "unknown score" in N.last_error()
    desc.score = N.TM_SCORE_FLCSM
    desc.precision = 0
    for i in range(3):
        desc.fast_shape[i] = 32
        desc.template_shape[i] = 64
    desc.batch = 4
    assert N.lib.tm_scan_create(ctypes.byref(desc), ctypes.byref(h)) == N.TM_E_INVALID
    assert "exceeds the transform length" in N.last_error()
    with pytest.raises(ValueError):
        N.check(N.TM_E_INVALID, "x")
    with pytest.raises(MemoryError):
        N.check(N.TM_E_OOM, "x")
    with pytest.raises(NotImplementedError):
        N.check(N.TM_E_UNSUPPORTED, "x")


def test_op_argument_checks_without_gpu():
    from pytme_b200 import _native as N

    assert N.lib.tm_rigid_transform(None, None, 4, 4, 4, None, 1, None, None, 4, 4, 4,
                                    None) == N.TM_E_INVALID
    assert N.lib.tm_norm_scores(None, None, None, 0.0, None, 1e-7, None, 10,
                                None) == N.TM_E_INVALID
    assert N.lib.tm_find_candidate_indices(None, -1, 3, None, None, None,
                                           None) == N.TM_E_INVALID
