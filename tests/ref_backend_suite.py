"""pytest plugin that runs the reference's backend test suite (tests/test_backends.py
of pyTME) against the B200 backend.

The suite builds ``BACKENDS_TO_TEST`` at import from every class in tme's backend
registry, constructing each with ``device="cpu"``, and compares every operation with
``NumpyFFTWBackend``. This plugin registers the B200 backend into tme before the suite
is imported, under a subclass that constructs it on the current CUDA device whatever
device the suite names (the B200 backend has no CPU mode), and keeps only the tests
parametrised with it. Loaded with ``-p ref_backend_suite`` by
tests/test_gpu_tme_dropin.py.
"""


def pytest_configure(config):
    from tme.backends import backend as tme_be

    from pytme_b200.tme_plugin import register

    register(strict=True)
    base = tme_be._BACKEND_REGISTRY["b200"]

    class B200Backend(base):
        def __init__(self, device="cuda", **kwargs):
            super().__init__(device="cuda", **kwargs)

    tme_be._BACKEND_REGISTRY["b200"] = B200Backend


def pytest_collection_modifyitems(config, items):
    from pytme_b200.backend import B200Backend

    def is_b200(item):
        cs = getattr(item, "callspec", None)
        b = cs.params.get("backend") if cs is not None else None
        return isinstance(b, B200Backend) or (isinstance(b, type) and issubclass(b, B200Backend))

    keep = [it for it in items if is_b200(it)]
    drop = [it for it in items if not is_b200(it)]
    items[:] = keep
    config.hook.pytest_deselected(items=drop)
