"""pytest plugin that runs the reference's backend test suite (tests/test_backends.py
of pyTME) against the B200 backend.

The suite builds ``BACKENDS_TO_TEST`` at import from every class in tme's backend
registry, constructing each with ``device="cpu"``, and compares every operation with
``NumpyFFTWBackend``. This plugin registers the B200 backend into tme before the suite
is imported, under a subclass that constructs it on the current CUDA device whatever
device the suite names (the B200 backend has no CPU mode), and keeps only the tests
parametrised with it. Loaded with ``-p ref_backend_suite`` by
tests/test_gpu_tme_dropin.py.

A few of the suite's checks hand backend arrays straight to NumPy (``np.allclose(arr,
arr_b)`` in test_rigid_transform_batch), which works for the reference's backends because
the suite builds them on the CPU. The B200 backend's arrays are CUDA tensors, which
``torch.Tensor.__array__`` refuses to convert; in the suite's own process (and only there)
the conversion copies a CUDA tensor to the host first, so those checks compare values as
they do for the reference's backends.
"""


def _host_array_conversion():
    import torch

    orig = torch.Tensor.__array__

    def __array__(self, dtype=None):
        if self.is_cuda:
            self = self.detach().cpu()
        return orig(self, dtype)

    torch.Tensor.__array__ = __array__


def pytest_configure(config):
    from tme.backends import backend as tme_be

    from pytme_b200.tme_plugin import register

    _host_array_conversion()
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
