"""Stand-in for the pyFFTW API surface that the reference imports.

Used only by ``tests/golden/make_golden.py`` to run the reference package in a
container without pyFFTW. Transforms go through ``scipy.fft`` (pocketfft), which
keeps float32 inputs in single precision, so the reference's FP32 path keeps its
precision; FFT rounding is pocketfft's rather than FFTW's.
"""
import sys
import types

import numpy as np
import scipy.fft as _sfft

simd_alignment = 64
FFTW = object


def zeros_aligned(shape, dtype=None, n=None):
    return np.zeros(shape, dtype=dtype)


def next_fast_len(target):
    # pyFFTW's rule: 2^a 3^b 5^c 7^d 11^e 13^f with e + f <= 1.
    target = int(target)
    best = None
    n = max(target, 1)
    while best is None:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m in (1, 11, 13):
            best = n
        n += 1
    return best


class _NumpyFFT:
    @staticmethod
    def rfftn(a, s=None, axes=None, **kwargs):
        return _sfft.rfftn(a, s=s, axes=axes)

    @staticmethod
    def irfftn(a, s=None, axes=None, **kwargs):
        return _sfft.irfftn(a, s=s, axes=axes)


interfaces = types.SimpleNamespace(numpy_fft=_NumpyFFT)


def _builder(kind):
    def build(arr, s=None, axes=None, **kwargs):
        func = _sfft.rfftn if kind == "r" else _sfft.irfftn

        def run(inp, out):
            out[...] = func(inp, s=s, axes=axes)
            return out

        return run

    return build


builders = types.ModuleType("pyfftw.builders")
builders.rfftn = _builder("r")
builders.irfftn = _builder("i")
sys.modules["pyfftw.builders"] = builders
