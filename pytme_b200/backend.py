"""The B200 matching backend.

``B200Backend`` provides the method surface of the reference's ``MatchingBackend``
(tme/backends/matching_backend.py:28-1271) over CUDA tensors. Array bookkeeping
(creation, slicing, reductions used off the scan loop) uses torch tensors as
device buffers; the hot-path methods run kernels of ``libpytme_b200.so``:
``rigid_transform`` (order 1), ``norm_scores``, ``max_score_over_rotations``,
``build_fft``/``rfftn``/``irfftn`` (cuFFT plans owned by the library),
``max_filter_coordinates`` and ``topk_indices``.

``backend`` is a small manager with the reference's ``change_backend`` call; the
only backend it knows is "b200", whose keyword options select the scan plan:
``precision`` ("fp32" or "mixed"), ``rotation_batch`` (rotations per fused launch
group) and ``plain`` (one rotation at a time through full cuFFT transforms).
"""
from __future__ import annotations

import contextlib
from typing import Dict, Tuple

import numpy as np
import torch

from . import _native as N

__all__ = ["B200Backend", "backend", "current_options", "fft_plan", "FFTPlan"]

_DEFAULTS = {"precision": "fp32", "rotation_batch": 32, "plain": False, "xpass": "auto",
             "ypass": "auto", "zpass": "auto"}
_OPTIONS = dict(_DEFAULTS)


def current_options() -> Dict:
    return dict(_OPTIONS)


def _set_options(**kwargs):
    """Options of a new backend instance: the defaults, updated by ``kwargs``."""
    _OPTIONS.clear()
    _OPTIONS.update(_DEFAULTS)
    for k, v in kwargs.items():
        if k in _DEFAULTS:
            _OPTIONS[k] = v
    if _OPTIONS["precision"] not in ("fp32", "mixed"):
        raise ValueError("precision must be 'fp32' or 'mixed'")
    for key in ("xpass", "ypass", "zpass"):
        allowed = ("auto", "fft", "tensor") + (("tensor2", "tensor-inplace") if key == "ypass"
                                               else ())
        if _OPTIONS[key] not in allowed:
            raise ValueError(f"{key} must be one of {', '.join(allowed)}")
    _OPTIONS["rotation_batch"] = int(_OPTIONS["rotation_batch"])
    if not 1 <= _OPTIONS["rotation_batch"] <= 4096:
        raise ValueError("rotation_batch must be in [1, 4096]")


_TORCH_DTYPES = {
    np.float32: torch.float32, np.float64: torch.float64, np.float16: torch.float16,
    np.int32: torch.int32, np.int64: torch.int64, np.complex64: torch.complex64,
    np.complex128: torch.complex128, np.bool_: torch.bool, bool: torch.bool,
    int: torch.int32, float: torch.float32, complex: torch.complex64,
}


def _tdtype(dtype):
    if dtype is None:
        return torch.float32
    if isinstance(dtype, torch.dtype):
        return dtype
    try:
        return _TORCH_DTYPES[np.dtype(dtype).type]
    except (TypeError, KeyError):
        return _TORCH_DTYPES.get(dtype, torch.float32)


class FFTPlan:
    """cuFFT r2c/c2r pair for one real shape (``tm_fft_plan``). ``irfftn`` applies
    NumPy's 1/prod(shape) normalisation."""

    def __init__(self, shape: Tuple[int, ...], double: bool = False):
        self.shape = tuple(int(x) for x in shape)
        self.double = bool(double)
        arr = (N.c_int * len(self.shape))(*self.shape)
        h = N.c_void_p()
        N.check(N.lib.tm_fft_plan_create(len(self.shape), arr, 1, int(self.double),
                                         N.ctypes.byref(h)), "tm_fft_plan_create")
        self._h = h
        self.ft_shape = self.shape[:-1] + (self.shape[-1] // 2 + 1,)

    def rfftn(self, x: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
        rd = torch.float64 if self.double else torch.float32
        cd = torch.complex128 if self.double else torch.complex64
        x = x.to(dtype=rd).contiguous()
        if out is None:
            out = torch.empty(self.ft_shape, dtype=cd, device=x.device)
        N.check(N.lib.tm_fft_r2c(self._h, N.ptr(x), N.ptr(out), N.stream_ptr()), "tm_fft_r2c")
        return out

    def irfftn(self, x: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
        rd = torch.float64 if self.double else torch.float32
        cd = torch.complex128 if self.double else torch.complex64
        tmp = x.to(dtype=cd).contiguous().clone()  # c2r overwrites its input
        if out is None:
            out = torch.empty(self.shape, dtype=rd, device=x.device)
        scale = 1.0 / float(np.prod(self.shape))
        N.check(N.lib.tm_fft_c2r(self._h, N.ptr(tmp), N.ptr(out), scale, N.stream_ptr()),
                "tm_fft_c2r")
        return out

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.lib.tm_fft_plan_destroy(self._h)
                self._h = None
        except Exception:
            pass


_FFT_CACHE: Dict = {}


def fft_plan(shape, double: bool = False) -> FFTPlan:
    key = (tuple(int(x) for x in shape), bool(double), torch.cuda.current_device())
    plan = _FFT_CACHE.get(key)
    if plan is None:
        plan = FFTPlan(shape, double)
        _FFT_CACHE[key] = plan
    return plan


class B200Backend:
    """MatchingBackend surface on CUDA tensors (see module docstring)."""

    def __init__(self, device: str = "cuda", float_dtype=torch.float32,
                 complex_dtype=torch.complex64, int_dtype=torch.int32,
                 overflow_safe_dtype=torch.float32, **kwargs):
        if not torch.cuda.is_available():
            raise RuntimeError("B200Backend needs a CUDA device; there is no CPU fallback")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError(f"B200Backend runs on CUDA devices only, not {device!r}")
        self._array_backend = torch
        self._float_dtype = _tdtype(float_dtype)
        self._complex_dtype = _tdtype(complex_dtype)
        self._int_dtype = _tdtype(int_dtype)
        self._overflow_safe_dtype = _tdtype(overflow_safe_dtype)
        self._fundamental_dtypes = {int: self._int_dtype, float: self._float_dtype,
                                    complex: self._complex_dtype}
        _set_options(**kwargs)

    # ------------------------------------------------------------ conversion
    def to_backend_array(self, arr):
        if isinstance(arr, torch.Tensor):
            return arr.to(self.device) if arr.device != self.device else arr
        return torch.as_tensor(np.asarray(arr), device=self.device)

    def to_numpy_array(self, arr):
        if isinstance(arr, torch.Tensor):
            return arr.detach().cpu().numpy()
        return np.asarray(arr)

    def to_cpu_array(self, arr):
        return arr.cpu() if isinstance(arr, torch.Tensor) else arr

    def to_sharedarr(self, arr, shared_memory_handler=None):
        return arr

    def from_sharedarr(self, arr):
        return arr

    def free_cache(self):
        torch.cuda.empty_cache()

    def get_fundamental_dtype(self, arr):
        dt = arr.dtype if hasattr(arr, "dtype") else np.asarray(arr).dtype
        if isinstance(dt, torch.dtype):
            if dt.is_complex:
                return complex
            return float if dt.is_floating_point else int
        if np.issubdtype(dt, np.integer):
            return int
        if np.issubdtype(dt, np.complexfloating):
            return complex
        return float

    # ------------------------------------------------------------ creation
    def zeros(self, shape, dtype=None):
        return torch.zeros(shape, dtype=_tdtype(dtype), device=self.device)

    def full(self, shape, fill_value, dtype=None):
        return torch.full(tuple(np.atleast_1d(shape)) if not isinstance(shape, tuple) else shape,
                          fill_value, dtype=_tdtype(dtype), device=self.device)

    def fill(self, arr, value):
        arr.fill_(value)
        return arr

    def arange(self, *args, **kwargs):
        return torch.arange(*args, device=self.device, **kwargs)

    def astype(self, arr, dtype):
        if torch.is_complex(arr):
            arr = arr.real
        return arr.to(_tdtype(dtype))

    def eps(self, dtype):
        return torch.finfo(_tdtype(dtype)).eps

    def datatype_bytes(self, dtype):
        return torch.tensor([], dtype=_tdtype(dtype)).element_size()

    def size(self, arr):
        return arr.numel()

    def tobytes(self, arr):
        return self.to_numpy_array(arr).tobytes()

    # ------------------------------------------------------------ elementwise / reductions
    def add(self, x1, x2, out=None, **kw):
        return torch.add(self.to_backend_array(x1), x2, out=out)

    def subtract(self, x1, x2, out=None, **kw):
        return torch.subtract(self.to_backend_array(x1), x2, out=out)

    def multiply(self, x1, x2, out=None, **kw):
        return torch.multiply(self.to_backend_array(x1), x2, out=out)

    def divide(self, x1, x2, out=None, **kw):
        return torch.divide(self.to_backend_array(x1), x2, out=out)

    def mod(self, x1, x2, out=None, **kw):
        return torch.remainder(self.to_backend_array(x1), x2, out=out)

    def sum(self, arr, axis=None, keepdims=False, **kw):
        if axis is None:
            return arr.sum() if not keepdims else arr.sum().reshape((1,) * arr.ndim)
        return arr.sum(dim=axis, keepdim=keepdims)

    def mean(self, arr, axis=None, keepdims=False, **kw):
        return arr.mean() if axis is None else arr.mean(dim=axis, keepdim=keepdims)

    def std(self, arr, axis=None, keepdims=False, **kw):
        return arr.std(unbiased=False) if axis is None else arr.std(dim=axis, keepdim=keepdims,
                                                                   unbiased=False)

    def max(self, arr, axis=None, **kw):
        return arr.max() if axis is None else arr.amax(dim=axis)

    def min(self, arr, axis=None, **kw):
        return arr.min() if axis is None else arr.amin(dim=axis)

    def maximum(self, x1, x2, out=None, **kw):
        x2 = x2 if isinstance(x2, torch.Tensor) else torch.as_tensor(x2, device=self.device,
                                                                      dtype=x1.dtype)
        return torch.maximum(x1, x2, out=out)

    def minimum(self, x1, x2, out=None, **kw):
        x2 = x2 if isinstance(x2, torch.Tensor) else torch.as_tensor(x2, device=self.device,
                                                                      dtype=x1.dtype)
        return torch.minimum(x1, x2, out=out)

    def sqrt(self, arr, out=None, **kw):
        return torch.sqrt(arr, out=out)

    def square(self, arr, out=None, **kw):
        return torch.square(arr, out=out)

    def abs(self, arr, out=None, **kw):
        return torch.abs(arr, out=out)

    def power(self, x1, x2, out=None, **kw):
        return torch.pow(x1, x2, out=out)

    def clip(self, arr, a_min, a_max, out=None):
        return torch.clamp(arr, a_min, a_max, out=out)

    def einsum(self, *args, **kwargs):
        return torch.einsum(*args)

    def transpose(self, arr, *args, **kwargs):
        return arr.permute(*reversed(range(arr.ndim))) if not args else arr.permute(*args)

    def where(self, condition, *args):
        return torch.where(condition, *args) if args else torch.nonzero(condition, as_tuple=True)

    def unique(self, arr, return_index=False, return_inverse=False, return_counts=False,
               axis=None, **kwargs):
        out = np.unique(self.to_numpy_array(arr), return_index=return_index,
                        return_inverse=return_inverse, return_counts=return_counts, axis=axis)
        if isinstance(out, tuple):
            return tuple(self.to_backend_array(x) for x in out)
        return self.to_backend_array(out)

    def argsort(self, arr, *args, **kwargs):
        return torch.argsort(arr)

    def concatenate(self, arrays, *args, **kwargs):
        return torch.cat([self.to_backend_array(a) for a in arrays], *args)

    def stack(self, arrays, *args, **kwargs):
        return torch.stack([self.to_backend_array(a) for a in arrays], *args)

    def repeat(self, arr, repeats, axis=None):
        return torch.repeat_interleave(arr, repeats, dim=axis)

    def reshape(self, arr, shape, **kw):
        return arr.reshape(shape)

    def indices(self, dimensions, dtype=int, **kwargs):
        """np.indices on the device: one index grid per axis, stacked first."""
        grids = torch.meshgrid(*[torch.arange(int(n), device=self.device)
                                 for n in dimensions], indexing="ij")
        return torch.stack(grids).to(self._int_dtype if dtype is int else _tdtype(dtype))

    def extract_center(self, arr, newshape):
        """The centred box of ``newshape`` (tme/backends/npfftw_backend.py:308-315)."""
        starts = [(int(c) - int(n)) // 2 for c, n in zip(arr.shape, newshape)]
        return arr[tuple(slice(a, a + int(n)) for a, n in zip(starts, newshape))]

    def center_of_mass(self, arr, cutoff=None):
        """Centre of mass of the values above ``cutoff`` (all values when None), in
        double precision (tme/backends/npfftw_backend.py:451-484)."""
        a = self.to_backend_array(arr).to(torch.float64)
        cutoff = float(a.min()) - 1 if cutoff is None else float(cutoff)
        a = torch.where(a > cutoff, a, torch.zeros_like(a))
        den = a.sum()
        out = []
        for axis, n in enumerate(a.shape):
            shape = [1] * a.ndim
            shape[axis] = n
            grid = torch.arange(n, dtype=torch.float64, device=a.device).reshape(shape)
            out.append(((a * grid) / den).sum())
        return torch.stack(out)

    def unravel_index(self, indices, shape):
        return np.unravel_index(self.to_numpy_array(indices), shape)

    def tril_indices(self, *args, **kwargs):
        return torch.tril_indices(*args, device=self.device)

    @staticmethod
    def at(arr, idx, value):
        arr[idx] = value
        return arr

    def roll(self, a, shift, axis, **kwargs):
        return torch.roll(a, shifts=tuple(int(s) for s in shift), dims=tuple(axis))

    @staticmethod
    def reverse(arr, axis=None):
        dims = tuple(range(arr.ndim)) if axis is None else tuple(axis)
        return torch.flip(arr, dims=dims)

    # ------------------------------------------------------------ hot-path methods
    def topleft_pad(self, arr, shape, padval=0):
        arr = self.to_backend_array(arr)
        b = torch.full(tuple(int(x) for x in shape), padval, dtype=arr.dtype, device=self.device)
        box = tuple(slice(0, min(a, s)) for a, s in zip(arr.shape, shape))
        b[box] = arr[box]
        return b

    def compute_convolution_shapes(self, arr1_shape, arr2_shape):
        from .matching import compute_convolution_shapes

        return compute_convolution_shapes(arr1_shape, arr2_shape)

    def build_fft(self, fwd_shape, inv_shape, real_dtype=None, cmpl_dtype=None, fftargs=None,
                  inv_output_shape=None, temp_fwd=None, temp_inv=None, fwd_axes=None,
                  inv_axes=None):
        """cuFFT r2c / normalised c2r callables with the reference's (arr, out) signature
        (tme/backends/npfftw_backend.py:243-293)."""
        if fwd_axes is not None or inv_axes is not None:
            raise NotImplementedError("batched FFT axes are not supported")
        out_shape = tuple(fwd_shape if inv_output_shape is None else inv_output_shape)
        fwd = fft_plan(tuple(fwd_shape))
        inv = fft_plan(out_shape)

        def rfftn(arr, out=None, *args, **kwargs):
            res = fwd.rfftn(arr)
            if out is not None:
                out.copy_(res)
                return out
            return res

        def irfftn(arr, out=None, *args, **kwargs):
            res = inv.irfftn(arr)
            if out is not None:
                out.copy_(res)
                return out
            return res

        return rfftn, irfftn

    def rfftn(self, arr, s=None, axes=None, **kwargs):
        arr = self.to_backend_array(arr)
        if axes is not None:
            raise NotImplementedError("rfftn over a subset of axes is not supported")
        shape = tuple(arr.shape) if s is None else tuple(int(x) for x in s)
        if shape != tuple(arr.shape):
            arr = self.topleft_pad(arr, shape)
        return fft_plan(shape, arr.dtype == torch.float64).rfftn(arr)

    def irfftn(self, arr, s=None, axes=None, **kwargs):
        arr = self.to_backend_array(arr)
        if axes is not None:
            raise NotImplementedError("irfftn over a subset of axes is not supported")
        shape = tuple(arr.shape[:-1]) + (2 * (arr.shape[-1] - 1),) if s is None else tuple(s)
        return fft_plan(shape, arr.dtype == torch.complex128).irfftn(arr)

    def _rigid_transform_matrix(self, rotation_matrix, translation=None, center=None):
        """float32 homogeneous pull matrix (tme/backends/npfftw_backend.py:326-355)."""
        from .matching import rigid_transform_matrices

        rot = self.to_numpy_array(rotation_matrix).astype(np.float32)
        c = np.zeros(3) if center is None else self.to_numpy_array(center)
        if translation is not None and np.any(self.to_numpy_array(translation)):
            raise NotImplementedError("rigid transforms with a translation are not supported")
        return self.to_backend_array(rigid_transform_matrices(rot[None], c)[0])

    def rigid_transform(self, arr, rotation_matrix, arr_mask=None, translation=None,
                        use_geometric_center: bool = False, out=None, out_mask=None,
                        order: int = 3, cache: bool = False, batched: bool = False):
        """Rigid transform on the device; the reference's NumpyFFTWBackend.rigid_transform
        (tme/backends/npfftw_backend.py:357-449) with SciPy's constant mode. Order 1 is
        trilinear (tm_rigid_transform); order 3 is the cubic B-spline with the data
        prefiltered and the mask not (tm_spline_prefilter + tm_rigid_transform_cubic).
        A square rotation matrix turns about the geometric centre or, by default as in the
        reference, the data's centre of mass; a homogeneous matrix is used as given.
        2D data run as one plane of a 3D volume; ``batched`` transforms every item along
        the leading axis with the same matrix, as the reference loops over them."""
        if int(order) not in (1, 3):
            raise NotImplementedError("only order 1 (trilinear) and 3 (cubic B-spline) rigid "
                                      "transforms are supported")
        arr = self.to_backend_array(arr)
        if out is None:
            out = torch.zeros_like(arr)
        if arr_mask is not None:
            arr_mask = self.to_backend_array(arr_mask)
            if out_mask is None:
                out_mask = torch.zeros_like(arr_mask)
        matrix = self.to_backend_array(rotation_matrix)
        ndim = arr.ndim - int(bool(batched))
        if matrix.shape[-1] == ndim:
            if use_geometric_center:
                center = np.divide(np.asarray(arr.shape[-ndim:]) - 1, 2)
            else:
                center = self.to_numpy_array(self.center_of_mass(arr, cutoff=0))[-ndim:]
            if translation is not None and np.any(self.to_numpy_array(translation)):
                raise NotImplementedError("rigid transforms with a translation are not "
                                          "supported")
            matrix = self._homogeneous(matrix, center)
        if batched:
            for i in range(arr.shape[0]):
                self._transform_one(arr[i], matrix, out[i],
                                    None if arr_mask is None else arr_mask[i],
                                    None if arr_mask is None else out_mask[i], int(order))
            return out, out_mask
        self._transform_one(arr, matrix, out, arr_mask, out_mask, int(order))
        return out, out_mask

    def _homogeneous(self, rotation, center):
        """Pull matrix of a rotation about ``center`` with the reference's float32
        arithmetic, lifted to 3D for 2D data (an untouched leading axis)."""
        from .matching import rigid_transform_matrices

        rot = self.to_numpy_array(rotation).astype(np.float32)
        c = np.asarray(center, dtype=np.float64)
        if rot.shape[-1] == 2:
            r3 = np.eye(3, dtype=np.float32)
            r3[1:, 1:] = rot
            rot, c = r3, np.concatenate(([0.0], c))
        return self.to_backend_array(rigid_transform_matrices(rot[None], c)[0])

    def _transform_one(self, arr, matrix, out, mask, out_mask, order):
        """One volume (2D or 3D) through the library's kernels, into float32 scratch when
        the output is another type or shares the input's memory."""
        if arr.ndim not in (2, 3):
            raise NotImplementedError("rigid transforms of 2D and 3D data only")
        lift = (lambda t: t.reshape((1,) + tuple(t.shape))) if arr.ndim == 2 else (lambda t: t)
        a = lift(arr.to(torch.float32).contiguous())
        if a.data_ptr() == arr.data_ptr():
            a = a.clone()  # the output may be this very buffer
        m = None if mask is None else lift(mask.to(torch.float32).contiguous()).clone()
        direct = out.dtype == torch.float32 and out.is_contiguous() and \
            out.data_ptr() not in (arr.data_ptr(), 0 if mask is None else mask.data_ptr())
        o = lift(out) if direct else torch.zeros(lift(out).shape, dtype=torch.float32,
                                                  device=a.device)
        om = None
        if m is not None:
            mdirect = out_mask.dtype == torch.float32 and out_mask.is_contiguous() and \
                out_mask.data_ptr() not in (arr.data_ptr(), mask.data_ptr())
            om = lift(out_mask) if mdirect else torch.zeros(lift(out_mask).shape,
                                                            dtype=torch.float32,
                                                            device=a.device)
        mat = matrix.to(torch.float32)
        if mat.numel() == 9:  # homogeneous matrix of 2D data: lift to 3D
            m4 = torch.eye(4, dtype=torch.float32, device=mat.device)
            m4[1:, 1:] = mat.reshape(3, 3)
            mat = m4
        mat = mat.contiguous().reshape(1, 16)
        if order == 3:
            coef = torch.empty(a.shape, dtype=torch.float64, device=a.device)
            N.check(N.lib.tm_spline_prefilter(N.ptr(a), N.ptr(coef), *a.shape, 1,
                                              N.stream_ptr()), "tm_spline_prefilter")
            mcoef = None if m is None else m.to(torch.float64).contiguous()
            N.check(N.lib.tm_rigid_transform_cubic(
                N.ptr(coef), N.ptr(mcoef), *a.shape, N.ptr(mat), 1, N.ptr(o),
                N.ptr(om), *o.shape, N.stream_ptr()), "tm_rigid_transform_cubic")
        else:
            N.check(N.lib.tm_rigid_transform(N.ptr(a), N.ptr(m), *a.shape, N.ptr(mat), 1,
                                             N.ptr(o), N.ptr(om), *o.shape, N.stream_ptr()),
                    "tm_rigid_transform")
        if not direct:
            out.copy_(o.reshape(out.shape))
        if om is not None and om.data_ptr() != lift(out_mask).data_ptr():
            out_mask.copy_(om.reshape(out_mask.shape))

    def norm_scores(self, arr, exp_sq, sq_exp, n_obs, eps, out):
        """tm_norm_scores: the reference's norm_scores (tme/backends/npfftw_backend.py:
        537-587) in double precision."""
        a = None if not isinstance(arr, torch.Tensor) else arr.contiguous()
        if a is None and float(arr) != 1.0:
            raise NotImplementedError("norm_scores with a scalar other than 1")
        n_dev = None
        n_host = 0.0
        if isinstance(n_obs, torch.Tensor):
            n_dev = n_obs.to(torch.float32).reshape(1).contiguous()
        else:
            n_host = float(n_obs)
        es, se = exp_sq.contiguous(), sq_exp.contiguous()
        N.check(N.lib.tm_norm_scores(N.ptr(a), N.ptr(es), N.ptr(se), n_host, N.ptr(n_dev),
                                     float(eps), N.ptr(out), int(out.numel()), N.stream_ptr()),
                "tm_norm_scores")
        return out

    def max_score_over_rotations(self, scores, max_scores, rotations, rotation_index: int):
        """tm_max_score_over_rotations (strict >, tme/backends/npfftw_backend.py:503-535)."""
        N.check(N.lib.tm_max_score_over_rotations(
            N.ptr(scores.contiguous()), N.ptr(max_scores), N.ptr(rotations), int(rotation_index),
            int(max_scores.numel()), N.stream_ptr()), "tm_max_score_over_rotations")
        return max_scores, rotations

    def topk_indices(self, arr, k: int):
        """Indices of the k largest values, largest first
        (tme/backends/npfftw_backend.py:177-182)."""
        flat = arr.reshape(-1)
        k = min(int(k), flat.numel())
        vals, idx = torch.topk(flat, k, largest=True, sorted=True)
        return self.unravel_index(idx, arr.shape)

    def max_filter_coordinates(self, score_space, min_distance):
        """Local maxima under a box maximum filter of edge ``min_distance``
        (tme/backends/npfftw_backend.py:200-206): the library's kernel for 3D maps, torch's
        max pooling over a zero-padded map (SciPy's constant mode, window
        [i - d//2, i - d//2 + d - 1]) for 1D and 2D ones."""
        from .peaks import max_filter_coordinates

        s = self.to_backend_array(score_space)
        if s.ndim == 3:
            return max_filter_coordinates(s, min_distance)
        if s.ndim not in (1, 2):
            raise NotImplementedError("maximum filters of 1D, 2D and 3D maps only")
        d = int(min_distance)
        x = s.to(torch.float32)
        lo, hi = d // 2, d - 1 - d // 2
        xp = torch.nn.functional.pad(x[None, None], [lo, hi] * x.ndim, value=0.0)
        pool = torch.nn.functional.max_pool1d if x.ndim == 1 else torch.nn.functional.max_pool2d
        mf = pool(xp, kernel_size=d, stride=1)[0, 0]
        return torch.nonzero(mf == x).cpu().numpy().astype(np.int64)

    # ------------------------------------------------------------ device handling
    def get_available_memory(self) -> int:
        free, _ = torch.cuda.mem_get_info()
        return int(free)

    @contextlib.contextmanager
    def set_device(self, device_index: int):
        with torch.cuda.device(int(device_index)):
            yield None

    def device_count(self) -> int:
        return torch.cuda.device_count()


class _BackendManager:
    """Mirror of tme.backends.BackendManager for the single "b200" backend."""

    def __init__(self):
        self._backend = None
        self._backend_name = "b200"
        self._backend_args: Dict = {}

    def change_backend(self, backend_name: str = "b200", **kwargs):
        if backend_name != "b200":
            raise NotImplementedError(f"Available backends are b200 - not {backend_name}.")
        self._backend = B200Backend(**kwargs)
        self._backend_name = backend_name
        self._backend_args = kwargs

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        if self._backend is None:
            self.change_backend("b200")
        return getattr(self._backend, name)


backend = _BackendManager()
