"""Fourier filters of the matching path, built on the host once per scan.

Restates, with the reference's arithmetic (float64 grids cast to float32 where it
casts), the filters a scan multiplies into template and target spectra:

* ``CTFReconstructed`` — tme/filters/ctf.py:260-336 with ``create_ctf`` (:528-655)
  and the electron wavelength (:508-525);
* ``WedgeReconstructed`` with ``create_continuous_wedge=True`` —
  tme/filters/wedge.py:282-374;
* ``LinearWhiteningFilter`` — tme/filters/whitening.py:23-186;
* ``Compose`` — tme/filters/compose.py:17-59.

Each filter is called like the reference's (``f(shape=..., return_real_fourier=True,
...)``) and returns a dict whose ``data`` is a float32 NumPy array in rfft layout
(DC at index 0). ``device_filter`` builds CTFs, continuous wedges and their Compose
directly on the GPU (``csrc/filters.cu``) with the same per-voxel arithmetic; the scan
path uses it whenever a filter is one of those.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Tuple

import numpy as np

__all__ = ["fftfreqn", "shift_fourier", "crop_real_fourier", "create_ctf",
           "CTFReconstructed", "WedgeReconstructed", "LinearWhiteningFilter", "Compose",
           "device_filter", "needs_spectrum"]


def fftfreqn(shape, sampling_rate, compute_euclidean_norm=False, shape_is_real_fourier=False):
    """tme/filters/_utils.py:146-202 (dense/euclidean forms)."""
    norm = np.full(len(shape), fill_value=1, dtype=np.float32)
    center = np.divide(shape, 2).astype(np.int32)
    if sampling_rate is not None:
        norm = np.multiply(shape, sampling_rate).astype(int)
    if shape_is_real_fourier:
        center[-1], norm[-1] = 0, 1
        if sampling_rate is not None:
            norm[-1] = (shape[-1] - 1) * 2 * sampling_rate
    grids = []
    for i, x in enumerate(shape):
        dims = tuple(1 if i != t else x for t in range(len(shape)))
        g = (np.arange(x, dtype=np.int32) - center[i]) / norm[i]
        grids.append(g.astype(np.float32).reshape(dims))
    if compute_euclidean_norm:
        out = sum(np.square(x) for x in grids)
        return np.sqrt(out, out=out)
    flesh = np.full(shape, fill_value=1, dtype=np.float32)
    return np.stack(tuple(g * flesh for g in grids))


def shift_fourier(data, shape_is_real_fourier=False):
    """tme/filters/_utils.py:233-246: move the DC term from the centre to index 0."""
    shape = np.asarray(data.shape)
    shift = [int(x) for x in np.add(np.divide(shape, 2), np.mod(shape, 2))]
    if shape_is_real_fourier:
        shift[-1] = 0
    return np.roll(data, shift, tuple(range(len(shift))))


def crop_real_fourier(data):
    return data[..., : 1 + (data.shape[-1] // 2)]


def _electron_wavelength(acceleration_voltage):
    """Relativistic electron wavelength in Angstrom (tme/filters/ctf.py:508-525)."""
    h = 6.62606896e-34
    e = 1.60217646e-19
    m = 9.10938215e-31
    c = 299792458
    energy = e * acceleration_voltage
    den = energy ** 2
    den += 2 * energy * m * c ** 2
    lam = np.divide(h * c, np.sqrt(den))
    lam *= 1e10
    return lam


def create_ctf(shape, defocus_x, acceleration_voltage=300, defocus_angle=0, phase_shift=0,
               defocus_y=None, sampling_rate=1, spherical_aberration=2.7e7,
               amplitude_contrast=0.07, cutoff_frequency=0.5, **kwargs):
    """CTF with DC at the centre (tme/filters/ctf.py:528-655), without astigmatism
    gradients or tilt: chi = pi lambda k^2 (df - Cs lambda^2 k^2 / 2) + phase +
    atan(A / sqrt(1 - A^2)); returns sin(-chi) inside the frequency cutoff."""
    lam = _electron_wavelength(acceleration_voltage)
    lam /= sampling_rate
    aberration = (spherical_aberration / sampling_rate) * lam ** 2
    if defocus_y is not None:
        sampling = tuple(float(x) for x in np.divide(sampling_rate, shape))
        grid = [g for g in _sparse_grid(shape, sampling)]
        ds = np.add(defocus_x, defocus_y)
        dd = np.subtract(defocus_x, defocus_y)
        ang = np.arctan2(grid[1], grid[0])
        dd = np.multiply(dd, np.cos(2 * (ang - defocus_angle)))
        defocus_x = np.add(ds, dd)
        defocus_x *= 0.5
    freq = fftfreqn(shape, sampling_rate=True, compute_euclidean_norm=True)
    mask = freq < cutoff_frequency
    freq = np.square(freq, out=freq)
    chi = defocus_x - 0.5 * aberration * freq
    chi = np.multiply(chi, np.pi * lam, out=chi)
    chi = np.multiply(chi, freq, out=chi)
    chi += phase_shift
    chi += np.arctan(np.divide(amplitude_contrast, np.sqrt(1 - np.square(amplitude_contrast))))
    chi = np.sin(-chi, out=chi)
    chi = np.multiply(chi, mask, out=chi)
    return chi


def _sparse_grid(shape, sampling):
    center = np.divide(shape, 2).astype(np.int32)
    norm = np.multiply(shape, sampling).astype(int)
    out = []
    for i, x in enumerate(shape):
        dims = tuple(1 if i != t else x for t in range(len(shape)))
        g = (np.arange(x, dtype=np.int32) - center[i]) / norm[i]
        out.append(g.astype(np.float32).reshape(dims))
    return out


@dataclass
class CTFReconstructed:
    """Single CTF for a reconstructed volume (tme/filters/ctf.py:260-336)."""

    shape: Tuple[int] = None
    defocus_x: float = None
    angles: Tuple[float] = None
    opening_axis: int = 2
    tilt_axis: int = 0
    sampling_rate: float = 1
    acceleration_voltage: float = 300e3
    spherical_aberration: float = 2.7e7
    amplitude_contrast: float = 0.07
    phase_shift: float = 0
    defocus_angle: float = 0
    defocus_y: float = None
    flip_phase: bool = True
    return_real_fourier: bool = False

    def __post_init__(self):
        self.defocus_angle = np.radians(self.defocus_angle)
        self.phase_shift = np.radians(self.phase_shift)

    def __call__(self, **kwargs) -> Dict:
        args = dict(vars(self))
        args.update(kwargs)
        shape = args["shape"]
        stack = create_ctf(shape=shape, defocus_x=args["defocus_x"],
                           defocus_y=args.get("defocus_y"),
                           sampling_rate=np.max(args.get("sampling_rate", 1)),
                           acceleration_voltage=self.acceleration_voltage,
                           spherical_aberration=args.get("spherical_aberration", 2.7e3),
                           cutoff_frequency=args.get("cutoff_frequency", 0.5),
                           phase_shift=args.get("phase_shift", 0),
                           defocus_angle=args.get("defocus_angle", 0),
                           amplitude_contrast=args.get("amplitude_contrast", 0.07))
        stack = shift_fourier(stack, shape_is_real_fourier=False)
        np.negative(stack, out=stack)
        if args.get("flip_phase", True):
            np.abs(stack, out=stack)
        stack = np.squeeze(stack)
        if args.get("return_real_fourier", False):
            stack = crop_real_fourier(stack)
        return {"data": stack.astype(np.float32), "shape": shape,
                "return_real_fourier": args.get("return_real_fourier"),
                "is_multiplicative_filter": True}


@dataclass
class WedgeReconstructed:
    """Continuous missing wedge (tme/filters/wedge.py:282-374); the binary form used
    by the matching path (``weight_wedge=False``)."""

    angles: Tuple[float] = None
    weights: Tuple[float] = None
    weight_wedge: bool = False
    create_continuous_wedge: bool = True
    frequency_cutoff: float = 0.5
    tilt_axis: int = 0
    opening_axis: int = 2
    reconstruction_filter: str = None
    sampling_rate: float = 1

    def __post_init__(self):
        if not self.create_continuous_wedge:
            raise NotImplementedError("only the continuous wedge is implemented")
        if self.weight_wedge:
            raise NotImplementedError("weighted wedges are not implemented")
        self.angles = (min(self.angles), max(self.angles))

    @staticmethod
    def continuous_wedge(shape, angles, opening_axis, tilt_axis, **kwargs):
        angles = np.abs(np.asarray(angles))
        aspect = shape[opening_axis] / shape[tilt_axis]
        angles = np.degrees(np.arctan(np.tan(np.radians(angles)) * aspect))
        start = np.tan(np.radians(90 - angles[0]))
        stop = np.tan(np.radians(-1 * (90 - angles[1])))
        grid = np.array(np.meshgrid(*[np.arange(s) - s // 2 for s in shape], indexing="ij"))
        with np.errstate(divide="ignore", invalid="ignore"):
            ratios = np.where(grid[opening_axis] == 0, np.tan(np.radians(90)) + 1,
                              grid[tilt_axis] / grid[opening_axis])
        return np.logical_or(start <= ratios, stop >= ratios).astype(np.float32)

    def __call__(self, shape, return_real_fourier: bool = False, **kwargs) -> Dict:
        args = dict(vars(self))
        args.update(kwargs)
        ret = self.continuous_wedge(shape=shape, angles=args["angles"],
                                    opening_axis=args["opening_axis"],
                                    tilt_axis=args["tilt_axis"])
        cutoff = args.get("frequency_cutoff", None)
        if cutoff is not None:
            fm = fftfreqn(shape=shape, sampling_rate=1, compute_euclidean_norm=True)
            ret = np.multiply(ret, fm <= cutoff, out=ret)
        ret = (ret > 0) * 1.0
        ret = ret.astype(np.float32)
        ret = shift_fourier(ret, shape_is_real_fourier=False)
        if return_real_fourier:
            ret = crop_real_fourier(ret)
        return {"data": np.ascontiguousarray(ret), "shape": shape,
                "return_real_fourier": return_real_fourier, "is_multiplicative_filter": True}


class LinearWhiteningFilter:
    """Inverse square root of the radially averaged power spectrum of the target,
    normalised to a maximum of 1 and interpolated linearly
    (tme/filters/whitening.py:23-186)."""

    def __init__(self, *args, **kwargs):
        pass

    @staticmethod
    def _compute_spectrum(data_rfft, n_bins=None):
        from scipy.ndimage import mean as ndimean

        shape = tuple(data_rfft.shape)
        max_bins = max(max(shape[:-1]) // 2 + 1, shape[-1])
        n_bins = max_bins if n_bins is None else n_bins
        n_bins = int(min(n_bins, max_bins))
        bins = fftfreqn(shape=shape, sampling_rate=0.5, shape_is_real_fourier=True,
                        compute_euclidean_norm=True)
        bins = np.floor(bins * (n_bins - 1) + 0.5).astype(int)
        spec = np.fft.fftshift(data_rfft, axes=tuple(range(data_rfft.ndim - 1)))
        spec = np.abs(spec)
        np.square(spec, out=spec)
        radial = ndimean(spec, labels=bins, index=np.arange(n_bins))
        np.sqrt(radial, out=radial)
        np.reciprocal(radial, out=radial)
        np.divide(radial, radial.max(), out=radial)
        return bins, radial

    @staticmethod
    def _interpolate_spectrum(spectrum, shape, shape_is_real_fourier=True, order=1):
        from scipy.ndimage import map_coordinates

        grid = fftfreqn(shape=shape, sampling_rate=0.5,
                        shape_is_real_fourier=shape_is_real_fourier,
                        compute_euclidean_norm=True)
        # the reference scales in place; its "+ 0.5" result is discarded
        np.multiply(grid, (spectrum.shape[0] - 1), out=grid)
        out = map_coordinates(spectrum, grid.reshape(1, -1), order=order)
        return out.reshape(grid.shape)

    def __call__(self, shape, data=None, data_rfft=None, n_bins=None, order: int = 1,
                 return_real_fourier: bool = True, **kwargs) -> Dict:
        if data_rfft is None:
            data_rfft = np.fft.rfftn(np.asarray(data))
        data_rfft = np.asarray(data_rfft)
        _, radial = self._compute_spectrum(data_rfft, n_bins)
        shape = tuple(int(x) for x in shape)
        shape_filter = shape
        if return_real_fourier:
            shape_filter = list(shape)
            shape_filter[-1] = 1 + shape_filter[-1] // 2
            shape_filter = tuple(shape_filter)
        ret = self._interpolate_spectrum(radial, shape_filter,
                                         shape_is_real_fourier=return_real_fourier)
        ret = shift_fourier(ret, shape_is_real_fourier=return_real_fourier)
        return {"data": ret, "shape": shape, "return_real_fourier": return_real_fourier,
                "is_multiplicative_filter": True}


class Compose:
    """Chain filters; multiplicative filters multiply into one array
    (tme/filters/compose.py:36-59)."""

    def __init__(self, transforms):
        self.transforms = transforms

    def __call__(self, **kwargs) -> Dict:
        meta = {}
        if not len(self.transforms):
            return meta
        meta = self.transforms[0](**kwargs)
        for t in self.transforms[1:]:
            kwargs.update(meta)
            ret = t(**kwargs)
            if "data" not in ret:
                continue
            if ret.get("is_multiplicative_filter", False):
                prev = meta.pop("data")
                ret["data"] = np.multiply(ret["data"], prev)
                ret["merge"] = None
            meta = ret
        return meta


# ----------------------------------------------------------------------------- device
def _ctf_component(f: "CTFReconstructed", kwargs: Dict):
    """Float64 scalars of ``create_ctf`` for one CTF (the per-voxel part runs on the
    device)."""
    args = dict(vars(f))
    args.update(kwargs)
    if args.get("defocus_y") is not None or np.ndim(args["defocus_x"]) != 0:
        raise NotImplementedError("astigmatic or per-tilt CTFs are built on the host")
    sampling_rate = np.max(args.get("sampling_rate", 1))
    lam = _electron_wavelength(f.acceleration_voltage)
    lam /= sampling_rate
    aberration = (args.get("spherical_aberration", 2.7e3) / sampling_rate) * lam ** 2
    amp = args.get("amplitude_contrast", 0.07)
    amp_phase = np.arctan(np.divide(amp, np.sqrt(1 - np.square(amp))))
    return (1, [float(args["defocus_x"]), float(0.5 * aberration), float(np.pi * lam),
                float(args.get("phase_shift", 0)), float(amp_phase),
                float(args.get("cutoff_frequency", 0.5)),
                1.0 if args.get("flip_phase", True) else 0.0])


def _wedge_component(f: "WedgeReconstructed", shape, kwargs: Dict):
    """Float64 bounds of ``continuous_wedge`` for one wedge."""
    args = dict(vars(f))
    args.update(kwargs)
    oa, ta = int(args["opening_axis"]), int(args["tilt_axis"])
    angles = np.abs(np.asarray(args["angles"]))
    aspect = shape[oa] / shape[ta]
    angles = np.degrees(np.arctan(np.tan(np.radians(angles)) * aspect))
    start = np.tan(np.radians(90 - angles[0]))
    stop = np.tan(np.radians(-1 * (90 - angles[1])))
    at_zero = np.tan(np.radians(90)) + 1
    cutoff = args.get("frequency_cutoff", None)
    return (2, [float(start), float(stop), float(at_zero), float(oa), float(ta),
                -1.0 if cutoff is None else float(cutoff)])


def needs_spectrum(filt) -> bool:
    """Whether evaluating ``filt`` needs the data spectrum (``data_rfft``): everything but
    CTFs and wedges (whitening, unknown classes) gets it."""
    items = filt.transforms if isinstance(filt, Compose) else [filt]
    return any(type(f) not in (CTFReconstructed, WedgeReconstructed) for f in items)


def device_filter(filt, shape, return_real_fourier: bool = True, data_rfft=None, **kwargs):
    """Build ``CTFReconstructed``, ``WedgeReconstructed``, ``LinearWhiteningFilter`` or a
    ``Compose`` of them on the current GPU (``tm_build_filter``, ``tm_whitening_filter``)
    and return it as a float32 torch tensor with the DC term at index 0, equal to
    ``filt(shape=shape, return_real_fourier=..., data_rfft=data_rfft)["data"]``.

    Whitening needs ``data_rfft``, the complex64 rfft of the data on the device. It is
    built on the device alone or composed with at most one CTF and any wedges, where the
    reference's float64 product rounds the same whatever the order. Raises
    ``NotImplementedError`` for what it does not cover (astigmatic CTFs, weighted or
    per-angle wedges, several whitening filters or CTFs with whitening, other classes)."""
    import torch

    from . import _native as N

    shape = tuple(int(x) for x in shape)
    if len(shape) != 3:
        raise NotImplementedError("device filters are built for 3D shapes")
    if not torch.cuda.is_available():
        raise NotImplementedError("no CUDA device: filters are built on the host")
    items = filt.transforms if isinstance(filt, Compose) else [filt]
    comps, whiten = [], []
    for f in items:
        if type(f) is CTFReconstructed:
            comps.append(_ctf_component(f, kwargs))
        elif type(f) is WedgeReconstructed:
            comps.append(_wedge_component(f, shape, kwargs))
        elif type(f) is LinearWhiteningFilter:
            whiten.append(f)
        else:
            raise NotImplementedError(f"{type(f).__name__} is built on the host")
    if len(comps) > N.TM_FILTER_MAX_COMPONENTS or not (comps or whiten):
        raise NotImplementedError("1 to 4 filter components are built on the device")
    if len(whiten) > 1 or (whiten and sum(k == 1 for k, _ in comps) > 1):
        raise NotImplementedError("this whitening composition is built on the host")
    if whiten and (not isinstance(data_rfft, torch.Tensor) or not data_rfft.is_cuda
                   or data_rfft.dim() != 3):
        raise NotImplementedError("whitening on the device needs the data spectrum on the GPU")
    if whiten and (kwargs.get("order", 1) != 1 or kwargs.get("batch_dimension") is not None):
        raise NotImplementedError("whitening with order != 1 or batches is built on the host")
    out_shape = shape[:-1] + ((shape[-1] // 2 + 1) if return_real_fourier else shape[-1],)
    out = torch.empty(out_shape, dtype=torch.float32, device=torch.device("cuda"))
    dims = (N.c_int * 3)(*shape)
    rf = int(bool(return_real_fourier))
    if comps:
        arr = (N.FilterComponent * len(comps))()
        for i, (kind, p) in enumerate(comps):
            arr[i].kind = kind
            for j, v in enumerate(p):
                arr[i].p[j] = v
        N.check(N.lib.tm_build_filter(arr, len(comps), dims, rf, N.ptr(out), N.stream_ptr()),
                "tm_build_filter")
    if whiten:
        spec = data_rfft.to(torch.complex64).contiguous()
        ft = (N.c_int * 3)(*spec.shape)
        n_bins = kwargs.get("n_bins")
        n_bins = 0 if n_bins is None else int(n_bins)
        nb = N.lib.tm_whitening_bins(ft, n_bins)
        if nb < 2:
            raise ValueError(f"whitening: {nb} bins")
        work = torch.empty(3 * nb, dtype=torch.float64, device=out.device)
        # the other components' product (if any) is the float32 factor of the whitening
        N.check(N.lib.tm_whitening_filter(N.ptr(spec), ft, n_bins, dims, rf, N.ptr(work),
                                          N.ptr(out) if comps else None, N.ptr(out),
                                          N.stream_ptr()), "tm_whitening_filter")
    return out
