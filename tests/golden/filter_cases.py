"""Filter parameter sets shared by the golden-vector generator and the filter tests:
each case is built once with the reference's classes (tests/golden/make_golden.py) and
once with this package's host and device builders."""

FILTER_CASES = [
    # (shape, components, return_real_fourier); components: ("ctf", kwargs) / ("wedge", kwargs)
    ((12, 12, 12), [("wedge", dict(angles=(60, 60), opening_axis=2, tilt_axis=0)),
                    ("ctf", dict(defocus_x=30000.0, sampling_rate=6.8))], True),
    ((13, 11, 9), [("ctf", dict(defocus_x=15000.0, sampling_rate=6.8, flip_phase=False))], True),
    ((13, 11, 9), [("wedge", dict(angles=(40, 55), opening_axis=1, tilt_axis=0))], False),
    ((32, 32, 32), [("ctf", dict(defocus_x=45000.0, sampling_rate=1.0,
                                 acceleration_voltage=200e3, amplitude_contrast=0.1,
                                 phase_shift=30.0)),
                    ("wedge", dict(angles=(50, 65), opening_axis=0, tilt_axis=2))], True),
    ((40, 36, 30), [("wedge", dict(angles=(60, 60), opening_axis=2, tilt_axis=0,
                                   frequency_cutoff=0.35))], True),
    ((21, 20, 19), [("wedge", dict(angles=(55, 55), opening_axis=2, tilt_axis=1)),
                    ("ctf", dict(defocus_x=25000.0, sampling_rate=4.4, flip_phase=True))], False),
    ((64, 48, 40), [("ctf", dict(defocus_x=35000.0, sampling_rate=13.6,
                                 spherical_aberration=2.0e7))], True),
]


def build_filter_case(case, ctf_cls, wedge_cls, compose_cls):
    """The case's filter from the given classes (the reference's or this package's)."""
    shape, comps, rfft = case
    objs = []
    for kind, kw in comps:
        if kind == "ctf":
            objs.append(ctf_cls(**kw))
        else:
            objs.append(wedge_cls(create_continuous_wedge=True, **kw))
    return compose_cls(objs)(shape=shape, return_real_fourier=rfft)["data"]




# Whitening by the power spectrum of seeded data: (data shape, filter shape,
# return_real_fourier, n_bins). The data is normal noise times a radial ramp (a spectrum
# that is not flat), seed = case index; its rfft in complex64 is what the filter gets.
WHITENING_CASES = [
    ((24, 20, 16), (24, 20, 16), True, None),
    ((21, 17, 15), (21, 17, 15), True, None),
    ((24, 20, 16), (12, 12, 12), True, None),
    ((16, 16, 16), (16, 16, 16), False, None),
    ((20, 24, 18), (20, 24, 18), True, 7),
]


def whitening_data(case_index, shape):
    """The seeded data of a whitening case and its complex64 rfft."""
    import numpy as np

    rng = np.random.default_rng(case_index)
    grids = np.meshgrid(*[np.arange(n) - n / 2 for n in shape], indexing="ij")
    ramp = 1.0 + np.sqrt(sum(g * g for g in grids))
    data = (rng.normal(size=shape) * ramp).astype(np.float32)
    return data, np.fft.rfftn(data).astype(np.complex64)
