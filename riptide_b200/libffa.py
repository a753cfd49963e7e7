"""FFA helper functions (libffa.py of the reference), computed on the GPU."""
import numpy as np
from numpy import cos, exp, log, pi, sin

from . import libcpp


def generate_signal(nsamp, period, phi0=0.5, ducy=0.02, amplitude=10.0, stdnoise=1.0, rng=None):
    """Von Mises pulse train plus white noise (libffa.py:15-68). `amplitude` is the expected
    folded S/N with a matched filter. `rng` (numpy Generator) defaults to np.random."""
    kappa = log(2.0) / (2.0 * sin(pi * ducy / 2.0) ** 2)
    phase_radians = (np.arange(nsamp, dtype=float) / period - phi0) * (2 * pi)
    signal = exp(kappa * (cos(phase_radians) - 1.0))
    scale_factor = amplitude * (signal ** 2).sum() ** -0.5
    signal *= scale_factor
    if stdnoise > 0.0:
        gen = rng if rng is not None else np.random
        noise = gen.normal(size=nsamp, loc=0.0, scale=stdnoise)
    else:
        noise = 0.0
    return signal + noise


def ffa2(data):
    """FFA transform of a (m, p) array (libffa.py:71-91)."""
    return libcpp.ffa2(data)


def ffa1(data, p):
    """FFA transform of a 1D series at base period p samples (libffa.py:94-126)."""
    if not data.ndim == 1:
        raise ValueError("input data must be one-dimensional")
    if not (isinstance(p, int) and p > 0):
        raise ValueError("p must be an integer > 1")
    if p > data.size:
        raise ValueError("p must be smaller than the total number of samples")
    m = data.size // p
    return ffa2(data[: m * p].reshape(m, p))


def ffafreq(N, p, dt=1.0):
    """Trial frequencies of the FFA output rows (libffa.py:129-169)."""
    if not (isinstance(N, int) and N > 0):
        raise ValueError("N must be a strictly positive integer")
    if not (isinstance(p, int) and p > 1):
        raise ValueError("p must be an integer > 1")
    if not N >= p:
        raise ValueError("p must be smaller than (or equal to) N")
    if not dt > 0:
        raise ValueError("dt must be strictly positive")
    f0 = 1.0 / p
    m = N // p
    if m == 1:
        f = np.asarray([f0])
    else:
        s = np.arange(m)
        f = f0 - s / (m - 1.0) * f0 ** 2
    f /= dt
    return f


def ffaprd(N, p, dt=1.0):
    """Trial periods of the FFA output rows (libffa.py:172-191)."""
    return 1.0 / ffafreq(N, p, dt=dt)


def boxcar_snr(data, widths, stdnoise=1.0):
    """S/N of profiles (last axis = phase) for boxcar widths (libffa.py:194-225)."""
    widths = np.asarray(widths, dtype=np.uint64)
    b = data.shape[-1]
    cppinput = data.reshape(-1, b).astype(np.float32)
    snr = libcpp.snr2(cppinput, widths, stdnoise)
    shape = list(data.shape[:-1]) + [widths.size]
    return snr.reshape(shape)


def downsample(data, factor):
    """Downsample by a real-valued factor (libffa.py:228-243)."""
    return libcpp.downsample(data, factor)
