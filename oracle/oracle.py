"""TEST INFRASTRUCTURE ONLY -- the CPU checker for riptide's FFA search path.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` import this module. The product package (``riptide_b200``) never
does: its kernels run on the GPU or raise.

Two checkers live here:

* ``C``      -- ctypes binding of ``riptide_oracle.c`` (a restatement of the reference's
               C++ headers, cpp/*.hpp, float32 and FP64 variants).
* ``ref_libcpp()`` -- the reference's own pybind11 module ``libcpp`` compiled from its
               sources by ``oracle/Makefile`` (target ``ref``, run by the build entry point
               where the reference sources are present) into ``oracle/_ref/``. The built
               module is not committed; it exists in a working tree where that build ran,
               and is None elsewhere.

and a numpy restatement of the Python glue around them: ``generate_width_trials``
(ffautils.py:4-11), ``scrunch`` / ``fast_running_median`` (running_medians.py:40-85),
``deredden`` (time_series.py:95-124), ``normalise`` (time_series.py:67-93) and
``ffa_search`` (search.py:11-93). Parity of the glue is pinned against fixtures generated
by the reference's own Python code (tests/golden/make_golden.py).
"""
import ctypes
import glob
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(HERE, "_build", "libriptide_oracle.so")

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_sz = ctypes.c_size_t
_d = ctypes.c_double


def build():
    """Compile the C restatement (make -C oracle)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


class _COracle:
    def __init__(self, path=_LIB_PATH):
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        self.lib = lib
        lib.ora_last_error.restype = ctypes.c_char_p
        lib.ora_downsampled_size.restype = _sz
        lib.ora_downsampled_size.argtypes = [_sz, _d]
        lib.ora_downsampled_variance.restype = _d
        lib.ora_downsampled_variance.argtypes = [_sz, _d]
        lib.ora_periodogram_length.restype = ctypes.c_int
        lib.ora_periodogram_length.argtypes = [_sz, _d, _d, _d, _sz, _sz, ctypes.POINTER(_sz)]
        lib.ora_running_median.restype = ctypes.c_int
        lib.ora_running_median.argtypes = [_f32p, _sz, _sz, _f32p]
        for pre, fp in (("ora_", _f32p), ("ora64_", _f64p)):
            getattr(lib, pre + "ffa2").restype = ctypes.c_int
            getattr(lib, pre + "ffa2").argtypes = [fp, _sz, _sz, fp]
            getattr(lib, pre + "snr2").restype = None
            getattr(lib, pre + "snr2").argtypes = [
                fp, _sz, _sz, _u64p, _sz,
                ctypes.c_float if pre == "ora_" else _d, fp,
            ]
            getattr(lib, pre + "downsample").restype = ctypes.c_int
            getattr(lib, pre + "downsample").argtypes = [fp, _sz, _d, fp]
            getattr(lib, pre + "periodogram").restype = ctypes.c_int
            getattr(lib, pre + "periodogram").argtypes = [
                fp, _sz, _d, _u64p, _sz, _d, _d, _sz, _sz, _f64p, _u32p, fp,
            ]
            getattr(lib, pre + "circular_prefix_sum").restype = None
            getattr(lib, pre + "circular_prefix_sum").argtypes = [fp, _sz, _sz, fp]
            getattr(lib, pre + "rollback").restype = None
            getattr(lib, pre + "rollback").argtypes = [fp, _sz, _sz, fp]
            getattr(lib, pre + "fused_rollback_add").restype = None
            getattr(lib, pre + "fused_rollback_add").argtypes = [fp, fp, _sz, _sz, fp]
        lib.ora_check_snr_args.restype = ctypes.c_int
        lib.ora_check_snr_args.argtypes = [_u64p, _sz, _sz, ctypes.c_float]

    def _err(self):
        return ValueError(self.lib.ora_last_error().decode())

    @staticmethod
    def _dt(f64):
        return np.float64 if f64 else np.float32

    def ffa2(self, x, f64=False):
        x = np.ascontiguousarray(x, dtype=self._dt(f64))
        if x.ndim != 2:
            raise ValueError("input must be 2D")
        out = np.empty_like(x)
        fn = self.lib.ora64_ffa2 if f64 else self.lib.ora_ffa2
        if fn(x, x.shape[0], x.shape[1], out):
            raise self._err()
        return out

    def snr2(self, x, widths, stdnoise=1.0, f64=False):
        x = np.ascontiguousarray(x, dtype=self._dt(f64))
        widths = np.ascontiguousarray(widths, dtype=np.uint64)
        if self.lib.ora_check_snr_args(widths, widths.size, x.shape[1], stdnoise):
            raise self._err()
        out = np.empty((x.shape[0], widths.size), dtype=self._dt(f64))
        fn = self.lib.ora64_snr2 if f64 else self.lib.ora_snr2
        fn(x, x.shape[0], x.shape[1], widths, widths.size, stdnoise, out)
        return out

    def downsample(self, x, f, f64=False):
        x = np.ascontiguousarray(x, dtype=self._dt(f64))
        if not ((f > 1.0) and (f <= x.size)):
            raise ValueError("Downsampling factor must verify: 1 < f <= size")
        out = np.empty(self.lib.ora_downsampled_size(x.size, f), dtype=self._dt(f64))
        fn = self.lib.ora64_downsample if f64 else self.lib.ora_downsample
        if fn(x, x.size, f, out):
            raise self._err()
        return out

    def downsampled_size(self, n, f):
        return self.lib.ora_downsampled_size(n, f)

    def downsampled_variance(self, n, f):
        return self.lib.ora_downsampled_variance(n, f)

    def periodogram_length(self, size, tsamp, pmin, pmax, bmin, bmax):
        L = _sz(0)
        if self.lib.ora_periodogram_length(size, tsamp, pmin, pmax, bmin, bmax, ctypes.byref(L)):
            raise self._err()
        return L.value

    def periodogram(self, data, tsamp, widths, pmin, pmax, bmin, bmax, f64=False):
        data = np.ascontiguousarray(data, dtype=self._dt(f64))
        widths = np.ascontiguousarray(widths, dtype=np.uint64)
        L = self.periodogram_length(data.size, tsamp, pmin, pmax, bmin, bmax)
        periods = np.empty(L, dtype=np.float64)
        foldbins = np.empty(L, dtype=np.uint32)
        snrs = np.empty((L, widths.size), dtype=self._dt(f64))
        fn = self.lib.ora64_periodogram if f64 else self.lib.ora_periodogram
        if fn(data, data.size, tsamp, widths, widths.size, pmin, pmax, bmin, bmax,
              periods, foldbins, snrs):
            raise self._err()
        return periods, foldbins, snrs

    def running_median(self, x, width):
        x = np.ascontiguousarray(x, dtype=np.float32)
        if x.ndim != 1:
            raise ValueError("data must be 1D")
        out = np.empty_like(x)
        if self.lib.ora_running_median(x, x.size, width, out):
            raise self._err()
        return out

    def circular_prefix_sum(self, x, nsum, f64=False):
        x = np.ascontiguousarray(x, dtype=self._dt(f64))
        out = np.empty(max(nsum, x.size), dtype=self._dt(f64))
        fn = self.lib.ora64_circular_prefix_sum if f64 else self.lib.ora_circular_prefix_sum
        fn(x, x.size, nsum, out)
        return out[:nsum]


_C = None


def C():
    """The C restatement (built on first use)."""
    global _C
    if _C is None:
        _C = _COracle()
    return _C


def ref_libcpp():
    """The reference's own ``libcpp`` module built into oracle/_ref, or None."""
    paths = sorted(glob.glob(os.path.join(HERE, "_ref", "libcpp*.so")))
    if not paths:
        return None
    spec = importlib.util.spec_from_file_location("libcpp", paths[0])
    mod = importlib.util.module_from_spec(spec)
    try:
        spec.loader.exec_module(mod)
    except (ImportError, OSError):
        return None
    return mod


# ------------------------------------------------------------------------------------
# numpy restatement of the Python glue
# ------------------------------------------------------------------------------------
def generate_width_trials(nbins, ducy_max=0.20, wtsp=1.5):
    """ffautils.py:4-11"""
    widths = []
    w = 1
    wmax = int(max(1, ducy_max * nbins))
    while w <= wmax:
        widths.append(w)
        w = int(max(w + 1, wtsp * w))
    return np.asarray(widths)


def scrunch(data, factor):
    """running_medians.py:40-46 (float32 numpy mean over groups of `factor`)."""
    factor = int(factor)
    N = (data.size // factor) * factor
    return data[:N].reshape(-1, factor).mean(axis=1)


def fast_running_median(data, width_samples, min_points=101, rmed=None):
    """running_medians.py:49-85. `rmed` is the exact running median used on the
    scrunched series (default: the C restatement)."""
    rmed = rmed or C().running_median
    if not (min_points % 2):
        raise ValueError("min_points must be an odd number")
    scrunch_factor = int(max(1, width_samples / float(min_points)))
    if scrunch_factor == 1:
        return rmed(np.ascontiguousarray(data), width_samples)
    scrunched = scrunch(data, scrunch_factor)
    rmed_lores = rmed(np.ascontiguousarray(scrunched), min_points)
    x_lores = np.arange(scrunched.size) * scrunch_factor + 0.5 * (scrunch_factor - 1)
    return np.interp(np.arange(data.size), x_lores, rmed_lores)


def deredden(data, tsamp, width, minpts=101, rmed=None):
    """time_series.py:95-124 (out-of-place): float32(data - running median)."""
    data = np.asarray(data, dtype=np.float32)
    width_samples = int(round(width / tsamp))
    rm = fast_running_median(data, width_samples, minpts, rmed=rmed)
    return np.asarray(data - rm, dtype=np.float32)


def normalise(data):
    """time_series.py:67-93 (out-of-place): float32((x - mean) / std), f64 statistics."""
    data = np.asarray(data, dtype=np.float32)
    m = data.mean(dtype=np.float64)
    v = data.var(dtype=np.float64)
    norm = v ** 0.5
    return np.asarray((data - m) / norm, dtype=np.float32)


def ffa_search(data, tsamp, period_min=1.0, period_max=30.0, fpmin=8, bins_min=240,
               bins_max=260, ducy_max=0.20, wtsp=1.5, deredden_=True, rmed_width=4.0,
               rmed_minpts=101, already_normalised=False, libcpp=None):
    """search.py:11-93. Returns (searched float32 series, widths, periods, foldbins, snrs).
    `libcpp` selects the periodogram implementation: None -> the C restatement,
    or a module with the reference's `periodogram` / `running_median` signatures."""
    del fpmin  # accepted and ignored, as in search.py:15 vs :82-93
    data = np.asarray(data, dtype=np.float32)
    rmed = None if libcpp is None else libcpp.running_median
    if deredden_:
        data = deredden(data, tsamp, rmed_width, minpts=rmed_minpts, rmed=rmed)
    if not already_normalised:
        data = normalise(data)
    widths = generate_width_trials(bins_min, ducy_max=ducy_max, wtsp=wtsp)
    if libcpp is None:
        periods, foldbins, snrs = C().periodogram(
            data, tsamp, widths, period_min, period_max, bins_min, bins_max)
    else:
        periods, foldbins, snrs = libcpp.periodogram(
            data, tsamp, widths.astype(np.uint64), period_min, period_max, bins_min, bins_max)
    return data, widths, periods, foldbins, snrs


# ------------------------------------------------------------------------------------------
# Peak detection (peak_detection.py:38-240, clustering.py:4-48)
# ------------------------------------------------------------------------------------------
def cluster1d(x, r, already_sorted=False):
    """clustering.py:4-48: friends-of-friends in 1D, clusters as arrays of indices."""
    if not len(x):
        return []
    if not already_sorted:
        indices = x.argsort()
        diff = np.diff(x[indices])
    else:
        indices = np.arange(len(x))
        diff = np.diff(x)
    ibreaks = np.where(abs(diff) > r)[0]
    if not len(ibreaks):
        return [indices]
    ibounds = np.concatenate(([0], ibreaks + 1, [len(x)]))
    return [indices[a:b] for a, b in zip(ibounds[:-1], ibounds[1:])]


def segment_stats(f, s, T, segwidth=5.0):
    """peak_detection.py:38-86: centre frequency, median S/N and IQR-based S/N deviation of
    consecutive segments of `segwidth / T` Hz."""
    import math

    w = segwidth / T
    m = math.ceil(abs(f[-1] - f[0]) / w)
    p = len(f) // m
    n = m * p
    fc = np.median(f[:n].reshape(m, p), axis=1)
    s25, smed, s75 = np.percentile(s[:n].reshape(m, p), (25, 50, 75), axis=-1)
    return fc, smed, (s75 - s25) / 1.349


def find_peaks(periods, foldbins, snrs, widths, tobs, dm=None, smin=6.0, segwidth=5.0,
               nstd=6.0, minseg=10, polydeg=2, clrad=0.1):
    """peak_detection.py:112-240 on periodogram arrays. Returns (peaks, polycos): peaks as
    tuples (period, freq, width, ducy, iw, ip, snr, dm) sorted by decreasing S/N, polycos as
    {iw: coefficient list}."""
    f = 1.0 / periods
    T = tobs
    peaks, polycos = [], {}
    for iw, width in enumerate(widths):
        s = snrs[:, iw].astype(float)
        fc, smed, sstd = segment_stats(f, s, T, segwidth=segwidth)
        sc = smed + nstd * sstd
        if len(fc) >= minseg:
            poly = np.poly1d(np.polyfit(np.log(fc), sc, polydeg))
            polyco = poly.coefficients
        else:
            polyco = [smin]
            poly = np.poly1d(polyco)
        dynthr = poly(np.log(f))
        indices = np.where((s > dynthr) & (s > smin))[0]
        for cl in cluster1d(f[indices], clrad / T):
            ix = indices[cl]
            ip = ix[s[ix].argmax()]
            pf = f[ip]
            peaks.append((float(1.0 / pf), float(pf), int(width), float(width) / foldbins[ip],
                          int(iw), int(ip), float(s[ip]), dm))
        polycos[iw] = polyco
    peaks = sorted(peaks, key=lambda p: p[6], reverse=True)
    return peaks, polycos


def downsample_vertical(X, factor):
    """folding.py:6-18: each column downsampled by `factor` (the C restatement of
    downsample.hpp)."""
    m = X.shape[0]
    if not factor > 1:
        raise ValueError("factor must be > 1")
    if not factor < m:
        raise ValueError("factor must be strictly smaller than the number of input lines")
    Y = np.ascontiguousarray(X.T)
    return np.ascontiguousarray(np.asarray([C().downsample(col, factor) for col in Y]).T)


def fold(data, tsamp, period, bins, subints=None):
    """folding.py:21-85 (TimeSeries.fold): downsample by (period / bins) / tsamp, reshape to
    (m, bins), scale by (m * factor) ** -0.5 in float32, then sum / keep / column-downsample."""
    length = data.size * tsamp
    if period > length:
        raise ValueError("Period exceeds data length")
    tbin = period / bins
    if not tbin > tsamp:
        raise ValueError("Bin width is shorter than sampling time")
    if subints is not None:
        subints = int(subints)
        if not subints >= 1:
            raise ValueError("subints must be >= 1 or None")
        if subints > length / period:
            raise ValueError("subints exceeds the number of signal periods that fit in the data")
    factor = tbin / tsamp
    down = C().downsample(np.asarray(data, dtype=np.float32), factor)
    m = down.size // bins
    folded = down[:m * bins].reshape(m, bins).copy()
    folded *= (m * factor) ** -0.5
    if subints == 1 or m == 1:
        return folded.sum(axis=0)
    if subints is None or subints == m:
        return folded
    return downsample_vertical(folded, m / subints)
