"""Folding of time series at trial periods (folding.py of the reference), on the GPU
(rt_fold / rt_fold_batched)."""
import ctypes

import numpy as np

from . import _lib, libcpp
from .libffa import downsample


def downsample_vertical(X, factor):
    """Downsample each column of a 2D array by a real factor (folding.py:6-18)."""
    m, _ = X.shape
    if not factor > 1:
        raise ValueError("factor must be > 1")
    if not factor < m:
        raise ValueError("factor must be strictly smaller than the number of input lines")
    Y = np.ascontiguousarray(np.asarray(X, dtype=np.float32).T)
    out = np.asarray([downsample(col, factor) for col in Y])
    return np.ascontiguousarray(out.T)


def _subints_arg(subints):
    if subints is None:
        return -1
    s = int(subints)
    if s < 1:
        raise ValueError("subints must be >= 1 or None")
    return s


def fold_shape(nsamp, tsamp, period, bins, subints=None):
    """Shape of fold()'s output for a series of nsamp samples: (bins,) or (rows, bins)."""
    rows, ndim = ctypes.c_size_t(0), ctypes.c_int(0)
    _lib.check(_lib.load().rt_fold_shape(int(nsamp), float(tsamp), float(period), int(bins),
                                         _subints_arg(subints), ctypes.byref(rows),
                                         ctypes.byref(ndim)))
    return (int(bins),) if ndim.value == 1 else (int(rows.value), int(bins))


def fold_batched(ts, periods, bins, subints=None):
    """Fold one TimeSeries at many periods in one launch (candidate folding). `bins` and
    `subints` are scalars or one per period. Returns a list of numpy float32 arrays shaped as
    fold() returns them."""
    torch = libcpp._t()
    periods = np.ascontiguousarray(np.asarray(periods, dtype=np.float64).ravel())
    count = periods.size
    bins_a = np.ascontiguousarray(np.broadcast_to(np.asarray(bins, dtype=np.uint64), (count,)))
    subs = subints if isinstance(subints, (list, tuple, np.ndarray)) else [subints] * count
    subs_a = np.ascontiguousarray([_subints_arg(s) for s in subs], dtype=np.int64)
    shapes = [fold_shape(ts.nsamp, ts.tsamp, p, int(b), s)
              for p, b, s in zip(periods, bins_a, subs)]
    sizes = np.asarray([int(np.prod(s)) for s in shapes], dtype=np.uint64)
    offs = np.ascontiguousarray(np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.uint64))
    if count == 0:
        return []
    x, _ = libcpp._as_f32(np.ascontiguousarray(ts.data), 1)
    out = torch.empty(int(sizes.sum()), dtype=torch.float32, device=x.device)
    vp = ctypes.c_void_p
    _lib.check(_lib.load().rt_fold_batched(
        libcpp._ptr(x), x.numel(), float(ts.tsamp), periods.ctypes.data_as(vp),
        bins_a.ctypes.data_as(vp), subs_a.ctypes.data_as(vp), count,
        offs.ctypes.data_as(_lib._u64p), libcpp._ptr(out), libcpp._stream()))
    host = out.cpu().numpy()
    return [host[int(o):int(o) + int(n)].reshape(s) for o, n, s in zip(offs, sizes, shapes)]


def fold(ts, period, bins, subints=None):
    """Fold a TimeSeries at `period` seconds into `bins` phase bins (folding.py:21-85):
    (subints, bins) sub-integrations, all full periods when subints is None, or one profile of
    `bins` values when subints == 1. ValueError for the reference's invalid arguments."""
    return fold_batched(ts, [period], int(bins), subints)[0]


def candidate_subints(period, subints, length):
    """The sub-integrations a pipeline candidate is folded with (candidate.py:76-104): the
    requested number, or None (every full period in the data) when that many periods do not
    fit in the series."""
    if subints is not None and subints * period >= length:
        return None
    return subints


def fold_candidates(ts, periods, bins, subints=1):
    """Fold one TimeSeries at every candidate period in one launch, with the candidate stage's
    rule for sub-integrations (candidate_subints). Returns the list of folded arrays."""
    subs = [candidate_subints(float(p), subints, ts.length) for p in np.asarray(periods).ravel()]
    return fold_batched(ts, periods, bins, subs)
