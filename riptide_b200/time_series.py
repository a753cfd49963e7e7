"""TimeSeries (time_series.py of the reference): float32 data on the host, operations on
the GPU through the C ABI; PRESTO and SIGPROC files read by the library's parallel reader."""
import copy

import numpy as np

from . import _lib, libcpp
from .libffa import downsample, generate_signal
from .timing import timing


class TimeSeries(object):
    """Time series to search with the FFA. Use the classmethods to create one."""

    def __init__(self, data, tsamp, metadata=None, copy=False):
        if copy:
            self._data = np.asarray(data, dtype=np.float32).copy()
        else:
            self._data = np.asarray(data, dtype=np.float32)
        self._tsamp = float(tsamp)
        self.metadata = dict(metadata) if metadata is not None else {}
        self.metadata["tobs"] = self.length

    @property
    def data(self):
        """numpy float32 array of the samples."""
        return self._data

    @property
    def tsamp(self):
        return self._tsamp

    def copy(self):
        return copy.deepcopy(self)

    def _device_op(self, fn, *args):
        t, _ = libcpp._as_f32(np.ascontiguousarray(self._data), 1)
        out = libcpp._empty(t.shape, t.dtype, t)
        _lib.check(fn(libcpp._ptr(t), t.numel(), *args, libcpp._ptr(out), libcpp._stream()))
        return libcpp._out(out, False)

    def normalise(self, inplace=False):
        """Zero mean, unit variance (float64 statistics), time_series.py:67-93."""
        out = self._device_op(_lib.load().rt_normalise)
        if inplace:
            self._data = out
        else:
            return TimeSeries(out, self.tsamp, metadata=self.metadata)

    @timing
    def deredden(self, width, minpts=101, inplace=False):
        """Subtract an approximate running median of `width` seconds, time_series.py:95-124."""
        out = self._device_op(_lib.load().rt_deredden, float(self.tsamp), float(width), int(minpts))
        if inplace:
            self._data = out
        else:
            return TimeSeries(out, self.tsamp, metadata=self.metadata)

    def downsample(self, factor, inplace=False):
        """Downsample by a real-valued factor, time_series.py:126-151."""
        if inplace:
            self._data = downsample(self.data, factor)
            self._tsamp *= factor
        else:
            return TimeSeries(downsample(self.data, factor), factor * self.tsamp,
                              metadata=self.metadata)

    @classmethod
    def generate(cls, length, tsamp, period, phi0=0.5, ducy=0.02, amplitude=10.0, stdnoise=1.0):
        """Noisy von Mises pulse train (time_series.py:176-237)."""
        nsamp = int(round(length / tsamp))
        data = generate_signal(nsamp, period / tsamp, phi0=phi0, ducy=ducy, amplitude=amplitude,
                               stdnoise=stdnoise)
        metadata = {"source_name": "fake", "signal_shape": "Von Mises", "signal_period": period,
                    "signal_initial_phase": phi0, "signal_duty_cycle": ducy}
        return cls(data, tsamp, copy=False, metadata=metadata)

    @classmethod
    def from_numpy_array(cls, array, tsamp, copy=False):
        return cls(array, tsamp, copy=copy)

    @classmethod
    def from_binary(cls, fname, tsamp, dtype=np.float32):
        return cls(np.fromfile(fname, dtype=dtype), tsamp, copy=False)

    @classmethod
    def from_npy_file(cls, fname, tsamp):
        return cls(np.load(fname), tsamp, copy=False)

    @classmethod
    @timing
    def from_presto_inf(cls, fname):
        """TimeSeries of a PRESTO .inf file and its .dat samples (time_series.py:300-336).
        Warns for X-ray and gamma-ray data."""
        from .reading import SeriesFile, read_payload
        sf = SeriesFile.from_presto_inf(fname)
        return cls(read_payload(sf.path, sf.offset, sf.nsamp, sf.encoding), tsamp=sf.tsamp,
                   metadata=sf.metadata)

    @classmethod
    @timing
    def from_sigproc(cls, fname, extra_keys=None):
        """TimeSeries of a SIGPROC dedispersed time series, 32-bit float or 8-bit with a
        'signed' header key (time_series.py:338-379). `extra_keys`: {key: type} of
        non-standard header keys."""
        from .reading import SeriesFile, read_payload
        sf = SeriesFile.from_sigproc(fname, extra_keys=extra_keys)
        return cls(read_payload(sf.path, sf.offset, sf.nsamp, sf.encoding), tsamp=sf.tsamp,
                   metadata=sf.metadata)

    def fold(self, period, bins, subints=None):
        """Fold at `period` seconds into `bins` phase bins (time_series.py:153-174,
        folding.py:21-85)."""
        from .folding import fold
        return fold(self, period, bins, subints=subints)

    @property
    def nsamp(self):
        return self.data.size

    @property
    def length(self):
        return self.nsamp * self.tsamp

    @property
    def tobs(self):
        return self.length

    def __str__(self):
        return "{name} {{nsamp = {x.nsamp:d}, tsamp = {x.tsamp:.4e}, tobs = {x.length:.3f}}}".format(
            name=type(self).__name__, x=self)

    __repr__ = __str__

    @classmethod
    def from_dict(cls, items):
        return cls(items["data"], items["tsamp"], metadata=items["metadata"], copy=False)

    def to_dict(self):
        return {"data": self.data, "tsamp": self.tsamp, "metadata": self.metadata}
