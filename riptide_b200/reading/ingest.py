"""Loading of time series payloads through the library's file reader (rt_read_file,
rt_ingest_files): one file into host memory, or a batch of files straight into one packed
float32 device tensor, the layout BatchedSearch.run takes."""
import ctypes
import os
import typing

import numpy as np

from .. import _lib

_ENCODINGS = {"f32": _lib.RT_SAMPLES_F32, "u8": _lib.RT_SAMPLES_U8, "i8": _lib.RT_SAMPLES_I8}
_SAMPLE_BYTES = {"f32": 4, "u8": 1, "i8": 1}
_NUMPY = {"f32": np.float32, "u8": np.uint8, "i8": np.int8}


def _threads(threads):
    return int(threads) if threads else max(1, min(16, os.cpu_count() or 1))


class SeriesFile(typing.NamedTuple):
    """Where the samples of one time series file are: `nsamp` samples of `encoding`
    ("f32", "u8" or "i8") from byte `offset` of `path`; `tsamp` in seconds."""

    path: str
    offset: int
    nsamp: int
    encoding: str
    tsamp: float
    metadata: dict

    @classmethod
    def from_presto_inf(cls, fname):
        """The .dat payload of a PRESTO .inf file (time_series.py:300-336): all of the .dat
        file, float32. Warns for X-ray and gamma-ray data, as the reference does."""
        from ..metadata import Metadata
        from .presto import PrestoInf
        inf = PrestoInf(fname)
        md = Metadata.from_presto_inf(inf)
        _warn_band(fname, md)
        size = _file_size(inf.data_fname)
        return cls(inf.data_fname, 0, size // 4, "f32", float(inf["tsamp"]), md)

    @classmethod
    def from_sigproc(cls, fname, extra_keys=None):
        """The payload of a SIGPROC time series (time_series.py:338-379): after the header,
        float32 for nbits = 32, int8 / uint8 by the 'signed' key for nbits = 8."""
        from ..metadata import Metadata
        from .sigproc import SigprocHeader
        sh = SigprocHeader(fname, extra_keys=extra_keys)
        md = Metadata.from_sigproc(sh, extra_keys=extra_keys)
        enc = "f32" if md["nbits"] != 8 else ("i8" if md["signed"] else "u8")
        nsamp = (_file_size(sh.fname) - sh.bytesize) // _SAMPLE_BYTES[enc]
        return cls(sh.fname, int(sh.bytesize), int(nsamp), enc, float(sh["tsamp"]), md)


def _warn_band(fname, md):
    band = md.get("em_band")
    if band in ("X-ray", "Gamma"):
        import warnings
        warnings.warn(
            f" You have loaded file {fname!r}, which contains data observed at a high-energy "
            f"band {band!r}. riptide is NOT designed to process low photon count time series, "
            "i.e. where the background noise statistics are non-Gaussian. Be VERY careful when "
            "interpreting any search outputs.", category=UserWarning)


def _file_size(path):
    size = ctypes.c_uint64(0)
    _lib.check(_lib.load().rt_file_size(os.fsencode(path), ctypes.byref(size)))
    return int(size.value)


def read_payload(path, offset, nsamp, encoding, threads=None):
    """`nsamp` samples (all that follow `offset` when None) of `encoding` from a file, as a
    float32 host array (astype(np.float32) of the stored type)."""
    esz = _SAMPLE_BYTES[encoding]
    if nsamp is None:
        nsamp = (_file_size(path) - int(offset)) // esz
    raw = np.empty(int(nsamp), dtype=_NUMPY[encoding])
    _lib.check(_lib.load().rt_read_file(os.fsencode(path), int(offset), raw.nbytes,
                                        raw.ctypes.data_as(ctypes.c_void_p), _threads(threads)))
    return raw if encoding == "f32" else raw.astype(np.float32)


def describe(fnames, fmt="presto", extra_keys=None):
    """SeriesFile of each file name (`fmt`: "presto" for .inf files, "sigproc" for .tim)."""
    if fmt == "presto":
        return [SeriesFile.from_presto_inf(f) for f in fnames]
    if fmt == "sigproc":
        return [SeriesFile.from_sigproc(f, extra_keys=extra_keys) for f in fnames]
    raise ValueError(f"unknown time series format {fmt!r}")


def load_series_batch(files, device="cuda", threads=None, staging_bytes=64 << 20, out=None):
    """Load the payloads of `files` (SeriesFile list) into one packed float32 CUDA tensor,
    series back to back, on the current stream. 8-bit payloads are copied to the device as
    bytes and widened there. Returns (tensor, lengths int64 array)."""
    from .. import libcpp
    torch = libcpp._t()
    lengths = np.asarray([f.nsamp for f in files], dtype=np.int64)
    total = int(lengths.sum())
    if out is None:
        out = torch.empty(total, dtype=torch.float32, device=device)
    elif not (out.dtype == torch.float32 and out.is_cuda and out.is_contiguous()
              and out.numel() == total):
        raise ValueError("out must be a contiguous float32 CUDA tensor of the total length")
    if not files:
        return out, lengths
    staging = torch.empty(int(staging_bytes), dtype=torch.uint8, pin_memory=True)
    paths = (ctypes.c_char_p * len(files))(*[os.fsencode(f.path) for f in files])
    offs = np.ascontiguousarray([f.offset for f in files], dtype=np.uint64)
    ns = np.ascontiguousarray(lengths.astype(np.uint64))
    encs = (ctypes.c_int * len(files))(*[_ENCODINGS[f.encoding] for f in files])
    _lib.check(_lib.load().rt_ingest_files(
        paths, offs.ctypes.data_as(_lib._u64p), ns.ctypes.data_as(_lib._u64p), encs, len(files),
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(staging.data_ptr()), staging.numel(),
        _threads(threads), libcpp._stream()))
    return out, lengths
