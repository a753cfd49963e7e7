"""SIGPROC dedispersed time series headers (reading/sigproc.py of the reference).

The header is a sequence of (key, value) attributes between the strings HEADER_START and
HEADER_END. A string is a native int32 length followed by its bytes; a value is stored by the
type of its key: int as int32, float as a C double, bool as one unsigned byte, str as a
string. The payload (the samples) follows the header.
"""
import os
import struct

HEADER_START = "HEADER_START"
HEADER_END = "HEADER_END"

# Types of the standard keys (the table sigproc.py:17-60 of the reference uses; it is the
# SIGPROC header format, so it has to be the same).
sigproc_keydb = {}
for _k in ("filename", "telescope", "rawdatafile", "source_name", "obs_date", "obs_time"):
    sigproc_keydb[_k] = str
for _k in ("telescope_id", "machine_id", "data_type", "barycentric", "pulsarcentric", "nbits",
           "nsamples", "nchans", "nifs", "nbeams", "ibeam", "hdrlen", "orig_hdrlen",
           "new_hdrlen", "sampsize"):
    sigproc_keydb[_k] = int
for _k in ("az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "fch1", "foff",
           "fchannel", "refdm", "flux", "period", "pb", "ecc", "asini", "bandwidth", "fbottom",
           "ftop", "accel"):
    sigproc_keydb[_k] = float
sigproc_keydb["signed"] = bool
del _k

_FORMATS = {int: ("i", 4), float: ("d", 8), bool: ("B", 1)}


def _read_exact(f, n):
    b = f.read(n)
    if len(b) != n:
        raise ValueError("SIGPROC header ends before HEADER_END")
    return b


def _read_str(f):
    (size,) = struct.unpack("i", _read_exact(f, 4))
    if size < 0:
        raise ValueError(f"invalid SIGPROC string length {size}")
    return _read_exact(f, size).decode()


def read_sigproc_header(fobj, extra_keys=None):
    """(attributes dict, header size in bytes) of an open binary file (sigproc.py:101-145).
    `extra_keys`: {key: type} for non-standard keys, or to override a standard key's type.
    KeyError for a key of unknown type."""
    keydb = dict(sigproc_keydb)
    if extra_keys:
        keydb.update(extra_keys)
    fobj.seek(0)
    flag = _read_str(fobj)
    if flag != HEADER_START:
        raise AssertionError(f"File starts with '{flag}' flag instead of the expected '{HEADER_START}'")
    attrs = {}
    while True:
        key = _read_str(fobj)
        if key == HEADER_END:
            break
        kind = keydb.get(key)
        if kind is None:
            raise KeyError(f"Type of SIGPROC header attribute '{key}' is unknown, please specify it")
        if kind is str:
            val = _read_str(fobj)
        elif kind in _FORMATS:
            fmt, n = _FORMATS[kind]
            (val,) = struct.unpack(fmt, _read_exact(fobj, n))
            if kind is bool:
                val = bool(val)
        else:
            raise ValueError(f"Key '{key}' has unsupported type '{kind}'")
        attrs[key] = val
    return attrs, fobj.tell()


def parse_float_coord(f):
    """SIGPROC's packed decimal coordinate (hhmmss.s or ddmmss.s) in hours or degrees."""
    sign = -1.0 if f < 0 else (1.0 if f > 0 else 0.0)
    x = abs(f)
    hh, x = divmod(x, 10000.0)
    mm, ss = divmod(x, 100.0)
    return sign * (hh + mm / 60.0 + ss / 3600.0)


class SigprocHeader(dict):
    """The header attributes of a SIGPROC file (sigproc.py:160-202)."""

    def __init__(self, fname, extra_keys=None):
        self._fname = os.path.abspath(fname)
        with open(self._fname, "rb") as f:
            attrs, self._bytesize = read_sigproc_header(f, extra_keys)
        super().__init__(attrs)

    @property
    def fname(self):
        return self._fname

    @property
    def bytesize(self):
        """Bytes of the header; the payload starts there."""
        return self._bytesize

    @property
    def bytes_per_sample(self):
        return self["nchans"] * self["nbits"] // 8

    @property
    def nsamp(self):
        return (os.path.getsize(self.fname) - self.bytesize) // self.bytes_per_sample

    @property
    def tobs(self):
        return self.nsamp * self["tsamp"]

    @property
    def skycoord(self):
        """astropy SkyCoord of the source (requires astropy)."""
        import astropy.units as uu
        from astropy.coordinates import SkyCoord
        return SkyCoord(parse_float_coord(self["src_raj"]), parse_float_coord(self["src_dej"]),
                        unit=(uu.hour, uu.degree), frame="icrs")
