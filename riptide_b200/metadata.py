"""Metadata of an observation carried by TimeSeries and Periodogram (metadata.py of the
reference): a dict with the reserved keys source_name, skycoord, dm, mjd, tobs and fname
(None when unknown), built from PRESTO .inf or SIGPROC headers."""
import json
import os

from .reading import PrestoInf, SigprocHeader

RESERVED = ("source_name", "skycoord", "dm", "mjd", "tobs", "fname")


def _skycoord(header):
    try:
        return header.skycoord
    except ImportError:  # astropy is optional here
        return None


def _validate(items):
    """The checks of the reference's schema (metadata.py:11-21)."""
    for key, val in items.items():
        if not isinstance(key, str):
            raise ValueError(f"metadata key {key!r} is not a str")
        if val is None:
            continue
        if key in ("source_name", "fname") and not isinstance(val, str):
            raise ValueError(f"metadata {key!r} must be a str")
        elif key in ("dm", "mjd") and not (isinstance(val, float) and val >= 0):
            raise ValueError(f"metadata {key!r} must be a float >= 0")
        elif key == "tobs" and not (isinstance(val, float) and val > 0):
            raise ValueError("metadata 'tobs' must be a float > 0")
        elif key not in RESERVED:
            json.dumps(val)


class Metadata(dict):
    """dict of observation attributes; reserved keys default to None (metadata.py:24-50)."""

    def __init__(self, items=None):
        items = dict(items or {})
        _validate(items)
        super().__init__(items)
        for k in RESERVED:
            self.setdefault(k, None)

    @classmethod
    def from_presto_inf(cls, inf):
        """From a PRESTO .inf file or PrestoInf (metadata.py:53-71)."""
        if isinstance(inf, str):
            inf = PrestoInf(inf)
        attrs = dict(inf)
        attrs["skycoord"] = _skycoord(inf)
        attrs["fname"] = os.path.realpath(inf.fname)
        attrs["tobs"] = attrs["tsamp"] * attrs["nsamp"]
        return cls(attrs)

    @classmethod
    def from_sigproc(cls, sh, extra_keys=None):
        """From a SIGPROC file or SigprocHeader (metadata.py:73-113). ValueError for
        multi-channel data, for other than 8 or 32 bits per sample, and for 8-bit data whose
        header does not say whether the samples are signed."""
        if isinstance(sh, str):
            sh = SigprocHeader(sh, extra_keys=extra_keys)
        if sh["nchans"] > 1:
            raise ValueError(f"File {sh.fname!r} contains multi-channel data (nchans = "
                             f"{sh['nchans']}), instead of a dedispersed time series")
        nbits = sh["nbits"]
        if nbits not in (8, 32):
            raise ValueError(f"Only 8-bit and 32-bit SIGPROC data are supported. File "
                             f"{sh.fname!r} contains {nbits}-bit data")
        if nbits == 8 and "signed" not in sh:
            raise ValueError("SIGPROC Header says this is 8-bit data, but does not specify its "
                             "signedness via the 'signed' key")
        attrs = dict(sh)
        attrs["dm"] = attrs.get("refdm", None)
        attrs["skycoord"] = _skycoord(sh)
        attrs["source_name"] = attrs.get("source_name", None)
        attrs["mjd"] = attrs.get("tstart", None)
        attrs["fname"] = os.path.realpath(sh.fname)
        attrs["tobs"] = sh.tobs
        return cls(attrs)

    def to_dict(self):
        return dict(self)

    @classmethod
    def from_dict(cls, items):
        return cls(items)
