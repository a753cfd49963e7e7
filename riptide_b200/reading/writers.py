"""Writers of the two time series file formats the readers take: a SIGPROC dedispersed time
series (header + samples) and a PRESTO .inf / .dat pair. They write the header layout the
readers parse (reading/sigproc.py, reading/presto.py), for test data and for exporting
dedispersed series."""
import struct

import numpy as np

from .presto import SEP_COLUMN
from .sigproc import HEADER_END, HEADER_START, sigproc_keydb


def _pack_str(s):
    b = s.encode()
    return struct.pack("i", len(b)) + b


def write_sigproc(fname, data, header, extra_keys=None):
    """Write `data` with the SIGPROC `header` dict (values stored by the types of
    sigproc_keydb, updated by `extra_keys`). The samples are written as float32 for nbits =
    32 and as int8 / uint8 by header['signed'] for nbits = 8 (no 'signed' key: uint8)."""
    keydb = dict(sigproc_keydb)
    if extra_keys:
        keydb.update(extra_keys)
    out = [_pack_str(HEADER_START)]
    for key, val in header.items():
        kind = keydb[key]
        out.append(_pack_str(key))
        if kind is str:
            out.append(_pack_str(val))
        elif kind is int:
            out.append(struct.pack("i", int(val)))
        elif kind is float:
            out.append(struct.pack("d", float(val)))
        elif kind is bool:
            out.append(struct.pack("B", int(bool(val))))
        else:
            raise ValueError(f"unsupported type {kind} for key {key!r}")
    out.append(_pack_str(HEADER_END))
    nbits = header.get("nbits", 32)
    if nbits == 8:
        dtype = np.int8 if header.get("signed", False) else np.uint8
    else:
        dtype = np.float32
    with open(fname, "wb") as f:
        f.write(b"".join(out))
        f.write(np.asarray(data).astype(dtype).tobytes())


_INF_COMMON = (
    ("Data file name without suffix", "basename"), ("Telescope used", "telescope"),
    ("Instrument used", "instrument"), ("Object being observed", "source_name"),
    ("J2000 Right Ascension (hh:mm:ss.ssss)", "raj"),
    ("J2000 Declination     (dd:mm:ss.ssss)", "decj"), ("Data observed by", "observer"),
    ("Epoch of observation (MJD)", "mjd"), ("Barycentered?           (1 yes, 0 no)", "barycentered"),
    ("Number of bins in the time series", "nsamp"),
    ("Width of each time series bin (sec)", "tsamp"),
    ("Any breaks in the data? (1 yes, 0 no)", "breaks"))
_INF_BAND = {
    "Radio": (("Beam diameter (arcsec)", "fov_arcsec"), ("Dispersion measure (cm-3 pc)", "dm"),
              ("Central freq of low channel (Mhz)", "fbot"), ("Total bandwidth (Mhz)", "bandwidth"),
              ("Number of channels", "nchan"), ("Channel bandwidth (Mhz)", "cbw"),
              ("Data analyzed by", "analyst")),
    "X-ray": (("Field-of-view diameter (arcsec)", "fov_arcsec"),
              ("Central energy (kev)", "central_energy_kev"),
              ("Energy bandpass (kev)", "energy_bandpass_kev"), ("Data analyzed by", "analyst")),
}
_INF_BAND["Gamma"] = _INF_BAND["X-ray"]


def _inf_line(label, value):
    return " " + label.ljust(SEP_COLUMN - 1) + "=  " + str(value)


def _inf_value(v):
    if isinstance(v, bool):
        return int(v)
    return v


def write_presto(basename, data, items):
    """Write basename.dat (float32 samples) and basename.inf from `items` (the keys
    PrestoInf returns; 'onoff_pairs' listed when items['breaks'])."""
    lines = [_inf_line(label, _inf_value(items[key])) for label, key in _INF_COMMON]
    if items.get("breaks"):
        for i, (a, b) in enumerate(items.get("onoff_pairs", []), start=1):
            lines.append(_inf_line(f"On/Off bin pair #{i:3d}", f"{a:<11d}, {b}"))
    band = items["em_band"]
    lines.append(_inf_line("Type of observation (EM band)", band))
    lines += [_inf_line(label, _inf_value(items[key])) for label, key in _INF_BAND[band]]
    lines += [" Any additional notes:", "    none", ""]
    with open(basename + ".inf", "w") as f:
        f.write("\n".join(lines))
    np.asarray(data, dtype=np.float32).tofile(basename + ".dat")
