"""PRESTO .inf metadata files (reading/presto.py of the reference).

An .inf file is a sequence of "description = value" lines, the '=' at column 40; the first
twelve lines are common to all observations (file base name, telescope, ..., number of
samples, sampling time, data breaks), followed by the on/off sample pairs when the data have
breaks, then the EM band and a block that depends on it (radio: beam, DM, frequencies,
channels, analyst; X-ray / gamma: field of view, energies, analyst). The float32 samples are in
the .dat file of the same base name.
"""
import os

SEP_COLUMN = 40
FAKE_TELESCOPE = "None (Artificial Data Set)"

# (key, type) of the twelve leading lines (presto.py:72-85)
_COMMON = (("basename", str), ("telescope", str), ("instrument", str), ("source_name", str),
           ("raj", str), ("decj", str), ("observer", str), ("mjd", float),
           ("barycentered", "bool"), ("nsamp", int), ("tsamp", float), ("breaks", "bool"))
# blocks that depend on the EM band (presto.py:101-117)
_BAND = {
    "Radio": (("fov_arcsec", float), ("dm", float), ("fbot", float), ("bandwidth", float),
              ("nchan", int), ("cbw", float), ("analyst", str)),
    "X-ray": (("fov_arcsec", float), ("central_energy_kev", float),
              ("energy_bandpass_kev", float), ("analyst", str)),
}
_BAND["Gamma"] = _BAND["X-ray"]


def _value(line, kind):
    """The value of one .inf line, converted to `kind` (str, int, float, "bool" for a 0/1
    flag, "pair" for an "a , b" pair of ints). ValueError when the line has no '=' at
    column 40 or the value does not convert."""
    if len(line) <= SEP_COLUMN or line[SEP_COLUMN] != "=":
        raise ValueError(f"Expected '=' character at column {SEP_COLUMN}")
    text = line[SEP_COLUMN + 1:].strip()
    if kind == "bool":
        return int(text) != 0
    if kind == "pair":
        a, b = text.split(",")
        return int(a), int(b)
    return kind(text)


def inf2dict(text):
    """Parse the text of an .inf file into a dict (presto.py:60-121)."""
    lines = text.strip("\n").splitlines()
    items = {}
    for i, (key, kind) in enumerate(_COMMON):
        items[key] = _value(lines[i], kind)
        if key == "telescope" and items[key] == FAKE_TELESCOPE:
            raise ValueError("Reading data generated with PRESTO's makedata is not supported")
    rest = lines[len(_COMMON):]
    pairs = []
    if items["breaks"]:
        for line in rest:
            try:
                pairs.append(_value(line, "pair"))
            except Exception:
                break
    items["onoff_pairs"] = pairs
    rest = rest[len(pairs):]
    band = _value(rest[0], str)
    items["em_band"] = band
    if band not in _BAND:
        raise ValueError(f"EM Band {band!r} not supported")
    for i, (key, kind) in enumerate(_BAND[band], start=1):
        items[key] = _value(rest[i], kind)
    return items


class PrestoInf(dict):
    """The items of a PRESTO .inf file (presto.py:124-152)."""

    def __init__(self, fname):
        self._fname = os.path.realpath(fname)
        with open(fname, "r") as f:
            super().__init__(inf2dict(f.read()))

    @property
    def fname(self):
        """Absolute path of the .inf file."""
        return self._fname

    @property
    def data_fname(self):
        """Path of the associated .dat file."""
        return self.fname.rsplit(".", maxsplit=1)[0] + ".dat"

    @property
    def skycoord(self):
        """astropy SkyCoord of the source (requires astropy)."""
        import astropy.units as uu
        from astropy.coordinates import SkyCoord
        return SkyCoord(self["raj"], self["decj"], unit=(uu.hour, uu.degree))

    def load_data(self):
        """The .dat samples as a float32 numpy array (read by the library's parallel reader)."""
        from .ingest import read_payload
        return read_payload(self.data_fname, 0, None, "f32")
