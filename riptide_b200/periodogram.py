"""Periodogram container (periodogram.py:9-64 of the reference; plotting is not included)."""


class Periodogram(object):
    """Raw output of the FFA search of one time series.

    widths : trial pulse widths (phase bins); periods : trial periods (s);
    foldbins : phase bins used for each trial period; snrs : (num_periods, num_widths) S/N.
    """

    def __init__(self, widths, periods, foldbins, snrs, metadata=None):
        self.widths = widths
        self.periods = periods
        self.foldbins = foldbins
        self.snrs = snrs
        self.metadata = metadata if metadata is not None else {}

    @property
    def freqs(self):
        """Trial frequencies in Hz, in decreasing order."""
        return 1.0 / self.periods

    @property
    def tobs(self):
        """Length in seconds of the searched series."""
        return self.metadata["tobs"]

    def to_dict(self):
        return {"widths": self.widths, "periods": self.periods, "foldbins": self.foldbins,
                "snrs": self.snrs, "metadata": self.metadata}

    @classmethod
    def from_dict(cls, items):
        return cls(items["widths"], items["periods"], items["foldbins"], items["snrs"],
                   metadata=items["metadata"])
