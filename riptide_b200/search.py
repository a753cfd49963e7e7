"""ffa_search (search.py:11-93 of the reference) on the GPU."""
import numpy as np

from . import libcpp
from .batched import BatchedSearch
from .ffautils import generate_width_trials
from .periodogram import Periodogram
from .time_series import TimeSeries
from .timing import timing


@timing
def ffa_search(tseries, period_min=1.0, period_max=30.0, fpmin=8, bins_min=240, bins_max=260,
               ducy_max=0.20, wtsp=1.5, deredden=True, rmed_width=4.0, rmed_minpts=101,
               already_normalised=False):
    """FFA search of one TimeSeries: deredden, normalise, periodogram. Returns
    (searched TimeSeries, Periodogram). `fpmin` is accepted and ignored, as in the
    reference (search.py:15 vs :82-93)."""
    del fpmin
    widths = generate_width_trials(bins_min, ducy_max=ducy_max, wtsp=wtsp)
    if not deredden and already_normalised:
        periods, foldbins, snrs = libcpp.periodogram(
            tseries.data, tseries.tsamp, widths, period_min, period_max, bins_min, bins_max)
        return tseries, Periodogram(widths, periods, foldbins, snrs, metadata=tseries.metadata)
    bs = BatchedSearch([tseries.nsamp], tseries.tsamp, period_min=period_min,
                       period_max=period_max, bins_min=bins_min, bins_max=bins_max,
                       deredden=deredden, rmed_width=rmed_width, rmed_minpts=rmed_minpts,
                       already_normalised=already_normalised, widths=widths)
    try:
        (pg,), (z,) = bs.search([tseries.data], return_normalised=True)
    finally:
        bs.close()
    ts = TimeSeries(np.array(z, copy=True), tseries.tsamp, metadata=tseries.metadata)
    pg.metadata = ts.metadata
    return ts, pg
