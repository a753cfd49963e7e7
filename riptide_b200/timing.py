"""`@timing` decorator: logs wall time at DEBUG on the `riptide.timing` logger
(timing.py:6-17 of the reference)."""
import logging
import time
from functools import wraps


def timing(func):
    @wraps(func)
    def wrapped(*args, **kwargs):
        log = logging.getLogger("riptide.timing")
        t0 = time.time()
        output = func(*args, **kwargs)
        log.debug("{!r} runtime: {:.2f} ms".format(func.__name__, (time.time() - t0) * 1000.0))
        return output

    return wrapped
