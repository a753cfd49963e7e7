"""Readers of dedispersed time series files (reading/ of the reference): PRESTO .inf/.dat and
SIGPROC .tim headers, and a batched loader of their payloads into device memory."""
from .presto import PrestoInf, inf2dict
from .sigproc import SigprocHeader, read_sigproc_header, sigproc_keydb
from .ingest import SeriesFile, describe, load_series_batch, read_payload

__all__ = ["PrestoInf", "inf2dict", "SigprocHeader", "read_sigproc_header", "sigproc_keydb",
           "SeriesFile", "describe", "load_series_batch", "read_payload"]
