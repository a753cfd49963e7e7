"""The search stage of riptide's pipeline (pipeline/worker_pool.py:10-68 of the reference) as
batched GPU work.

The reference maps ``process_fname`` over a process pool. Each process loads one DM trial,
dereddens and normalises it once (worker_pool.py:53-59), and then runs ffa_search and
find_peaks for every search range of the configuration (:61-67).

Here a list of files is one batch:
  1. their payloads are loaded into one device tensor (reading.load_series_batch);
  2. the first range's plan dereddens, normalises and searches every trial in one launch,
     and leaves the normalised series on the device;
  3. every further range searches those series (deredden=False, already_normalised=True);
  4. find_peaks runs batched over all trials of a range (peaks.find_peaks_batched).
Trials are searched in chunks of `chunk_trials`, grouped by sampling time (a plan has one).
The next chunk's files are read and copied to the device on a side stream by a loader thread
while the current chunk is searched, and a finder thread runs find_peaks on the previous
chunk's periodograms (on a stream of its own) while the next one is searched. Peaks come back
in the reference's order: by file, then by range, then by decreasing S/N.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import libcpp
from .batched import BatchedSearch
from .peaks import find_peaks_batched
from .reading import describe, load_series_batch

_SEARCH_KEYS = ("period_min", "period_max", "bins_min", "bins_max", "ducy_max", "wtsp")


def _search_kwargs(conf):
    """BatchedSearch arguments of a range's 'ffa_search' section (fpmin is accepted and
    ignored, as ffa_search ignores it, search.py:15)."""
    kw = dict(conf["ffa_search"])
    kw.pop("fpmin", None)
    unknown = set(kw) - set(_SEARCH_KEYS)
    if unknown:
        raise ValueError(f"unknown ffa_search parameters {sorted(unknown)}")
    return kw


class WorkerPool(object):
    """Search many DM trial files over every configured search range.

    deredden_params : dict with rmed_width (s) and rmed_minpts
    range_confs : list of dicts with 'ffa_search' and 'find_peaks' sections (the 'ranges'
        section of the pipeline configuration)
    processes : accepted for compatibility; the GPU batch replaces the process pool
    fmt : "presto" (.inf files) or "sigproc" (.tim files)
    chunk_trials : trials searched per launch
    tuning : engine tile choices passed to every plan (riptide_b200.tuning)
    """

    TIMESERIES_FORMATS = ("sigproc", "presto")

    def __init__(self, deredden_params, range_confs, processes=1, fmt="presto",
                 chunk_trials=64, tuning=None):
        if fmt not in self.TIMESERIES_FORMATS:
            raise ValueError(f"format must be one of {self.TIMESERIES_FORMATS}")
        if not range_confs:
            raise ValueError("at least one search range is required")
        self.deredden_params = dict(deredden_params)
        self.range_confs = list(range_confs)
        self.processes = int(processes)
        self.fmt = fmt
        self.chunk_trials = max(1, int(chunk_trials))
        self.tuning = tuning
        self._search_kw = [_search_kwargs(c) for c in self.range_confs]
        self._plans = {}

    def _plan(self, irange, lengths, tsamp):
        key = (irange, tuple(int(x) for x in lengths), float(tsamp))
        bs = self._plans.get(key)
        if bs is None:
            first = irange == 0
            bs = BatchedSearch(lengths, tsamp, deredden=first, already_normalised=not first,
                               rmed_width=float(self.deredden_params["rmed_width"]),
                               rmed_minpts=int(self.deredden_params["rmed_minpts"]),
                               tuning=self.tuning, **self._search_kw[irange])
            self._plans[key] = bs
        return bs

    def process_fname_list(self, fnames):
        """Peaks of every file and range, flattened in the reference's order."""
        torch = libcpp._t()
        files = describe(list(fnames), self.fmt)
        per_file = [[] for _ in files]
        groups = {}
        for i, f in enumerate(files):
            groups.setdefault(f.tsamp, []).append(i)
        chunks = [(tsamp, idx[a:a + self.chunk_trials]) for tsamp, idx in groups.items()
                  for a in range(0, len(idx), self.chunk_trials)]
        if not chunks:
            return []
        main = torch.cuda.current_stream()
        side = torch.cuda.Stream()
        dev = torch.cuda.current_device()  # the helper threads work on the caller's device

        def load(chunk):
            with torch.cuda.device(dev), torch.cuda.stream(side):
                x, lengths = load_series_batch([files[i] for i in chunk[1]])
                ev = torch.cuda.Event()
                ev.record(side)
            return x, lengths, ev

        finder_stream = torch.cuda.Stream()
        pending = []
        with ThreadPoolExecutor(1) as loader, ThreadPoolExecutor(1) as finder:
            nxt = loader.submit(load, chunks[0])
            for k, (tsamp, idx) in enumerate(chunks):
                x, lengths, ev = nxt.result()
                if k + 1 < len(chunks):
                    nxt = loader.submit(load, chunks[k + 1])
                main.wait_event(ev)
                x.record_stream(main)
                chunk_files = [files[i] for i in idx]
                searched = self._search_chunk(x, lengths, tsamp)
                done = torch.cuda.Event()
                done.record(main)
                pending.append((idx, finder.submit(self._peaks_chunk, searched, done, dev,
                                                   finder_stream, lengths, chunk_files, tsamp)))
            for idx, fut in pending:
                for i, peaks in zip(idx, fut.result()):
                    per_file[i] = peaks
        return [p for plist in per_file for p in plist]

    def process_fname(self, fname):
        """Peaks of one file over every range (worker_pool.py:47-68)."""
        return self.process_fname_list([fname])

    def _search_chunk(self, data, lengths, tsamp):
        """Every range's periodograms of one chunk, in output tensors of this chunk's own."""
        torch = libcpp._t()
        z = torch.empty_like(data)
        searched = []
        for r in range(len(self.range_confs)):
            bs = self._plan(r, lengths, tsamp)
            outs = bs.allocate_outputs(data.device)
            if r == 0:
                bs.run(data, outs, normalised=z)
            else:
                bs.run(z, outs)
            searched.append((bs.row_offsets, bs.widths, outs))
        return searched

    def _peaks_chunk(self, searched, done, dev, stream, lengths, files, tsamp):
        """find_peaks of every range of one chunk, on device `dev` and `stream`, after the
        event `done`."""
        torch = libcpp._t()
        tobs = lengths.astype(np.float64) * tsamp
        dms = [f.metadata.get("dm") for f in files]
        out = [[] for _ in files]
        with torch.cuda.device(dev), torch.cuda.stream(stream):
            stream.wait_event(done)
            for (rows, widths, outs), conf in zip(searched, self.range_confs):
                for t in outs:
                    t.record_stream(stream)
                res = find_peaks_batched(outs[0], outs[1], outs[2], rows, tobs, widths,
                                         dms=dms, **dict(conf.get("find_peaks") or {}))
                for t, (peaks, _) in enumerate(res):
                    out[t].append(peaks)
        return [[p for plist in ranges for p in plist] for ranges in out]

    def close(self):
        for bs in self._plans.values():
            bs.close()
        self._plans = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
