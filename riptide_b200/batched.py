"""Batched FFA search: ffa_search over many DM trials of uneven length in one GPU pass.

A ``BatchedSearch`` owns a plan (C ABI rt_search_plan_*): every (trial, octave cycle, bins)
transform, its stage split and the work list of the persistent kernel. Plans depend only on
the trial lengths and the search parameters, so one plan serves every batch of that shape.
"""
import ctypes

import numpy as np

from . import _lib, libcpp
from .ffautils import generate_width_trials
from .periodogram import Periodogram


class BatchedSearch(object):
    """Search many series with the parameters of ffa_search (search.py:11-93)."""

    def __init__(self, lengths, tsamp, period_min=1.0, period_max=30.0, bins_min=240,
                 bins_max=260, ducy_max=0.20, wtsp=1.5, deredden=True, rmed_width=4.0,
                 rmed_minpts=101, already_normalised=False, widths=None, tuning=None,
                 rules=None):
        """`tuning`: engine tile choices, a dict with any of rows_fraction, snr_threads,
        lag_items, rows_fraction_deep (riptide_b200.tuning.autotune picks them). `rules`:
        per-(rows, bins) tile choices, a list of dicts with rows_min, rows_max, bins_min,
        bins_max and any of rows_fraction, snr_threads, max_levels
        (riptide_b200.tuning.autotune_rules picks them); the first rule holding a
        transform's (rows, bins) applies to it. Results do not depend on either."""
        self.lengths = np.ascontiguousarray(np.asarray(lengths, dtype=np.uint64).ravel())
        self.tsamp = float(tsamp)
        self.widths = (np.asarray(widths) if widths is not None
                       else generate_width_trials(bins_min, ducy_max=ducy_max, wtsp=wtsp))
        cfg = _lib.SearchConfig(
            tsamp=self.tsamp, period_min=float(period_min), period_max=float(period_max),
            bins_min=int(bins_min), bins_max=int(bins_max), deredden=int(bool(deredden)),
            rmed_width=float(rmed_width), rmed_minpts=int(rmed_minpts),
            already_normalised=int(bool(already_normalised)))
        self._cfg = cfg
        w, wp = _lib.u64_array(self.widths)
        lp = self.lengths.ctypes.data_as(_lib._u64p)
        h = ctypes.c_void_p()
        self.tuning = dict(tuning) if tuning else None
        self.rules = [dict(r) for r in rules] if rules else None
        if rules:
            tn = _lib.SearchTuning(rows_fraction=float((tuning or {}).get("rows_fraction", 0.0)),
                                   snr_threads=int((tuning or {}).get("snr_threads", 0)),
                                   lag_items=int((tuning or {}).get("lag_items", 0)),
                                   rows_fraction_deep=float((tuning or {}).get("rows_fraction_deep", 0.0)))
            arr = (_lib.TileRule * len(rules))()
            for i, r in enumerate(rules):
                arr[i] = _lib.TileRule(int(r["rows_min"]), int(r["rows_max"]), int(r["bins_min"]),
                                       int(r["bins_max"]), float(r.get("rows_fraction", 0.0)),
                                       int(r.get("snr_threads", 0)), int(r.get("max_levels", 0)))
            _lib.check(_lib.load().rt_search_plan_create_rules(
                lp, self.lengths.size, ctypes.byref(cfg), wp, w.size, ctypes.byref(tn), arr,
                len(rules), ctypes.byref(h)))
        elif tuning:
            tn = _lib.SearchTuning(rows_fraction=float(tuning.get("rows_fraction", 0.0)),
                                   snr_threads=int(tuning.get("snr_threads", 0)),
                                   lag_items=int(tuning.get("lag_items", 0)),
                                   rows_fraction_deep=float(tuning.get("rows_fraction_deep", 0.0)))
            _lib.check(_lib.load().rt_search_plan_create_tuned(
                lp, self.lengths.size, ctypes.byref(cfg), wp, w.size, ctypes.byref(tn),
                ctypes.byref(h)))
        else:
            _lib.check(_lib.load().rt_search_plan_create(lp, self.lengths.size, ctypes.byref(cfg),
                                                         wp, w.size, ctypes.byref(h)))
        self._plan = h
        rows = np.zeros(self.lengths.size + 1, dtype=np.uint64)
        _lib.check(_lib.load().rt_search_plan_rows(h, rows.ctypes.data_as(_lib._u64p)))
        self.row_offsets = rows.astype(np.int64)
        st = _lib.PlanStats()
        _lib.check(_lib.load().rt_search_plan_stats(h, ctypes.byref(st)))
        self.stats = {k: int(getattr(st, k)) for k, _ in _lib.PlanStats._fields_}
        self.sample_offsets = np.concatenate([[0], np.cumsum(self.lengths.astype(np.int64))])
        self._out = None

    # ------------------------------------------------------------------
    @property
    def num_trials(self):
        return int(self.lengths.size)

    @property
    def total_rows(self):
        return int(self.row_offsets[-1])

    def allocate_outputs(self, device="cuda"):
        """Device tensors (periods f64[L], foldbins i32[L], snrs f32[L, nw]) of the batch."""
        torch = libcpp._t()
        L, nw = self.total_rows, self.widths.size
        return (torch.empty((L,), dtype=torch.float64, device=device),
                torch.empty((L,), dtype=torch.int32, device=device),
                torch.empty((L, nw), dtype=torch.float32, device=device))

    def run(self, data, outputs=None, normalised=None, check=True):
        """Search `data` (CUDA float32 tensor, all series packed back to back). Returns the
        packed device outputs (periods, foldbins, snrs). Kernels run on the current torch
        stream; `check` synchronises it and raises on a device-side failure."""
        torch = libcpp._t()
        if not (libcpp._is_cuda_tensor(data) and data.dtype == torch.float32 and data.is_contiguous()):
            raise ValueError("data must be a contiguous float32 CUDA tensor")
        if data.numel() != int(self.sample_offsets[-1]):
            raise ValueError("data does not hold the planned number of samples")
        if outputs is None:
            if self._out is None:
                self._out = self.allocate_outputs(data.device)
            outputs = self._out
        periods, foldbins, snrs = outputs
        nptr = ctypes.c_void_p(normalised.data_ptr()) if normalised is not None else None
        st = libcpp._stream()
        _lib.check(_lib.load().rt_search_run(self._plan, ctypes.c_void_p(data.data_ptr()), nptr,
                                             ctypes.c_void_p(periods.data_ptr()),
                                             ctypes.c_void_p(foldbins.data_ptr()),
                                             ctypes.c_void_p(snrs.data_ptr()), st))
        if check:
            _lib.check(_lib.load().rt_search_check(self._plan, st))
        return outputs

    def search(self, series, return_normalised=False):
        """End-to-end search of host series (list of 1D arrays, or one packed array). Returns
        a list of Periodogram (host numpy arrays), and the searched series if asked."""
        torch = libcpp._t()
        if isinstance(series, np.ndarray) and series.ndim == 1 and series.size == self.sample_offsets[-1]:
            packed = np.ascontiguousarray(series, dtype=np.float32)
        else:
            packed = np.concatenate([np.asarray(s, dtype=np.float32).ravel() for s in series])
        if packed.size != self.sample_offsets[-1]:
            raise ValueError("series lengths do not match the plan")
        host = torch.from_numpy(packed).pin_memory()
        dev = host.to("cuda", non_blocking=True)
        norm = torch.empty_like(dev) if return_normalised else None
        periods, foldbins, snrs = self.run(dev, normalised=norm)
        p = periods.cpu().numpy()
        fb = foldbins.cpu().numpy().view(np.uint32)
        s = snrs.cpu().numpy()
        out = []
        for i in range(self.num_trials):
            a, b = self.row_offsets[i], self.row_offsets[i + 1]
            md = {"tobs": float(self.lengths[i]) * self.tsamp}
            out.append(Periodogram(self.widths, p[a:b], fb[a:b], s[a:b], metadata=md))
        if return_normalised:
            z = norm.cpu().numpy()
            zs = [z[self.sample_offsets[i]:self.sample_offsets[i + 1]] for i in range(self.num_trials)]
            return out, zs
        return out

    def enable_graph(self, enable=True):
        """Replay each run as one CUDA graph (captured again when the tensors change)."""
        _lib.check(_lib.load().rt_search_set_graph(self._plan, int(bool(enable))))

    @property
    def graph_captures(self):
        n = ctypes.c_int(0)
        _lib.check(_lib.load().rt_search_graph_captures(self._plan, ctypes.byref(n)))
        return int(n.value)

    def enable_timing(self, enable=True):
        """Record CUDA events around the stages of every run (see last_timing)."""
        _lib.check(_lib.load().rt_search_set_timing(self._plan, int(bool(enable))))

    def last_timing(self):
        """(ms deredden+stats, ms downsample, ms FFA+S/N kernel, kernel launches) of the last
        run with timing enabled."""
        ms = (ctypes.c_float * 3)()
        n = ctypes.c_int(0)
        _lib.check(_lib.load().rt_search_last_timing(self._plan, ms, ctypes.byref(n)))
        return float(ms[0]), float(ms[1]), float(ms[2]), int(n.value)

    def enable_profiling(self, enable=True):
        """Accumulate per-phase SM cycles inside the persistent kernel (see phase_cycles)."""
        _lib.check(_lib.load().rt_search_set_profiling(self._plan, int(bool(enable))))

    def phase_cycles(self, reset=True):
        """{phase: summed SM cycles} of the runs since the last reset."""
        c = np.zeros(16, dtype=np.uint64)
        _lib.check(_lib.load().rt_search_phase_cycles(self._plan, c.ctypes.data_as(_lib._u64p),
                                                      int(bool(reset))))
        names = ["fetch", "wait", "tree", "levels", "snr", "store", "decode", "sched_wait",
                 "blocked_slot", "blocked_stage", "claimed", "empty_polls", "level_values",
                 "levels_run", "root_rows", "later_stage_items"]
        return {n: int(c[i]) for i, n in enumerate(names)}

    def set_wait_limit(self, polls):
        """Bound of the waits inside the search kernel, in polls (default 20,000,000). A wait
        that runs out ends the run with RT_ETIMEOUT instead of hanging."""
        _lib.check(_lib.load().rt_search_set_wait_limit(self._plan, int(polls)))

    def inject_fault(self, kind, arg=0):
        """Host-side fault injection for tests of the error paths (no GPU fault is raised):
        "stage_wait" makes later-stage work items wait on a count that is never reached (the
        run ends with RT_ETIMEOUT after the wait limit); "alloc" releases the plan's device
        buffers and makes allocation number `arg` of the next run fail (RT_ENOMEM); None
        clears both."""
        kinds = {None: _lib.RT_FAULT_NONE, "stage_wait": _lib.RT_FAULT_STAGE_WAIT,
                 "alloc": _lib.RT_FAULT_ALLOC}
        _lib.check(_lib.load().rt_search_inject_fault(self._plan, kinds[kind], int(arg)))

    def close(self):
        if getattr(self, "_plan", None):
            _lib.load().rt_search_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ffa_search_batched(series, tsamp, **kwargs):
    """ffa_search over a list of series sharing tsamp and search parameters. Returns a list
    of Periodogram objects (host arrays)."""
    lengths = [np.asarray(s).size for s in series]
    bs = BatchedSearch(lengths, tsamp, **kwargs)
    try:
        return bs.search(series)
    finally:
        bs.close()


def _host_ptr(a, dtypes, n, name):
    """Address of a contiguous host buffer (numpy array or CPU torch tensor) of n values of
    one of `dtypes` (numpy dtype names)."""
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
        if a.is_cuda:
            raise ValueError(f"{name} must be in host memory")
        ok = a.is_contiguous() and a.numel() == n and str(a.dtype).replace("torch.", "") in dtypes
        ptr = a.data_ptr()
    else:
        ok = (isinstance(a, np.ndarray) and a.dtype.name in dtypes and a.flags.c_contiguous
              and a.size == n)
        ptr = a.ctypes.data if ok else 0
    if not ok:
        raise ValueError(f"{name} must be a contiguous host buffer of {n} {dtypes[0]}")
    return ptr


class SearchPipeline(object):
    """Batched search of series held in host memory (C ABI rt_search_pipeline_*).

    The trials are cut into chunks of ``chunk_trials`` consecutive trials (a quarter of that
    first and last, when there are enough trials); the copy of chunk i+1 to the GPU and the
    copy of chunk i-1's periodograms back to the host overlap the search of chunk i. Host buffers from ``allocate_host`` are page-locked, which the
    overlap needs. Same outputs as ``BatchedSearch`` (every trial is searched independently).
    """

    def __init__(self, lengths, tsamp, chunk_trials=16, period_min=1.0, period_max=30.0,
                 bins_min=240, bins_max=260, ducy_max=0.20, wtsp=1.5, deredden=True,
                 rmed_width=4.0, rmed_minpts=101, already_normalised=False, widths=None):
        self.lengths = np.ascontiguousarray(np.asarray(lengths, dtype=np.uint64).ravel())
        self.tsamp = float(tsamp)
        self.widths = (np.asarray(widths) if widths is not None
                       else generate_width_trials(bins_min, ducy_max=ducy_max, wtsp=wtsp))
        cfg = _lib.SearchConfig(
            tsamp=self.tsamp, period_min=float(period_min), period_max=float(period_max),
            bins_min=int(bins_min), bins_max=int(bins_max), deredden=int(bool(deredden)),
            rmed_width=float(rmed_width), rmed_minpts=int(rmed_minpts),
            already_normalised=int(bool(already_normalised)))
        w, wp = _lib.u64_array(self.widths)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().rt_search_pipeline_create(
            self.lengths.ctypes.data_as(_lib._u64p), self.lengths.size, ctypes.byref(cfg), wp,
            w.size, int(chunk_trials), ctypes.byref(h)))
        self._pipe = h
        rows = np.zeros(self.lengths.size + 1, dtype=np.uint64)
        _lib.check(_lib.load().rt_search_pipeline_rows(h, rows.ctypes.data_as(_lib._u64p)))
        self.row_offsets = rows.astype(np.int64)
        n = ctypes.c_size_t(0)
        _lib.check(_lib.load().rt_search_pipeline_chunks(h, ctypes.byref(n)))
        self.num_chunks = int(n.value)
        self.sample_offsets = np.concatenate([[0], np.cumsum(self.lengths.astype(np.int64))])

    @property
    def num_trials(self):
        return int(self.lengths.size)

    @property
    def total_rows(self):
        return int(self.row_offsets[-1])

    def allocate_host(self):
        """Page-locked host buffers: (input f32[samples], periods f64[L], foldbins i32[L],
        snrs f32[L, nw]) as CPU torch tensors."""
        torch = libcpp._t()
        L, nw = self.total_rows, self.widths.size
        return (torch.empty((int(self.sample_offsets[-1]),), dtype=torch.float32, pin_memory=True),
                (torch.empty((L,), dtype=torch.float64, pin_memory=True),
                 torch.empty((L,), dtype=torch.int32, pin_memory=True),
                 torch.empty((L, nw), dtype=torch.float32, pin_memory=True)))

    def run(self, host_data, host_outputs, check=True):
        """Search host_data (all series packed back to back) into host_outputs (periods,
        foldbins, snrs). Enqueued after the current torch stream's work; `check` waits for
        the results and raises on a device-side failure."""
        L, nw = self.total_rows, int(self.widths.size)
        periods, foldbins, snrs = host_outputs
        pd = _host_ptr(host_data, ("float32",), int(self.sample_offsets[-1]), "host_data")
        pp = _host_ptr(periods, ("float64",), L, "periods")
        pf = _host_ptr(foldbins, ("int32", "uint32"), L, "foldbins")
        ps = _host_ptr(snrs, ("float32",), L * nw, "snrs")
        st = libcpp._stream()
        _lib.check(_lib.load().rt_search_pipeline_run(self._pipe, ctypes.c_void_p(pd),
                                                      ctypes.c_void_p(pp), ctypes.c_void_p(pf),
                                                      ctypes.c_void_p(ps), st))
        if check:
            self.check()
        return host_outputs

    def check(self):
        """Wait for the last run and raise on a device-side failure."""
        _lib.check(_lib.load().rt_search_pipeline_check(self._pipe, libcpp._stream()))

    def search(self, series):
        """Search host series (list of 1D arrays, or one packed array); a list of
        Periodogram."""
        host_in, outs = self.allocate_host()
        x = host_in.numpy()
        if isinstance(series, np.ndarray) and series.ndim == 1:
            if series.size != x.size:
                raise ValueError("series lengths do not match the plan")
            x[:] = series
        else:
            if len(series) != self.num_trials:
                raise ValueError("series lengths do not match the plan")
            for i, s in enumerate(series):
                s = np.asarray(s, dtype=np.float32).ravel()
                if s.size != self.lengths[i]:
                    raise ValueError("series lengths do not match the plan")
                x[self.sample_offsets[i]:self.sample_offsets[i + 1]] = s
        self.run(host_in, outs)
        p, fb, s = outs[0].numpy(), outs[1].numpy().view(np.uint32), outs[2].numpy()
        out = []
        for i in range(self.num_trials):
            a, b = self.row_offsets[i], self.row_offsets[i + 1]
            md = {"tobs": float(self.lengths[i]) * self.tsamp}
            out.append(Periodogram(self.widths, p[a:b].copy(), fb[a:b].copy(), s[a:b].copy(),
                                   metadata=md))
        return out

    def close(self):
        if getattr(self, "_pipe", None):
            _lib.load().rt_search_pipeline_destroy(self._pipe)
            self._pipe = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
