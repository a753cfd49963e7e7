"""Autotuner of the engine's tile choices.

The persistent search kernel has choices that change its speed but not its results
(rt_search_tuning), made per transform from its rows (m) and bins (b):
  rows_fraction       rows per job, as a fraction of what shared memory holds at this b:
                      fewer rows make more, smaller jobs (less cone recomputation per job,
                      more per-job overhead);
  rows_fraction_deep  the same for the transforms of more than 8 jobs' worth of rows, the ones
                      cut into several stages;
  snr_threads         threads per profile in the S/N (8 or 16; 8 only for b <= 264): more
                      threads per profile finish a job's last, partial round sooner;
  lag_items           work items between two stages of a multi-stage transform: a longer lag
                      leaves the previous stage more time to finish (fewer waits), a shorter
                      one keeps its output in L2.
`autotune` times the engine on a sample of the workload (synthetic noise of the same
lengths, the same search parameters): first a grid of rows_fraction x snr_threads x
lag_items, then rows_fraction_deep around the best of the grid. It returns the fastest,
caching the answer per (search parameters, lengths) for the process and, optionally, in a
JSON file.
"""
import json
import os

import numpy as np

DEFAULT = {"rows_fraction": 1.0, "snr_threads": 0, "lag_items": 0, "rows_fraction_deep": 0.0}
DEEP_FRACTIONS = (0.9, 0.8, 0.7)


def candidates(bins_max):
    """The candidate grid: rows per job x S/N threads x stage lag."""
    out = []
    tprs = (0, 16) if bins_max <= 264 else (0,)
    for rf in (1.0, 0.9, 0.8):
        for tpr in tprs:
            for lag in (0, 320, 1280):
                out.append({"rows_fraction": rf, "snr_threads": tpr, "lag_items": lag,
                            "rows_fraction_deep": 0.0})
    return out


_CACHE = {}


def _key(lengths, tsamp, search_kw):
    L = np.asarray(lengths, dtype=np.int64)
    return json.dumps({"tsamp": float(tsamp), "n": int(L.size),
                       "len": [int(L.min()), int(L.max())],
                       "search": {k: (float(v) if isinstance(v, float) else v)
                                  for k, v in sorted(search_kw.items())}}, sort_keys=True)


def time_search(lengths, tsamp, tuning, data, repeats=3, **search_kw):
    """Median CUDA-event time (ms) of one engine run with `tuning` on `data`."""
    import torch

    from .batched import BatchedSearch

    bs = BatchedSearch(lengths, tsamp, tuning=tuning, **search_kw)
    try:
        outs = bs.allocate_outputs()
        bs.run(data, outs)  # allocations and first-touch outside the timing
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        times = []
        for _ in range(repeats):
            e0.record()
            bs.run(data, outs, check=False)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        bs.run(data, outs, check=True)
        return float(np.median(times))
    finally:
        bs.close()


def autotune(lengths, tsamp, sample_trials=16, repeats=3, cache_file=None, verbose=False,
             **search_kw):
    """Best tuning dict for searching series of these lengths with these parameters. Times
    every candidate on `sample_trials` seeded noise series drawn from `lengths`."""
    import torch

    key = _key(lengths, tsamp, search_kw)
    if key in _CACHE:
        return dict(_CACHE[key])
    if cache_file and os.path.exists(cache_file):
        with open(cache_file) as f:
            disk = json.load(f)
        if key in disk:
            _CACHE[key] = disk[key]["tuning"]
            return dict(_CACHE[key])
    L = np.asarray(lengths, dtype=np.int64)
    rng = np.random.default_rng(12345)
    sample = [int(x) for x in rng.choice(L, size=min(sample_trials, L.size), replace=False)]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(12345)
    data = torch.randn(int(sum(sample)), generator=gen, device="cuda", dtype=torch.float32)
    results = []

    def trial(cand):
        ms = time_search(sample, tsamp, cand, data, repeats=repeats, **search_kw)
        results.append((ms, cand))
        if verbose:
            print("autotune %s: %.3f ms" % (cand, ms), flush=True)

    for cand in candidates(int(search_kw.get("bins_max", 260))):
        trial(cand)
    grid_best = min(results, key=lambda r: r[0])[1]
    for fd in DEEP_FRACTIONS:  # the deep transforms' own rows per job, around the grid's best
        trial(dict(grid_best, rows_fraction_deep=fd))
    results.sort(key=lambda r: r[0])
    best = results[0][1]
    _CACHE[key] = best
    if cache_file:
        disk = {}
        if os.path.exists(cache_file):
            with open(cache_file) as f:
                disk = json.load(f)
        disk[key] = {"tuning": best, "ms": results[0][0],
                     "default_ms": next(ms for ms, c in results if c == DEFAULT)}
        with open(cache_file, "w") as f:
            json.dump(disk, f, indent=1)
    return dict(best)
