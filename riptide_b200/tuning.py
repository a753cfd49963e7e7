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


# --------------------------------------------------------------------------------------
# Tile choices per (rows, bins): rules for the plan (rt_tile_rule)
# --------------------------------------------------------------------------------------
RULE_CANDIDATES = [
    {"rows_fraction": rf, "snr_threads": tpr, "max_levels": lv}
    for rf in (1.0, 0.85, 0.7) for tpr in (8, 16) for lv in (8, 6)
]


def rows_octaves(lengths, tsamp, period_min, period_max, bins_min, bins_max):
    """The row octaves [2^k, 2^(k+1)) that the transforms of this search span. A transform
    folding at period P over an observation of T seconds has about T / P rows, so each
    octave is the sub-search over the periods (T / 2^(k+1), T / 2^k] (within the search's
    range), which the autotuner times on its own."""
    T = float(np.median(np.asarray(lengths, dtype=np.float64))) * float(tsamp)
    out = []
    k = 0
    while T / 2 ** k > period_min:
        lo, hi = max(period_min, T / 2 ** (k + 1)), min(period_max, T / 2 ** k)
        if hi > lo * (1.0 + 1e-9) and T / 2 ** (k + 1) < period_max:
            out.append({"octave": k, "rows_min": 2 ** k, "rows_max": 2 ** (k + 1) - 1,
                        "period_min": lo, "period_max": hi})
        k += 1
    return out


def autotune_rules(lengths, tsamp, sample_trials=16, repeats=5, candidates=None,
                   verbose=False, **search_kw):
    """Tile choices per row octave and bins range (the rules of BatchedSearch(rules=...)).

    Each octave of transform rows is timed on its own: the search restricted to the periods
    whose transforms have that many rows (rows_octaves), on `sample_trials` seeded noise
    series drawn from `lengths`, once per candidate (rows per job, S/N threads per profile,
    levels per job in shared memory), with CUDA events. The fastest candidate of each octave
    becomes its rule. Returns {"rules": [...], "per_octave": [{octave, period range, ms per
    candidate, best}], "ms_default": ..., "ms_rules": ...} where the last two time the
    search kernel on the whole sample search without and with the rules."""
    import torch

    kw = dict(search_kw)
    pmin, pmax = float(kw.pop("period_min", 1.0)), float(kw.pop("period_max", 30.0))
    bmin, bmax = int(kw.get("bins_min", 240)), int(kw.get("bins_max", 260))
    cands = list(candidates or RULE_CANDIDATES)
    if bmax > 264:
        cands = [c for c in cands if c["snr_threads"] != 8]
    L = np.asarray(lengths, dtype=np.int64)
    rng = np.random.default_rng(12345)
    sample = [int(x) for x in rng.choice(L, size=min(sample_trials, L.size), replace=False)]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(12345)
    data = torch.randn(int(sum(sample)), generator=gen, device="cuda", dtype=torch.float32)
    per_octave, rules = [], []
    for oc in rows_octaves(sample, tsamp, pmin, pmax, bmin, bmax):
        sub = dict(kw, period_min=oc["period_min"], period_max=oc["period_max"])
        res = []
        for c in cands:
            rule = dict(c, rows_min=oc["rows_min"], rows_max=oc["rows_max"], bins_min=bmin,
                        bins_max=bmax)
            try:
                ms = _time_rules(sample, tsamp, [rule], data, repeats, **sub)
            except ValueError:
                continue
            res.append((ms, c))
            if verbose:
                print("octave %d %s: %.4f ms" % (oc["octave"], c, ms), flush=True)
        if not res:
            continue
        res.sort(key=lambda r: r[0])
        best = res[0][1]
        per_octave.append(dict(oc, best=best, ms={json.dumps(c, sort_keys=True): ms for ms, c in res}))
        rules.append(dict(best, rows_min=oc["rows_min"], rows_max=oc["rows_max"], bins_min=bmin,
                          bins_max=bmax))
    full = dict(kw, period_min=pmin, period_max=pmax)
    ms_default = _time_rules(sample, tsamp, None, data, repeats, **full)
    ms_rules = _time_rules(sample, tsamp, rules, data, repeats, **full) if rules else ms_default
    return {"rules": rules, "per_octave": per_octave, "ms_default": ms_default,
            "ms_rules": ms_rules, "sample_trials": len(sample)}


def _time_rules(lengths, tsamp, rules, data, repeats, **search_kw):
    """Median CUDA-event time (ms) of the search kernel (the FFA + S/N launch, which the
    rules change) in one engine run with tile `rules` on `data`."""
    from .batched import BatchedSearch

    bs = BatchedSearch(lengths, tsamp, rules=rules, **search_kw)
    try:
        outs = bs.allocate_outputs()
        bs.run(data, outs)
        bs.enable_timing(True)
        times = []
        for _ in range(repeats):
            bs.run(data, outs, check=False)
            times.append(bs.last_timing()[2])
        bs.run(data, outs, check=True)
        return float(np.median(times))
    finally:
        bs.close()
