"""C ABI checks that need no GPU: the library loads, exports every function that
include/riptide_b200.h declares, and its host-side planning agrees with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O


def declared_functions():
    src = open(os.path.join(ROOT, "include", "riptide_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**\s*\**\s*(rt_[a-z0-9_]+)\s*\(",
                       src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from riptide_b200 import _lib

    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding table covers all of them
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_periodogram_length_matches_oracle():
    from riptide_b200 import libcpp

    cases = [(1 << 20, 1e-4, 0.5, 5.0, 240, 260), (4000000, 64e-6, 0.2, 30.0, 240, 260),
             (1 << 23, 64e-6, 0.2, 60.0, 480, 520), (50000, 1e-3, 0.24, 0.6, 240, 260)]
    for c in cases:
        assert libcpp.periodogram_length(*c) == O.C().periodogram_length(*c)
    with pytest.raises(ValueError, match="period_min >= tsamp"):
        libcpp.periodogram_length(1000, 1e-3, 0.1, 1.0, 240, 260)
    with pytest.raises(ValueError, match="bins_max must be >= bins_min"):
        libcpp.periodogram_length(1000, 1e-3, 0.5, 1.0, 240, 200)


def test_downsampled_size():
    from riptide_b200 import libcpp

    for n, f in [(1000, 1.5), (1 << 22, 13.020833333333334), (10, 10.0)]:
        assert libcpp.downsampled_size(n, f) == O.C().downsampled_size(n, f)


def test_batched_plan_rows_match_oracle_lengths():
    from riptide_b200 import BatchedSearch

    rng = np.random.default_rng(5)
    lengths = rng.integers(int(0.9 * 2 ** 22), 2 ** 22 + 1, size=6)
    bs = BatchedSearch(lengths, 64e-6, period_min=0.2, period_max=30.0)
    try:
        rows = np.diff(bs.row_offsets)
        expect = [O.C().periodogram_length(int(n), 64e-6, 0.2, 30.0, 240, 260) for n in lengths]
        assert list(rows) == expect
        assert bs.stats["num_cycles"] == 60
        assert bs.stats["total_samples"] == int(lengths.sum())
    finally:
        bs.close()


def test_batched_plan_errors():
    from riptide_b200 import BatchedSearch

    with pytest.raises(ValueError, match="period_max must be > period_min"):
        BatchedSearch([100000], 1e-3, period_min=2.0, period_max=1.0)
    with pytest.raises(ValueError, match="tsamp must be > 0"):
        BatchedSearch([100000], 0.0)
    with pytest.raises(ValueError, match="trial widths"):
        BatchedSearch([100000], 1e-3, period_min=0.5, period_max=2.0, widths=[1, 240])
    with pytest.raises(ValueError, match="min_points must be an odd number"):
        BatchedSearch([100000], 1e-3, period_min=0.5, period_max=2.0, rmed_minpts=100)
    with pytest.raises(ValueError, match="Downsampling factor"):
        # the last octave needs f > size
        BatchedSearch([200], 1e-3, period_min=0.24, period_max=60.0, deredden=False)


def test_tuned_plan_checks_and_shapes():
    # tuning changes the work split only: same periodogram rows; invalid values are rejected
    from riptide_b200 import BatchedSearch

    kw = dict(period_min=0.2, period_max=30.0)
    base = BatchedSearch([2 ** 22], 64e-6, **kw)
    tuned = BatchedSearch([2 ** 22], 64e-6, tuning={"rows_fraction": 0.7, "snr_threads": 16,
                                                     "lag_items": 100}, **kw)
    try:
        assert np.array_equal(base.row_offsets, tuned.row_offsets)
        assert tuned.stats["num_transforms"] == base.stats["num_transforms"]
        assert tuned.stats["num_work_items"] > base.stats["num_work_items"]  # smaller jobs
    finally:
        base.close()
        tuned.close()
    # rows_fraction_deep applies only to transforms of more than 8 jobs' worth of rows: a
    # smaller value cuts those into more jobs, but fewer than the same fraction everywhere
    plans = [BatchedSearch([2 ** 22], 64e-6, tuning=t, **kw)
             for t in ({"rows_fraction": 1.0}, {"rows_fraction_deep": 0.6}, {"rows_fraction": 0.6})]
    try:
        items = [p.stats["num_work_items"] for p in plans]
        assert all(np.array_equal(plans[0].row_offsets, p.row_offsets) for p in plans)
        assert items[0] < items[1] < items[2], items
    finally:
        for p in plans:
            p.close()
    for bad in ({"rows_fraction": 1.5}, {"snr_threads": 12}, {"lag_items": -1},
                {"rows_fraction_deep": -0.1}):
        with pytest.raises(ValueError):
            BatchedSearch([100000], 1e-3, period_min=0.5, period_max=2.0, tuning=bad)


def test_tile_rules_checks_and_shapes():
    # per-(rows, bins) rules change the work split of the transforms they hold only: the same
    # periodogram rows; fewer levels per job cut the deep transforms into more stages
    from riptide_b200 import BatchedSearch
    from riptide_b200 import tuning as TU

    kw = dict(period_min=0.2, period_max=30.0)
    base = BatchedSearch([2 ** 22], 64e-6, **kw)
    deep = [{"rows_min": 512, "rows_max": 4095, "bins_min": 240, "bins_max": 260, "max_levels": 5}]
    narrow = [{"rows_min": 64, "rows_max": 127, "bins_min": 240, "bins_max": 250,
               "rows_fraction": 0.5, "snr_threads": 16}]
    plans = [BatchedSearch([2 ** 22], 64e-6, rules=r, **kw) for r in (deep, narrow, deep + narrow)]
    try:
        items = [p.stats["num_work_items"] for p in plans]
        assert all(np.array_equal(base.row_offsets, p.row_offsets) for p in plans)
        assert all(p.stats["num_transforms"] == base.stats["num_transforms"] for p in plans)
        assert items[0] > base.stats["num_work_items"]           # more stages
        assert items[1] > base.stats["num_work_items"]           # smaller jobs
        assert items[2] == items[0] + items[1] - base.stats["num_work_items"]
    finally:
        base.close()
        for p in plans:
            p.close()
    good = {"rows_min": 8, "rows_max": 100, "bins_min": 240, "bins_max": 260}
    for bad in ({"rows_min": 10, "rows_max": 5}, {"bins_min": 261, "bins_max": 260},
                {"rows_fraction": 1.5}, {"snr_threads": 12}, {"max_levels": 9}):
        with pytest.raises(ValueError, match="tile rule"):
            BatchedSearch([100000], 1e-3, period_min=0.5, period_max=2.0, rules=[dict(good, **bad)])
    # the autotuner's octaves cover the search's periods, each with its rows range
    oct_ = TU.rows_octaves([2 ** 22] * 3, 64e-6, 0.2, 30.0, 240, 260)
    assert oct_[0]["period_max"] == 30.0 and abs(oct_[-1]["period_min"] - 0.2) < 1e-12
    for a, b in zip(oct_, oct_[1:]):
        assert abs(a["period_min"] - b["period_max"]) < 1e-9 and b["rows_min"] == 2 * a["rows_min"]
