"""GPU checks of the ingest path (rt_ingest_files, rt_samples_to_f32), of folding (rt_fold,
rt_fold_batched) against the reference's TimeSeries.fold fixtures, and of the batched
WorkerPool against the peaks of the reference's own WorkerPool."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mg():
    import importlib.util

    spec = importlib.util.spec_from_file_location("mg", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


# ---------------------------------------------------------------------------------- ingest
def test_samples_to_f32_exact():
    import torch

    from riptide_b200 import _lib, libcpp

    lib = _lib.load()
    raw = torch.arange(0, 256, dtype=torch.int32).to(torch.uint8).repeat(41)[:10001].cuda()
    for enc, np_t in ((_lib.RT_SAMPLES_U8, np.uint8), (_lib.RT_SAMPLES_I8, np.int8)):
        out = torch.empty(raw.numel(), dtype=torch.float32, device="cuda")
        _lib.check(lib.rt_samples_to_f32(libcpp._ptr(raw), enc, raw.numel(), libcpp._ptr(out),
                                         libcpp._stream()))
        ref = raw.cpu().numpy().view(np_t).astype(np.float32)
        assert np.array_equal(out.cpu().numpy(), ref)
    with pytest.raises(ValueError):
        _lib.check(lib.rt_samples_to_f32(libcpp._ptr(raw), 7, 4, libcpp._ptr(out),
                                         libcpp._stream()))


def test_load_series_batch(tmp_path):
    """Packed float32 device tensor equal to numpy's astype of each payload, across chunk
    boundaries of a small staging buffer and for ragged lengths."""
    import torch

    from riptide_b200.reading import SeriesFile, load_series_batch

    rng = np.random.default_rng(5)
    specs = [("f32", 300001), ("u8", 200003), ("i8", 77), ("f32", 1), ("u8", 0), ("i8", 150000)]
    files, refs = [], []
    for i, (enc, n) in enumerate(specs):
        off = 13 * i + 3
        if enc == "f32":
            v = rng.standard_normal(n).astype(np.float32)
        elif enc == "u8":
            v = rng.integers(0, 256, n).astype(np.uint8)
        else:
            v = rng.integers(-128, 128, n).astype(np.int8)
        fn = tmp_path / f"s{i}.bin"
        with open(fn, "wb") as f:
            f.write(b"\x01" * off)
            f.write(v.tobytes())
        files.append(SeriesFile(str(fn), off, n, enc, 1e-3, {}))
        refs.append(v.astype(np.float32))
    ref = np.concatenate(refs)
    for staging in (128 << 10, 1 << 20, 64 << 20):
        out, lengths = load_series_batch(files, staging_bytes=staging, threads=3)
        torch.cuda.synchronize()
        assert list(lengths) == [n for _, n in specs]
        assert np.array_equal(out.cpu().numpy(), ref), staging


# ---------------------------------------------------------------------------------- folding
def test_fold_matches_reference_fixtures():
    from riptide_b200 import TimeSeries

    g = load_golden("fold.npz")
    for i, (s, period, bins, subints) in enumerate(_mg().FOLD_CASES):
        ts = TimeSeries(g[f"x{s}"], float(g[f"tsamp{s}"]))
        y = ts.fold(period, bins, subints=subints)
        ref = g[f"y{i}"]
        assert y.shape == ref.shape, i
        # downsampled windows are summed in FP64 and rounded once; the reference sums in
        # float32 (vectorised): agreement to float32 rounding of the window sums
        assert np.allclose(y, ref, rtol=1e-5, atol=2e-6), (i, np.abs(y - ref).max())
        o = O.fold(g[f"x{s}"], float(g[f"tsamp{s}"]), period, bins, subints)
        assert np.allclose(y, o, rtol=1e-5, atol=2e-6), i


def test_fold_batched_equals_single_folds():
    from riptide_b200 import TimeSeries, fold_batched

    x = np.random.default_rng(8).standard_normal(1 << 17).astype(np.float32)
    ts = TimeSeries(x, 64e-6)
    periods = [0.0731, 0.25, 0.5, 1.0, 2.9, 7.9]
    subints = [None, 16, 3, 1, 2, None]
    many = fold_batched(ts, periods, 128, subints)
    for p, s, y in zip(periods, subints, many):
        assert np.array_equal(y, ts.fold(p, 128, subints=s))


def test_fold_candidates_rule():
    """Candidate folding (candidate.py:76-104): every period folded with the requested
    sub-integrations, or all full periods where that many do not fit."""
    from riptide_b200 import TimeSeries, fold_candidates

    x = np.random.default_rng(9).standard_normal(100000).astype(np.float32)
    ts = TimeSeries(x, 1e-4)  # 10 s
    periods = [0.25, 0.5, 1.0, 3.0]
    got = fold_candidates(ts, periods, 64, subints=16)
    for p, y in zip(periods, got):
        want = ts.fold(p, 64, subints=None if 16 * p >= ts.length else 16)
        assert np.array_equal(y, want)
    assert got[0].shape == (16, 64) and got[2].shape == (10, 64)


def test_fold_reference_methods():
    """tests/test_time_series.py:106-204 of the reference (the folding part)."""
    from riptide_b200 import TimeSeries

    np.random.seed(1)
    ts = TimeSeries.generate(10.0, 1.0e-3, 1.0, amplitude=25.0, stdnoise=1.0)
    bins = 100
    X10 = ts.fold(1.0, bins, subints=None)
    assert X10.shape == (10, bins)
    X2 = ts.fold(1.0, bins, subints=2)
    assert X2.shape == (2, bins)
    Xm = ts.fold(1.0, bins, subints=10)
    prof = ts.fold(1.0, bins, subints=1)
    assert np.allclose(prof, X2.sum(axis=0), atol=1e-5)
    assert np.allclose(prof, X10.sum(axis=0), atol=1e-5)
    assert np.allclose(prof, Xm.sum(axis=0), atol=1e-5)
    for kw in (dict(period=1.0, bins=bins, subints=1000000), dict(period=1.0, bins=bins, subints=0),
               dict(period=1.0, bins=1000000), dict(period=1.0e6, bins=bins),
               dict(period=1.0e-6, bins=bins)):
        with pytest.raises(ValueError):
            ts.fold(**kw)


# ------------------------------------------------------------------------------ worker pool
def test_worker_pool_matches_reference(tmp_path):
    """The reference's WorkerPool.process_fname_list on its pipeline test signal (three DM
    trials, ranges of tests/pipeline_config_A.yml: bins 480-520 and 960-1040): the same
    peaks (trial, width, period index) in the same order, S/N to float32 rounding."""
    from riptide_b200 import TimeSeries, WorkerPool
    from riptide_b200.reading.writers import write_presto

    mg = _mg()
    g = load_golden("workerpool.npz")
    fnames = []
    for i, (dm, amp, ducy) in enumerate(mg.WP_TRIALS):
        np.random.seed(0)
        ts = TimeSeries.generate(mg.WP_TOBS, mg.WP_TSAMP, mg.WP_PERIOD, amplitude=amp,
                                 ducy=ducy, stdnoise=1.0)
        assert ts.data.astype(np.float64).sum() == g[f"sum{i}"]
        base = str(tmp_path / f"fake_DM{dm:.3f}")
        write_presto(base, ts.data, mg.workerpool_inf(os.path.basename(base), ts.nsamp, dm))
        fnames.append(base + ".inf")
    pool = WorkerPool(mg.WP_DEREDDEN, mg.WP_RANGES, processes=2, fmt="presto")
    try:
        peaks = pool.process_fname_list(fnames)
        single = [p for f in fnames for p in pool.process_fname(f)]
    finally:
        pool.close()
    assert len(peaks) == len(g["snr"])
    for key in ("iw", "ip", "width", "dm"):
        assert np.array_equal(np.array([getattr(p, key) for p in peaks]), g[key]), key
    assert np.allclose([p.snr for p in peaks], g["snr"], rtol=1e-5)
    assert np.allclose([p.period for p in peaks], g["period"], rtol=1e-12)
    assert [(p.iw, p.ip, p.snr) for p in single] == [(p.iw, p.ip, p.snr) for p in peaks]


def test_worker_pool_sigproc_8bit_equals_float(tmp_path):
    """8-bit SIGPROC files (payload copied as bytes, widened on the GPU) give the same peaks as
    float32 PRESTO files holding the same values."""
    from riptide_b200 import WorkerPool, generate_signal
    from riptide_b200.reading.writers import write_presto, write_sigproc

    rng = np.random.default_rng(21)
    tsamp, n = 1e-3, 150000
    ranges = [{"ffa_search": {"period_min": 0.5, "period_max": 5.0, "bins_min": 240,
                              "bins_max": 260}, "find_peaks": {"smin": 6.0}}]
    dered = {"rmed_width": 4.0, "rmed_minpts": 101}
    tims, infs = [], []
    for i, signed in enumerate((True, False, True)):
        x = generate_signal(n, (0.7 + 0.3 * i) / tsamp, ducy=0.03, amplitude=25.0, rng=rng)
        v = np.clip(np.round(x * 12.0) + (0 if signed else 128), -128 if signed else 0,
                    127 if signed else 255)
        hdr = dict(source_name="fake", telescope_id=4, machine_id=10, data_type=2,
                   refdm=float(i), fch1=1400.0, nchans=1, nbits=8, signed=signed,
                   tstart=60000.0, tsamp=tsamp, nifs=1, src_raj=0.0, src_dej=0.0)
        fn = str(tmp_path / f"t{i}.tim")
        write_sigproc(fn, v, hdr)
        tims.append(fn)
        base = str(tmp_path / f"p{i}")
        write_presto(base, v.astype(np.float32), dict(
            basename=f"p{i}", telescope="Parkes", instrument="x", source_name="fake",
            raj="00:00:00.0000", decj="00:00:00.0000", observer="x", mjd=60000.0,
            barycentered=False, nsamp=n, tsamp=tsamp, breaks=False, em_band="Radio",
            fov_arcsec=1.0, dm=float(i), fbot=1200.0, bandwidth=400.0, nchan=1, cbw=1.0,
            analyst="x"))
        infs.append(base + ".inf")
    a = WorkerPool(dered, ranges, fmt="sigproc", chunk_trials=2)
    b = WorkerPool(dered, ranges, fmt="presto", chunk_trials=2)
    try:
        pa, pb = a.process_fname_list(tims), b.process_fname_list(infs)
    finally:
        a.close()
        b.close()
    assert pa and [(p.iw, p.ip, p.snr, p.dm) for p in pa] == [(p.iw, p.ip, p.snr, p.dm) for p in pb]
