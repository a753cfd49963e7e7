"""Parity of the CUDA path (through the C ABI) with the oracle and the reference's golden
fixtures. Tolerances: FFA transform, running median, scrunch, deredden, periods and fold bins
are bit-exact; the normalised series is within one float32 ulp (the float64 mean and standard
deviation are summed in another order than numpy's); S/N is bit-exact when its inputs are
identical. Downsampling and everything downstream of it (the reference's build reorders that
float32 sum) is held to rtol 1e-5 with an absolute floor of 2e-5 S/N units for values near
zero, where a relative bound means nothing; every peak (row and width) is the same."""
import numpy as np
import pytest

from oracle import oracle as O
from test_oracle_pins import FFA_IN_88, FFA_OUT_88

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import riptide_b200

    return riptide_b200


# ------------------------------------------------------------------------------ FFA
def test_ffa2_known_answer(rb):
    for shift in range(8):
        X = np.roll(FFA_IN_88, shift, axis=1)
        assert np.array_equal(rb.ffa2(X), np.roll(FFA_OUT_88, shift, axis=1))
        assert np.array_equal(rb.ffa1(X.ravel(), 8), np.roll(FFA_OUT_88, shift, axis=1))
    for extra in range(8):
        X = np.hstack([FFA_IN_88, np.zeros((8, extra), np.float32)])
        truth = np.hstack([FFA_OUT_88, np.zeros((8, extra), np.float32)])
        assert np.array_equal(rb.ffa2(X), truth)


def test_ffa2_errors(rb):
    with pytest.raises(ValueError):
        rb.ffa2(np.zeros(4))
    with pytest.raises(ValueError):
        rb.ffa1(np.zeros((4, 4)), 4)
    with pytest.raises(ValueError):
        rb.ffa1(np.zeros(10), 11)
    with pytest.raises(ValueError):
        rb.ffa1(np.zeros(10), 4.0)
    with pytest.raises(ValueError, match="contiguous"):
        rb.libcpp.ffa2(np.zeros((8, 8), np.float32)[:, ::2])


def test_ffa2_golden(rb, golden):
    g = golden("ffa2.npz")
    off = 0
    for m, b in g["shapes"]:
        n = int(m * b)
        x = g["inputs"][off:off + n].reshape(m, b)
        assert np.array_equal(rb.libcpp.ffa2(x), g["outputs"][off:off + n].reshape(m, b)), (m, b)
        off += n


@pytest.mark.parametrize("m,b", [(1, 7), (2, 240), (3, 260), (63, 241), (107, 260), (108, 259),
                                 (150, 250), (511, 240), (1342, 240), (1241, 260), (2684, 480),
                                 (1290, 520), (5000, 61), (20000, 3), (257, 1000)])
def test_ffa2_random_bit_exact(rb, m, b):
    x = np.random.default_rng(m * 1000 + b).standard_normal((m, b)).astype(np.float32)
    assert np.array_equal(rb.libcpp.ffa2(x), O.C().ffa2(x))


def test_ffa2_device_tensor(rb):
    import torch

    x = np.random.default_rng(1).standard_normal((300, 251)).astype(np.float32)
    t = torch.from_numpy(x).cuda()
    y = rb.libcpp.ffa2(t)
    assert y.is_cuda and np.array_equal(y.cpu().numpy(), O.C().ffa2(x))


# ------------------------------------------------------------------------------ S/N
def test_snr2_golden_bit_exact(rb, golden):
    g = golden("snr2.npz")
    for i in range(int(g["n"])):
        y = rb.libcpp.snr2(g[f"x{i}"], g[f"w{i}"], float(g[f"s{i}"]))
        assert np.array_equal(y, g[f"y{i}"]), i


@pytest.mark.parametrize("b,widths", [
    (240, O.generate_width_trials(240)), (260, O.generate_width_trials(240)),
    (251, O.generate_width_trials(251)), (480, O.generate_width_trials(480)),
    (520, O.generate_width_trials(480)), (300, O.generate_width_trials(300, ducy_max=0.3)),
    (64, np.arange(1, 64)), (33, [1, 5, 7, 32]), (1000, [3, 30, 300])])
def test_snr2_random_bit_exact(rb, b, widths):
    x = (np.random.default_rng(b).standard_normal((777, b)) * 4).astype(np.float32)
    y = rb.libcpp.snr2(x, widths, 1.75)
    assert np.array_equal(y, O.C().snr2(x, widths, 1.75))


def test_snr_properties(rb):
    # tests/test_snr.py of the reference: errors, shapes, phase-roll invariance, top hat
    data = np.zeros(32, dtype="float32")
    for bad in ([0, 1], [1, 32]):
        with pytest.raises(ValueError):
            rb.boxcar_snr(data, bad)
    with pytest.raises(ValueError):
        rb.boxcar_snr(data, [1, 2], stdnoise=-42.0)
    w = [1, 2, 3, 5]
    assert rb.boxcar_snr(np.zeros(32, np.float32), w).shape == (4,)
    assert rb.boxcar_snr(np.zeros((4, 32), np.float32), w).shape == (4, 4)
    assert rb.boxcar_snr(np.zeros((3, 4, 32), np.float32), w).shape == (3, 4, 4)
    d = np.random.default_rng(2).normal(size=(4, 32)).astype("float32")
    ref = rb.boxcar_snr(d, [1, 2, 5, 11, 18, 31])
    for shift in range(1, 33):
        assert np.allclose(rb.boxcar_snr(np.roll(d, shift, axis=-1), [1, 2, 5, 11, 18, 31]), ref)
    n = 64
    data = np.zeros(n, dtype="float32")
    for width in range(1, n):
        data[:width] = 1.0
        snr = rb.boxcar_snr(data, np.arange(1, n))
        assert snr.argmax() == width - 1
        assert np.allclose(snr.max(), width * np.sqrt((n - width) / (n * width)))


# ------------------------------------------------------------------------------ downsample
def test_downsample_golden_and_oracle(rb, golden):
    g = golden("downsample.npz")
    x = g["x"]
    for i, f in enumerate(g["factors"]):
        y = rb.downsample(x, float(f))
        assert y.shape == g[f"y{i}"].shape
        assert np.allclose(y, g[f"y{i}"], rtol=1e-5, atol=1e-6 * np.sqrt(f)), f
        y64 = O.C().downsample(x.astype(np.float64), float(f), f64=True)
        assert np.max(np.abs(y - y64)) <= 1e-6 * max(1.0, np.abs(y64).max()), f


def test_downsample_wide_and_errors(rb):
    # wide windows: the reference's float32 running sum over f samples carries rounding of
    # order f * eps * rms; the GPU sum is formed in FP64 and rounded once.
    x = np.random.default_rng(9).standard_normal(200003).astype(np.float32)
    for f in [4093.5, 5000.0, 12345.678, 200003.0]:
        y = rb.downsample(x, f)
        y64 = O.C().downsample(x.astype(np.float64), f, f64=True)
        assert np.max(np.abs(y - y64)) <= 1e-6 * max(1.0, np.abs(y64).max()), f
        assert np.allclose(y, O.C().downsample(x, f), rtol=1e-5, atol=1.2e-7 * f)
    for f in [0.55, 1.0, 200004.0]:
        with pytest.raises(ValueError, match="Downsampling factor"):
            rb.downsample(x, f)


def test_downsample_independent_of_alignment(rb):
    # a device view starting 1-3 floats past a 16-byte boundary takes the kernel's realigned
    # staging path; its outputs equal those of an aligned copy of the same samples
    import torch

    x = np.random.default_rng(12).standard_normal(300_007).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    for f in [1.5, 13.02, 100.37, 1953.1, 4000.0]:
        for k in range(4):
            view = xt[k:]
            assert view.data_ptr() % 16 == (xt.data_ptr() + 4 * k) % 16
            got = rb.libcpp.downsample(view, f).cpu().numpy()
            assert np.array_equal(got, rb.libcpp.downsample(x[k:].copy(), f)), (f, k)
            y64 = O.C().downsample(x[k:].astype(np.float64), f, f64=True)
            assert np.max(np.abs(got - y64)) <= 1e-6 * max(1.0, np.abs(y64).max()), (f, k)
    # a long series: several hundred segments, more CTAs than the SMs hold at once
    x = np.random.default_rng(13).standard_normal(3_000_017).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    for f in [2.5, 1953.1]:
        for k in (0, 3):
            got = rb.libcpp.downsample(xt[k:], f).cpu().numpy()
            assert np.array_equal(got, rb.libcpp.downsample(x[k:].copy(), f)), (f, k)
            y64 = O.C().downsample(x[k:].astype(np.float64), f, f64=True)
            assert np.max(np.abs(got - y64)) <= 1e-6 * max(1.0, np.abs(y64).max()), (f, k)
    # a series that is not 4-byte aligned is refused before any launch
    out = torch.empty(1000, dtype=torch.float32, device="cuda")
    lib = rb._lib.load()
    st = rb.libcpp._stream()
    assert lib.rt_downsample(xt.data_ptr() + 2, 1000, 7.5, out.data_ptr(), st) == rb._lib.RT_EINVAL
    assert "aligned" in lib.rt_last_error().decode()
    assert lib.rt_downsample(xt.data_ptr() + 4, 1000, 7.5, out.data_ptr(), st) == rb._lib.RT_OK


# ------------------------------------------------------------------------------ running median
def test_running_median(rb, golden):
    g = golden("running_median.npz")
    for w in g["widths"]:
        assert np.array_equal(rb.running_median(g["x"], int(w)), g[f"y{w}"]), w
    data = np.random.default_rng(4).normal(size=300).reshape(100, 3).astype("float32")
    for col in data.T:  # non-contiguous column slices
        for w in [1, 3, 5, 7, 11, 25, 37]:
            assert np.array_equal(rb.running_median(col, w), O.C().running_median(col, w))
    d10 = np.arange(10, dtype="float32")
    for args in [(d10, 2), (d10, 10), (d10[:9], 9), (np.zeros((4, 8)), 3)]:
        with pytest.raises(ValueError):
            rb.running_median(*args)


@pytest.mark.parametrize("width,minpts", [(40000, 101), (202001, 101), (505001, 101), (1200, 7)])
def test_fast_running_median_scrunch_orders(rb, width, minpts):
    # scrunch factors 396, 2000, 5000, 171: the recursion of numpy's pairwise sum has 4, 16,
    # 64 and 2 leaves (the lane-parallel kernel up to 32 leaves, the warp-per-point one above)
    x = (np.random.default_rng(width).standard_normal(3_000_017) * 2 + 5).astype(np.float32)
    assert np.array_equal(rb.fast_running_median(x, width, minpts),
                          O.fast_running_median(x, width, minpts))


def test_fast_running_median_noscrunch(rb):
    x = np.random.default_rng(5).normal(size=100)
    for w in [1, 3, 5, 7, 11, 25, 37]:
        assert np.array_equal(rb.running_median(x, w), rb.fast_running_median(x, w, min_points=39))
    with pytest.raises(ValueError):
        rb.fast_running_median(np.zeros(100), 3, min_points=10)


# ------------------------------------------------------------------------------ glue
def _within_one_ulp(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ulp = np.spacing(np.maximum(np.abs(a), np.abs(b)))
    return a.shape == b.shape and bool(np.all(np.abs(a.astype(np.float64) - b) <= ulp))


def test_normalise_deredden_golden(rb, golden):
    g = golden("glue.npz")
    ts = rb.TimeSeries(g["x"], 1e-3)
    assert _within_one_ulp(ts.normalise().data, g["norm"])
    assert np.array_equal(ts.deredden(0.5, minpts=51).data, g["dered_w0.5_m51"])
    assert np.array_equal(ts.deredden(4.0, minpts=101).data, g["dered_w4_m101"])
    assert np.array_equal(rb.fast_running_median(g["x"], 2001, 101), g["frm_w2001_m101"])
    assert np.array_equal(rb.fast_running_median(g["x"], 37, 41), g["frm_w37_m41"])
    tc = rb.TimeSeries(np.full(10000, 42.42, np.float32), 1e-3)
    assert np.allclose(tc.deredden(0.5, minpts=51).data, 0.0, atol=1e-5)


# ------------------------------------------------------------------------------ periodogram
def _check_pgram(p, fb, s, p_ref, fb_ref, s_ref, rtol=1e-5, atol=2e-5):
    assert np.array_equal(p, p_ref)
    assert np.array_equal(fb, fb_ref)
    assert s.shape == s_ref.shape
    assert np.allclose(s, s_ref, rtol=rtol, atol=atol)
    assert np.argmax(s.max(axis=1)) == np.argmax(s_ref.max(axis=1))
    assert np.argmax(s.max(axis=0)) == np.argmax(s_ref.max(axis=0))


def test_periodogram_golden(rb, golden):
    g = golden("periodogram.npz")
    for i, (tsamp, pmin, pmax, bmin, bmax) in enumerate(g["cfgs"]):
        args = (g["x"], tsamp, g[f"w{i}"], pmin, pmax, int(bmin), int(bmax))
        out = rb.libcpp.periodogram(*args)
        _check_pgram(*out, g[f"p{i}"], g[f"fb{i}"], g[f"s{i}"])
        plain = rb.libcpp.periodogram_plain(*args)
        for a, b in zip(out, plain):
            assert np.array_equal(a, b)


def test_periodogram_config1_full_size(rb):
    # 2^20 samples, 100 us, P 0.5-5 s, bins 240-260: the reference's own C++ when built here
    rng = np.random.default_rng(100000)
    x = rb.generate_signal(1 << 20, 1.0 / 1e-4, ducy=0.02, amplitude=20.0, rng=rng)
    x = O.normalise(x)
    w = O.generate_width_trials(240)
    R = O.ref_libcpp()
    ref = (R.periodogram(x, 1e-4, w.astype(np.uint64), 0.5, 5.0, 240, 260) if R is not None
           else O.C().periodogram(x, 1e-4, w, 0.5, 5.0, 240, 260))
    out = rb.libcpp.periodogram(x, 1e-4, w, 0.5, 5.0, 240, 260)
    _check_pgram(*out, *ref)


def test_periodogram_empty_is_an_error_like_the_reference(rb):
    with pytest.raises(IndexError):
        rb.libcpp.periodogram(np.zeros(200, np.float32), 1e-3, [1, 2], 0.24, 60.0, 240, 260)


def test_ffa_search_golden(rb, golden):
    g = golden("ffa_search.npz")
    for i in range(int(g["n"])):
        kw = {k.split("_", 1)[1]: g[k].item() for k in g if k.startswith(f"kw{i}_")}
        ts = rb.TimeSeries(g[f"x{i}"], float(g[f"tsamp{i}"]))
        tsdr, pg = rb.ffa_search(ts, **kw)
        assert _within_one_ulp(tsdr.data, g[f"z{i}"])
        assert np.array_equal(pg.widths, g[f"w{i}"])
        _check_pgram(pg.periods, pg.foldbins, pg.snrs, g[f"p{i}"], g[f"fb{i}"], g[f"s{i}"])
    ts = rb.TimeSeries(g["x0"], float(g["tsamp0"]))
    tsdr, pg = rb.ffa_search(ts, period_min=0.5, period_max=5.0, deredden=False,
                             already_normalised=True)
    assert tsdr is ts  # search.py:41-50 of the reference tests


# ------------------------------------------------------------------------------ batched
def test_batched_equals_single(rb):
    rng = np.random.default_rng(77)
    lengths = [70001, 65536, 90000, 50000, 81234]
    series = [rb.generate_signal(n, 0.9 / 5e-4 + 13 * i, ducy=0.04, amplitude=15.0, rng=rng)
              .astype(np.float32) + 0.5 for i, n in enumerate(lengths)]
    kw = dict(period_min=0.2, period_max=3.0, bins_min=240, bins_max=260, rmed_width=1.0)
    pgs = rb.ffa_search_batched(series, 5e-4, **kw)
    for s, pg in zip(series, pgs):
        tsdr, one = rb.ffa_search(rb.TimeSeries(s, 5e-4), **kw)
        assert np.array_equal(pg.snrs, one.snrs)
        assert np.array_equal(pg.periods, one.periods)
        z, widths, p, fb, sn = O.ffa_search(s, 5e-4, **kw)
        _check_pgram(pg.periods, pg.foldbins, pg.snrs, p, fb, sn)


def test_batched_full_size_trial(rb):
    # one 2^22-sample trial at the batched configuration, against the oracle
    rng = np.random.default_rng(300007)
    x = rb.generate_signal(1 << 22, 0.731 / 64e-6, ducy=0.03, amplitude=25.0, rng=rng).astype(np.float32)
    pgs, zs = rb.BatchedSearch([x.size], 64e-6, period_min=0.2, period_max=30.0).search(
        [x], return_normalised=True)
    z, widths, p, fb, sn = O.ffa_search(x, 64e-6, period_min=0.2, period_max=30.0)
    assert _within_one_ulp(zs[0], z)
    _check_pgram(pgs[0].periods, pgs[0].foldbins, pgs[0].snrs, p, fb, sn)


def test_pipeline_equals_batched(rb):
    # host-buffer pipeline (4 chunks of 1, 2, 1, 1 trials: quarter chunks first and last, both
    # device buffer pairs reused) against the device-resident batched search of the same
    # trials: identical outputs
    rng = np.random.default_rng(78)
    lengths = [70001, 65536, 90000, 50000, 81234]
    series = [rb.generate_signal(n, 0.9 / 5e-4 + 11 * i, ducy=0.04, amplitude=12.0, rng=rng)
              .astype(np.float32) + 0.25 for i, n in enumerate(lengths)]
    kw = dict(period_min=0.2, period_max=3.0, bins_min=240, bins_max=260, rmed_width=1.0)
    pipe = rb.SearchPipeline(lengths, 5e-4, chunk_trials=2, **kw)
    assert pipe.num_chunks == 4
    for _ in range(2):  # second run reuses every buffer and event
        pgs = pipe.search(series)
    ref = rb.ffa_search_batched(series, 5e-4, **kw)
    for a, b in zip(pgs, ref):
        assert np.array_equal(a.periods, b.periods)
        assert np.array_equal(a.foldbins, b.foldbins)
        assert np.array_equal(a.snrs, b.snrs)
    host_in, outs = pipe.allocate_host()
    with pytest.raises(ValueError):
        pipe.run(host_in[:-1], outs)
    pipe.close()


def test_batched_graph_replay(rb):
    # the whole run replayed as one CUDA graph gives the same periodograms as direct launches;
    # replays with the same tensors reuse the graph, new output tensors capture a new one
    import torch

    rng = np.random.default_rng(79)
    lengths = [70001, 65536, 90000]
    series = [rng.standard_normal(n).astype(np.float32) for n in lengths]
    kw = dict(period_min=0.2, period_max=3.0, bins_min=240, bins_max=260, rmed_width=1.0)
    bs = rb.BatchedSearch(lengths, 5e-4, **kw)
    data = torch.from_numpy(np.concatenate(series)).cuda()
    ref = [t.clone() for t in bs.run(data)]
    bs.enable_graph(True)
    outs = bs.allocate_outputs()
    for _ in range(2):
        for t in outs:
            t.zero_()
        bs.run(data, outs)
        for a, b in zip(outs, ref):
            assert torch.equal(a, b)
    assert bs.graph_captures == 1
    outs2 = bs.allocate_outputs()
    bs.run(data, outs2)
    assert bs.graph_captures == 2
    for a, b in zip(outs2, ref):
        assert torch.equal(a, b)
    bs.close()


@pytest.mark.parametrize("bmin,bmax,ducy,pmax", [
    (480, 520, 0.2, 8.0),    # the large batched configuration's bins (12 widths, 16-thread S/N)
    (100, 110, 0.2, 4.0),    # bins outside the unrolled ranges (generic level loops)
    (300, 320, 0.3, 6.0),    # more widths than the 10-width register window (generic widths)
])
def test_batched_engine_other_bins(rb, bmin, bmax, ducy, pmax):
    # the persistent engine at bins and width sets other than the default, against the oracle
    # (C restatement) on the same dereddened + normalised series
    rng = np.random.default_rng(bmin)
    n = 1 << 21
    x = rb.generate_signal(n, 0.61 / 64e-6, ducy=0.02, amplitude=20.0, rng=rng).astype(np.float32)
    kw = dict(period_min=0.2, period_max=pmax, bins_min=bmin, bins_max=bmax, ducy_max=ducy)
    bs = rb.BatchedSearch([n], 64e-6, **kw)
    pgs, zs = bs.search([x], return_normalised=True)
    z, widths, p, fb, sn = O.ffa_search(x, 64e-6, **kw)
    assert np.array_equal(pgs[0].widths, widths)
    assert _within_one_ulp(zs[0], z)
    _check_pgram(pgs[0].periods, pgs[0].foldbins, pgs[0].snrs, p, fb, sn)
    bs.close()


def test_tuned_engine_is_bit_identical(rb):
    # the tile choices change the work split, never the periodogram; the autotuner returns
    # one of its candidates
    import torch

    from riptide_b200 import tuning as TU

    rng = np.random.default_rng(81)
    lengths = [300001, 262144, 280000]
    x = torch.from_numpy(np.concatenate([rng.standard_normal(n).astype(np.float32)
                                         for n in lengths])).cuda()
    kw = dict(period_min=0.2, period_max=8.0, bins_min=240, bins_max=260)
    ref = [t.clone() for t in rb.BatchedSearch(lengths, 64e-6, **kw).run(x)]
    for tun in ({"rows_fraction": 0.6}, {"snr_threads": 16}, {"lag_items": 64},
                {"rows_fraction": 0.8, "snr_threads": 16, "lag_items": 2000}):
        bs = rb.BatchedSearch(lengths, 64e-6, tuning=tun, **kw)
        out = bs.run(x)
        for a, b in zip(out, ref):
            assert torch.equal(a, b), tun
        bs.close()
    best = TU.autotune(lengths, 64e-6, sample_trials=2, repeats=1, **kw)
    grid = TU.candidates(260)
    assert best in grid or (best["rows_fraction_deep"] in TU.DEEP_FRACTIONS
                            and dict(best, rows_fraction_deep=0.0) in grid)
    assert TU.autotune(lengths, 64e-6, sample_trials=2, repeats=1, **kw) == best  # cached
    # a 2^22-sample series has transforms of more than 8 jobs' worth of rows, which the deep
    # fraction cuts into more jobs: the same periodogram
    y = torch.from_numpy(rng.standard_normal(1 << 22).astype(np.float32)).cuda()
    kw = dict(period_min=0.2, period_max=30.0)
    a = rb.BatchedSearch([1 << 22], 64e-6, **kw)
    b = rb.BatchedSearch([1 << 22], 64e-6, tuning={"rows_fraction_deep": 0.5}, **kw)
    assert b.stats["num_work_items"] > a.stats["num_work_items"]
    for u, v in zip(a.run(y), b.run(y)):
        assert torch.equal(u, v)
    a.close()
    b.close()


def test_tile_rules_are_bit_identical(rb):
    # per-(rows, bins) rules (rows per job, S/N threads, levels per job in shared memory)
    # change the work split, never the periodogram; the per-octave autotuner returns rules
    # over the octaves it timed
    import torch

    from riptide_b200 import tuning as TU

    rng = np.random.default_rng(82)
    lengths = [1 << 22, 4000000]
    x = torch.from_numpy(np.concatenate([rng.standard_normal(n).astype(np.float32)
                                         for n in lengths])).cuda()
    kw = dict(period_min=0.2, period_max=30.0)
    base = rb.BatchedSearch(lengths, 64e-6, **kw)
    ref = [t.clone() for t in base.run(x)]
    base.close()
    for rules in ([{"rows_min": 512, "rows_max": 4095, "bins_min": 240, "bins_max": 260,
                    "max_levels": 5}],
                  [{"rows_min": 1, "rows_max": 1 << 20, "bins_min": 240, "bins_max": 249,
                    "rows_fraction": 0.7, "snr_threads": 16},
                   {"rows_min": 100, "rows_max": 300, "bins_min": 250, "bins_max": 260,
                    "max_levels": 4, "rows_fraction": 0.85}]):
        bs = rb.BatchedSearch(lengths, 64e-6, rules=rules, **kw)
        for a, b in zip(bs.run(x), ref):
            assert torch.equal(a, b), rules
        bs.close()
    res = TU.autotune_rules(lengths[:1], 64e-6, sample_trials=1, repeats=1,
                            candidates=TU.RULE_CANDIDATES[:2], period_min=0.2, period_max=30.0)
    assert res["rules"] and len(res["rules"]) == len(res["per_octave"])
    assert res["ms_rules"] > 0 and res["ms_default"] > 0
    bs = rb.BatchedSearch(lengths, 64e-6, rules=res["rules"], **kw)
    for a, b in zip(bs.run(x), ref):
        assert torch.equal(a, b)
    bs.close()


@pytest.mark.parametrize("config_id", [2, 5])
def test_survey_configurations_full_size(rb, config_id):
    """One full-size series of the single survey-length configuration (2^23 samples, white +
    1/f noise, three pulsars, P 0.2-60 s) and of the large sweep's generator (2^23 samples,
    bins 480-520, 12 widths), through the batched engine, against the
    reference's own libcpp periodogram (the oracle's glue for deredden and normalise; the C
    restatement where the reference could not be built)."""
    from riptide_b200 import synth

    cfg = synth.CONFIGS[config_id]
    n = int(synth.trial_lengths(config_id, 1, 0)[0])
    x, _ = synth.make_trial(config_id, 0, n, cfg["tsamp"], "cuda")
    x = x.cpu().numpy()
    kw = dict(cfg["search"])
    bs = rb.BatchedSearch([n], cfg["tsamp"], **kw)
    pgs, zs = bs.search([x], return_normalised=True)
    bs.close()
    z, widths, p, fb, sn = O.ffa_search(x, cfg["tsamp"], libcpp=O.ref_libcpp(), **kw)
    assert np.array_equal(pgs[0].widths, widths)
    assert _within_one_ulp(zs[0], z)
    _check_pgram(pgs[0].periods, pgs[0].foldbins, pgs[0].snrs, p, fb, sn)


def _peak_key(pk):
    return [(int(q[4]), int(q[5])) for q in sorted(pk, key=lambda q: (q[4], q[5]))]


def _check_peaks(peaks, polycos, ref_peaks, ref_polycos, periods):
    """Every peak (width index, row) identical, peak S/N within 1e-5 relative, and the
    dynamic thresholds (each width's fitted polynomial at every trial period) within 1e-5."""
    assert _peak_key(peaks) == _peak_key(ref_peaks)
    a = np.array([q[6] for q in sorted(peaks, key=lambda q: (q[4], q[5]))])
    b = np.array([q[6] for q in sorted(ref_peaks, key=lambda q: (q[4], q[5]))])
    assert np.allclose(a, b, rtol=1e-5, atol=0)
    logf = np.log(1.0 / np.asarray(periods))
    assert sorted(polycos) == sorted(ref_polycos)
    for iw in ref_polycos:
        ta = np.polyval(np.asarray(polycos[iw], np.float64), logf)
        tb = np.polyval(np.asarray(ref_polycos[iw], np.float64), logf)
        assert np.allclose(ta, tb, rtol=1e-5, atol=0), iw


def test_headline_batch_against_reference(rb):
    """Trials of the 512-trial benchmark configuration (U[0.9, 1]*2^22 samples, 64 us, white
    + 1/f noise, pulsars in 30%, P 0.2-30 s, bins 240-260), generated and packed exactly as
    the benchmark does and searched in one BatchedSearch replayed as a CUDA graph. Each trial
    is compared with the reference's own libcpp periodogram (glue restated in numpy, as the
    reference's search.py runs it): dereddened series bit-identical, normalised series within
    one ulp, periods and fold bins identical, S/N within rtol 1e-5, and the peaks that
    find_peaks reports on the device identical to those of the reference's find_peaks
    (restated) on the reference's periodogram."""
    from riptide_b200 import synth

    cfg = synth.CONFIGS[3]
    tsamp, kw = cfg["tsamp"], dict(cfg["search"])
    data, lengths, infos = synth.make_batch(3, 8, first_index=0)
    bs = rb.BatchedSearch(lengths, tsamp, **kw)
    bs.enable_graph(True)
    periods, foldbins, snrs = bs.run(data)
    peaks = rb.find_peaks_batched(periods, foldbins, snrs, bs.row_offsets,
                                  [n * tsamp for n in lengths], bs.widths)
    p_all, fb_all, s_all = (periods.cpu().numpy(), foldbins.cpu().numpy().view(np.uint32),
                            snrs.cpu().numpy())
    host = data.cpu().numpy()
    bs.close()
    npulsar = 0
    for t, n in enumerate(lengths):
        x = host[int(bs.sample_offsets[t]):int(bs.sample_offsets[t + 1])]
        z, widths, p, fb, sn = O.ffa_search(x, tsamp, libcpp=O.ref_libcpp(), **kw)
        a, b = bs.row_offsets[t], bs.row_offsets[t + 1]
        _check_pgram(p_all[a:b], fb_all[a:b], s_all[a:b], p, fb, sn)
        ref_peaks, ref_poly = O.find_peaks(p, fb, sn, widths, n * tsamp)
        _check_peaks(peaks[t][0], peaks[t][1], ref_peaks, ref_poly, p)
        npulsar += bool(infos[t]["pulsars"])
    assert npulsar >= 1  # the sample carries injected pulsars as well as noise-only trials


def test_error_against_fp64(rb):
    """The error of each output against FP64 arithmetic on the same input, next to the
    reference's own error (its libcpp, float32):
    * S/N: FP64 periodogram (FP64 downsample, FFA and boxcar S/N) of the FP64 normalised
      series; the GPU sums the downsampled samples in FP64 and rounds once, the reference in
      float32;
    * dereddened series: the FP64 running-median pipeline (FP64 scrunch mean);
    * downsampled series: FP64 window sums."""
    from riptide_b200 import synth

    cfg = synth.CONFIGS[3]
    tsamp, kw = cfg["tsamp"], dict(cfg["search"])
    n = int(synth.trial_lengths(3, 1, 3)[0])
    x, _ = synth.make_trial(3, 3, n, tsamp, "cuda")
    x = x.cpu().numpy()
    bs = rb.BatchedSearch([n], tsamp, **kw)
    pgs, zs = bs.search([x], return_normalised=True)
    bs.close()
    y = rb.TimeSeries(x, tsamp).deredden(kw["rmed_width"], minpts=kw["rmed_minpts"]).data
    y64 = x.astype(np.float64) - _fast_running_median_f64(x.astype(np.float64),
                                                           int(round(kw["rmed_width"] / tsamp)),
                                                           kw["rmed_minpts"])
    z64 = (y.astype(np.float64) - y.mean(dtype=np.float64)) / y.std(dtype=np.float64)
    w = O.generate_width_trials(kw["bins_min"])
    _, _, s64 = O.C().periodogram(z64, tsamp, w, kw["period_min"], kw["period_max"],
                                  kw["bins_min"], kw["bins_max"], f64=True)
    R = O.ref_libcpp()
    _, _, sref = (R.periodogram(zs[0], tsamp, w.astype(np.uint64), kw["period_min"],
                                kw["period_max"], kw["bins_min"], kw["bins_max"]) if R is not None
                  else O.C().periodogram(zs[0], tsamp, w, kw["period_min"], kw["period_max"],
                                         kw["bins_min"], kw["bins_max"]))
    scale = np.maximum(1.0, np.abs(s64))
    err_gpu = float(np.max(np.abs(pgs[0].snrs - s64) / scale))
    err_ref = float(np.max(np.abs(sref - s64) / scale))
    err_dered = float(np.max(np.abs(y - y64)))
    f = 100.37
    d = rb.downsample(zs[0], f)
    d64 = O.C().downsample(zs[0].astype(np.float64), f, f64=True)
    err_ds = float(np.max(np.abs(d - d64)) / np.abs(d64).max())
    print(f"\nerror vs FP64: S/N {err_gpu:.3g} (reference {err_ref:.3g}); dereddened "
          f"{err_dered:.3g}; downsampled {err_ds:.3g} relative to the largest value")
    assert err_gpu <= 1e-5 and err_gpu <= err_ref * 1.5
    assert err_dered <= 1e-3
    assert err_ds <= 1e-6


def _fast_running_median_f64(x, width_samples, min_points):
    """running_medians.py:49-85 in FP64: FP64 scrunch mean, exact median, np.interp."""
    k = int(max(1, width_samples / float(min_points)))
    if k == 1:
        return O.C().running_median(x.astype(np.float32), width_samples).astype(np.float64)
    N = (x.size // k) * k
    lo = x[:N].reshape(-1, k).mean(axis=1)
    half = min_points // 2
    pad = np.concatenate([np.full(half, lo[0]), lo, np.full(half, lo[-1])])
    win = np.lib.stride_tricks.sliding_window_view(pad, min_points)
    rm = np.median(win, axis=1)
    xl = np.arange(lo.size) * k + 0.5 * (k - 1)
    return np.interp(np.arange(x.size), xl, rm)
