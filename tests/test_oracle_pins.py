"""Pins the CPU oracle (oracle/) to the reference: its own known-answer tests and the golden
fixtures that the reference produced (tests/golden/make_golden.py). No GPU."""
import numpy as np
import pytest

from oracle import oracle as O

# tests/test_ffa_base_functions.py:12-36 of the reference: pulse in the last column.
FFA_IN_88 = np.zeros((8, 8), dtype=np.float32)
FFA_IN_88[:, 7] = 1
FFA_OUT_88 = np.array([
    [0, 0, 0, 0, 0, 0, 0, 8],
    [0, 0, 0, 0, 0, 0, 4, 4],
    [0, 0, 0, 0, 0, 2, 4, 2],
    [0, 0, 0, 0, 2, 2, 2, 2],
    [0, 0, 0, 1, 2, 2, 2, 1],
    [0, 0, 1, 2, 1, 1, 2, 1],
    [0, 1, 1, 1, 2, 1, 1, 1],
    [1, 1, 1, 1, 1, 1, 1, 1],
], dtype=np.float32)


def test_ffa_known_answer_and_invariances():
    C = O.C()
    for shift in range(8):
        X = np.roll(FFA_IN_88, shift, axis=1)
        assert np.array_equal(C.ffa2(X), np.roll(FFA_OUT_88, shift, axis=1))
    for extra in range(8):
        X = np.hstack([FFA_IN_88, np.zeros((8, extra), np.float32)])
        truth = np.hstack([FFA_OUT_88, np.zeros((8, extra), np.float32)])
        assert np.array_equal(C.ffa2(X), truth)


def test_ffa2_golden_bit_exact(golden):
    g = golden("ffa2.npz")
    off = 0
    for m, b in g["shapes"]:
        n = int(m * b)
        x = g["inputs"][off:off + n].reshape(m, b)
        y = g["outputs"][off:off + n].reshape(m, b)
        assert np.array_equal(O.C().ffa2(x), y), (m, b)
        off += n


def test_snr_top_hat_known_answer():
    # tests/test_snr.py:62-78 of the reference
    n = 64
    widths = np.arange(1, n)
    data = np.zeros(n, dtype=np.float32)
    for w in range(1, n):
        data[:w] = 1.0
        snr = O.C().snr2(data.reshape(1, -1), widths)[0]
        assert snr.argmax() == w - 1
        h = np.sqrt((n - w) / (n * w))
        assert np.allclose(snr.max(), w * h)


def test_snr2_golden_bit_exact(golden):
    g = golden("snr2.npz")
    for i in range(int(g["n"])):
        y = O.C().snr2(g[f"x{i}"], g[f"w{i}"], float(g[f"s{i}"]))
        assert np.array_equal(y, g[f"y{i}"]), i


def test_snr_errors():
    with pytest.raises(ValueError, match="trial widths"):
        O.C().snr2(np.zeros((1, 32), np.float32), [0, 1])
    with pytest.raises(ValueError, match="trial widths"):
        O.C().snr2(np.zeros((1, 32), np.float32), [1, 32])
    with pytest.raises(ValueError, match="stdnoise"):
        O.C().snr2(np.zeros((1, 32), np.float32), [1, 2], stdnoise=-42.0)


def test_downsample_golden(golden):
    g = golden("downsample.npz")
    for i, f in enumerate(g["factors"]):
        y = O.C().downsample(g["x"], float(f))
        ref = g[f"y{i}"]
        assert y.shape == ref.shape
        # the reference build reorders the float sum (-fassociative-math): rounding only
        assert np.allclose(y, ref, rtol=1e-5, atol=1e-6 * np.sqrt(f)), f


def running_median_naive(data, w):
    # tests/test_running_median.py:7-17 of the reference
    h = w // 2
    padded = np.pad(data, (h, h), mode="edge")
    return np.asarray([np.median(padded[i:i + w]) for i in range(data.size)])


def test_running_median_naive_and_golden(golden):
    x = np.random.default_rng(3).normal(size=100).astype(np.float32)
    for w in [1, 3, 5, 7, 11, 25, 37]:
        assert np.array_equal(O.C().running_median(x, w), running_median_naive(x, w))
    g = golden("running_median.npz")
    for w in g["widths"]:
        assert np.array_equal(O.C().running_median(g["x"], int(w)), g[f"y{w}"])
    with pytest.raises(ValueError, match="odd"):
        O.C().running_median(x, 2)
    with pytest.raises(ValueError, match="< size"):
        O.C().running_median(x[:99], 99)


def test_periodogram_golden(golden):
    g = golden("periodogram.npz")
    for i, (tsamp, pmin, pmax, bmin, bmax) in enumerate(g["cfgs"]):
        p, fb, s = O.C().periodogram(g["x"], tsamp, g[f"w{i}"], pmin, pmax, int(bmin), int(bmax))
        assert np.array_equal(p, g[f"p{i}"]) and np.array_equal(fb, g[f"fb{i}"])
        assert np.allclose(s, g[f"s{i}"], rtol=1e-5, atol=1e-5)
        assert O.C().periodogram_length(g["x"].size, tsamp, pmin, pmax, int(bmin), int(bmax)) == p.size


def test_ffafreq_formula():
    # tests/test_ffa_base_functions.py:84-99 of the reference, against the package function
    from riptide_b200.libffa import ffafreq, ffaprd

    m, p = 42, 127
    dt = np.pi / 1000.0
    s = np.arange(m, dtype=float)
    true_periods = p ** 2 / (p - s / (m - 1.0)) * dt
    assert np.allclose(ffaprd(m * p, p, dt=dt), true_periods)
    assert ffafreq(p, p, dt=dt)[0] == 1.0 / (p * dt)
    for args in [(0, p), (np.pi, p), (m * p, 1), (m * p, np.pi), (m * p, m * p + 1)]:
        with pytest.raises(ValueError):
            ffafreq(*args, dt=dt)
    with pytest.raises(ValueError):
        ffafreq(m * p, p, dt=0)


def test_glue_golden(golden):
    g = golden("glue.npz")
    x = g["x"]
    assert np.array_equal(O.normalise(x), g["norm"])
    assert np.array_equal(O.deredden(x, 1e-3, 0.5, 51), g["dered_w0.5_m51"])
    assert np.array_equal(O.deredden(x, 1e-3, 4.0, 101), g["dered_w4_m101"])
    assert np.array_equal(O.fast_running_median(x, 2001, 101), g["frm_w2001_m101"])
    assert np.array_equal(O.fast_running_median(x, 37, 41), g["frm_w37_m41"])


def test_ffa_search_golden(golden):
    g = golden("ffa_search.npz")
    for i in range(int(g["n"])):
        kw = {k.split("_", 1)[1]: g[k].item() for k in g if k.startswith(f"kw{i}_")}
        dered = kw.pop("deredden", True)
        z, widths, p, fb, s = O.ffa_search(g[f"x{i}"], float(g[f"tsamp{i}"]), deredden_=dered, **kw)
        assert np.array_equal(z, g[f"z{i}"])
        assert np.array_equal(widths, g[f"w{i}"])
        assert np.array_equal(p, g[f"p{i}"]) and np.array_equal(fb, g[f"fb{i}"])
        # the C restatement sums downsampled samples in order; the reference's build
        # reassociates that float32 sum
        assert np.allclose(s, g[f"s{i}"], rtol=1e-5, atol=1e-5)
        assert np.argmax(s.max(axis=1)) == np.argmax(g[f"s{i}"].max(axis=1))


@pytest.mark.skipif(O.ref_libcpp() is None, reason="reference libcpp not built here")
def test_oracle_matches_built_reference_random():
    R = O.ref_libcpp()
    rng = np.random.default_rng(11)
    for m, b in [(3, 5), (17, 240), (333, 260), (1000, 250), (2500, 77)]:
        x = rng.standard_normal((m, b)).astype(np.float32)
        assert np.array_equal(O.C().ffa2(x), R.ffa2(x))
    w = O.generate_width_trials(240)
    x = rng.standard_normal((400, 257)).astype(np.float32) * 3
    assert np.array_equal(O.C().snr2(x, w, 2.5), R.snr2(x, w.astype(np.uint64), 2.5))


def _find_peaks_cases(golden):
    """(periods, foldbins, snrs, widths, tobs, expected) of every find_peaks golden case."""
    g = golden("find_peaks.npz")
    fs = golden("ffa_search.npz")
    out = []
    for i in range(int(g["n"])):
        if i < int(g["n_from_ffa_search"]):
            p, fb, s, w = fs[f"p{i}"], fs[f"fb{i}"], fs[f"s{i}"], fs[f"w{i}"]
        else:
            p, fb, s, w = g[f"p{i}"], g[f"fb{i}"], g[f"s{i}"], g[f"w{i}"]
        exp = {k: g[f"{k}{i}"] for k in ("ip", "iw", "snr", "freq", "ducy", "polycos")}
        out.append((p, fb, s, w, float(g[f"tobs{i}"]), exp))
    return out


def test_find_peaks_golden(golden):
    # the numpy restatement against the reference's own find_peaks (peak_detection.py)
    for p, fb, s, w, tobs, exp in _find_peaks_cases(golden):
        peaks, polycos = O.find_peaks(p, fb, s, w, tobs)
        assert [k[5] for k in peaks] == list(exp["ip"])
        assert [k[4] for k in peaks] == list(exp["iw"])
        assert np.array_equal([k[6] for k in peaks], exp["snr"])
        assert np.array_equal([k[1] for k in peaks], exp["freq"])
        assert np.array_equal([k[3] for k in peaks], exp["ducy"])
        for iw, c in polycos.items():
            ref = exp["polycos"][iw]
            assert np.array_equal(np.asarray(c), ref[~np.isnan(ref)])


def test_cluster1d_known_answers():
    assert O.cluster1d(np.array([]), 1.0) == []
    cl = O.cluster1d(np.array([5.0, 1.0, 1.5, 9.0, 4.6]), 0.6)
    assert [list(c) for c in cl] == [[1, 2], [4, 0], [3]]
