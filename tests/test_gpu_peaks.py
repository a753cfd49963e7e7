"""Peak detection on the device (riptide_b200.peaks) against the reference's find_peaks
(golden peak lists, tests/golden/find_peaks.npz) and the oracle restatement: the same peaks
(period-trial index, width index, S/N, frequency, duty cycle) and the same threshold
polynomials, exactly."""
import numpy as np
import pytest

from oracle import oracle as O
from test_oracle_pins import _find_peaks_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import riptide_b200

    return riptide_b200


def _same(peaks, polycos, exp):
    assert [k.ip for k in peaks] == list(exp["ip"])
    assert [k.iw for k in peaks] == list(exp["iw"])
    assert np.array_equal([k.snr for k in peaks], exp["snr"])
    assert np.array_equal([k.freq for k in peaks], exp["freq"])
    assert np.array_equal([k.ducy for k in peaks], exp["ducy"])
    for iw, c in polycos.items():
        ref = exp["polycos"][iw]
        assert np.array_equal(np.asarray(c, dtype=np.float64), ref[~np.isnan(ref)])


def test_find_peaks_golden(rb, golden):
    for p, fb, s, w, tobs, exp in _find_peaks_cases(golden):
        pg = rb.Periodogram(w, p, fb, s, metadata={"tobs": tobs, "dm": None})
        peaks, polycos = rb.find_peaks(pg)
        _same(peaks, polycos, exp)


def test_find_peaks_batched_equals_single(rb, golden):
    import torch

    cases = [c for c in _find_peaks_cases(golden)]
    w = cases[0][3]
    cases = [c for c in cases if np.array_equal(c[3], w)]
    assert len(cases) >= 2
    p = torch.from_numpy(np.concatenate([c[0] for c in cases])).cuda()
    fb = torch.from_numpy(np.concatenate([c[1].astype(np.int64) for c in cases])).cuda()
    s = torch.from_numpy(np.concatenate([c[2] for c in cases])).cuda()
    rows = np.concatenate([[0], np.cumsum([c[0].size for c in cases])])
    res = rb.find_peaks_batched(p, fb, s, rows, [c[4] for c in cases], w)
    for (peaks, polycos), c in zip(res, cases):
        _same(peaks, polycos, c[5])


def test_search_then_peaks_on_device(rb):
    # the batched search's device outputs straight into peak detection, against the oracle's
    # find_peaks on the same periodograms copied to the host
    rng = np.random.default_rng(17)
    lengths = [1 << 18, 200000]
    series = [rb.generate_signal(n, 0.83 / 1e-3, ducy=0.03, amplitude=18.0, rng=rng)
              .astype(np.float32) for n in lengths]
    bs = rb.BatchedSearch(lengths, 1e-3, period_min=0.5, period_max=5.0)
    import torch

    x = torch.from_numpy(np.concatenate(series)).cuda()
    per, fb, sn = bs.run(x)
    tobs = np.asarray(lengths) * 1e-3
    res = rb.find_peaks_batched(per, fb, sn, bs.row_offsets, tobs, bs.widths)
    P, F, S = per.cpu().numpy(), fb.cpu().numpy().view(np.uint32), sn.cpu().numpy()
    for t, (peaks, polycos) in enumerate(res):
        a, b = bs.row_offsets[t], bs.row_offsets[t + 1]
        ref, refpc = O.find_peaks(P[a:b], F[a:b], S[a:b], bs.widths, tobs[t])
        assert [(k.ip, k.iw, k.snr) for k in peaks] == [(k[5], k[4], k[6]) for k in ref]
        assert peaks and abs(peaks[0].period - 0.83) < 0.01
        for iw in polycos:
            assert np.array_equal(np.asarray(polycos[iw], dtype=np.float64),
                                  np.asarray(refpc[iw], dtype=np.float64))
    bs.close()


def _segment_case(rng, m, p, extra, T):
    """A periodogram of m segments of p points (+ extra trailing points), frequencies
    decreasing over (m - 0.5) segment widths, S/N with ties."""
    w = 5.0 / T
    n = m * p + extra
    f = 3.0 - np.linspace(0.0, (m - 0.5) * w, n)
    s = np.round(rng.standard_normal((n, 3)) * 2.0 + 5.0, 1).astype(np.float32)
    return 1.0 / f, s


@pytest.mark.parametrize("ps", [[3, 5, 64, 127], [129, 1000, 3000], [4312, 5000],
                                [5, 129, 1000, 4312, 9000, 16000]])
def test_peak_segments_sizes(rb, ps):
    """rt_peak_segments against numpy's median / percentiles (the oracle's segment_stats) for
    segments of 3 to 16000 points: every on-chip sort size (128 to 16384 values) and several
    trials of different segment sizes in one launch."""
    import ctypes

    import torch

    from riptide_b200 import _lib, libcpp

    rng = np.random.default_rng(len(ps) * 7 + ps[0])
    T = 100.0
    cases = [_segment_case(rng, 11 + k, p, k % 3, T) for k, p in enumerate(ps)]
    per = torch.from_numpy(np.concatenate([c[0] for c in cases])).cuda()
    snr = torch.from_numpy(np.concatenate([c[1] for c in cases])).cuda()
    rows = np.concatenate([[0], np.cumsum([c[0].size for c in cases])]).astype(np.uint64)
    tobs = np.full(len(cases), T)
    segoff = np.zeros(len(cases) + 1, dtype=np.uint64)
    lib, dp = _lib.load(), ctypes.POINTER(ctypes.c_double)
    args = (libcpp._ptr(per), None, 3, rows.ctypes.data_as(_lib._u64p), len(cases),
            tobs.ctypes.data_as(dp), 5.0, 6.0, segoff.ctypes.data_as(_lib._u64p))
    _lib.check(lib.rt_peak_segments(*args, None, None, libcpp._stream()))
    fc = torch.empty(int(segoff[-1]), dtype=torch.float64, device="cuda")
    sc = torch.empty((int(segoff[-1]), 3), dtype=torch.float64, device="cuda")
    _lib.check(lib.rt_peak_segments(libcpp._ptr(per), libcpp._ptr(snr), *args[2:],
                                    libcpp._ptr(fc), libcpp._ptr(sc), libcpp._stream()))
    fc, sc = fc.cpu().numpy(), sc.cpu().numpy()
    for t, (periods, s) in enumerate(cases):
        a, b = int(segoff[t]), int(segoff[t + 1])
        for iw in range(3):
            # the reference casts each width's S/N to float64 first (peak_detection.py:205)
            f_ref, smed, sstd = O.segment_stats(1.0 / periods, s[:, iw].astype(float), T)
            assert b - a == f_ref.size
            assert np.array_equal(fc[a:b], f_ref)
            assert np.array_equal(sc[a:b, iw], smed + 6.0 * sstd), (t, iw)
