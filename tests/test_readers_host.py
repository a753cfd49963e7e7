"""Readers, metadata, fold argument checks and the fold oracle: host-side checks that need no
GPU. The reader fixtures were written by riptide_b200.reading.writers and parsed by the
reference's own readers (tests/golden/make_golden.py readers); the fold fixtures are the
reference's TimeSeries.fold outputs (make_golden.py fold)."""
import json
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from oracle import oracle as O

# The reference's reader test data (16 samples 0..15 at 64 us, tests/data/README.md), read
# only where the reference tree is present: RIPTIDE_REF_TESTDATA, else the tree that
# oracle/_ref was built from (recorded there by oracle/Makefile).
def _ref_testdata():
    if os.environ.get("RIPTIDE_REF_TESTDATA"):
        return os.environ["RIPTIDE_REF_TESTDATA"]
    rec = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                       "_ref", "source_root.txt")
    if os.path.exists(rec):
        with open(rec) as f:
            return os.path.join(f.read().strip(), "tests", "data")
    return ""


REF_DATA = _ref_testdata()


def _cases():
    g = load_golden("readers.npz")
    return g, json.loads(bytes(g["json"]).decode())


def _write_case(tmp_path, i, doc, g):
    from riptide_b200.reading.writers import write_presto, write_sigproc

    items = dict(doc["items"])
    if doc["kind"] == "presto":
        items["onoff_pairs"] = [tuple(p) for p in items["onoff_pairs"]]
        base = str(tmp_path / f"case{i}")
        write_presto(base, g[f"in{i}"], items)
        return base + ".inf"
    fn = str(tmp_path / f"case{i}.tim")
    write_sigproc(fn, g[f"in{i}"], items)
    return fn


def test_writers_reproduce_fixture_bytes(tmp_path):
    g, docs = _cases()
    for i, doc in enumerate(docs):
        fn = _write_case(tmp_path, i, doc, g)
        if doc["kind"] == "presto":
            assert open(fn, "rb").read() == bytes(g[f"inf{i}"])
            assert open(fn[:-4] + ".dat", "rb").read() == bytes(g[f"dat{i}"])
        else:
            assert open(fn, "rb").read() == bytes(g[f"tim{i}"])


def test_readers_match_reference_parse(tmp_path):
    import warnings

    from riptide_b200 import TimeSeries
    from riptide_b200.reading import PrestoInf, SigprocHeader

    g, docs = _cases()
    for i, doc in enumerate(docs):
        fn = _write_case(tmp_path, i, doc, g)
        if doc["kind"] == "presto":
            hdr = dict(PrestoInf(fn))
            hdr["onoff_pairs"] = [list(p) for p in hdr["onoff_pairs"]]
            with warnings.catch_warnings(record=True) as w:
                warnings.simplefilter("always")
                ts = TimeSeries.from_presto_inf(fn)
            assert bool(w) == (doc["items"]["em_band"] != "Radio")
        else:
            sh = SigprocHeader(fn)
            hdr = dict(sh)
            hdr["_bytesize"] = sh.bytesize
            ts = TimeSeries.from_sigproc(fn)
        assert hdr == doc["header"], i
        assert ts.data.dtype == np.float32
        assert np.array_equal(ts.data, g[f"data{i}"]), i
        assert ts.tsamp == doc["tsamp"]
        assert ts.metadata["dm"] == doc["dm"]
        assert ts.metadata["tobs"] == doc["tobs"]


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference test data not mounted")
def test_reference_data_files():
    """tests/test_time_series.py:16-62 of the reference on its own data files."""
    from riptide_b200 import TimeSeries

    ref = np.arange(16)
    for fn in ("fake_presto_radio.inf", "fake_presto_radio_breaks.inf"):
        ts = TimeSeries.from_presto_inf(os.path.join(REF_DATA, fn))
        assert ts.nsamp == 16 and ts.tsamp == 64e-6 and ts.data.dtype == np.float32
        assert np.allclose(ts.data, ref)
    with pytest.warns(UserWarning):
        ts = TimeSeries.from_presto_inf(os.path.join(REF_DATA, "fake_presto_xray.inf"))
    assert np.allclose(ts.data, ref)
    for fn in ("fake_sigproc_float32.tim", "fake_sigproc_uint8.tim", "fake_sigproc_int8.tim"):
        ts = TimeSeries.from_sigproc(os.path.join(REF_DATA, fn))
        assert ts.nsamp == 16 and ts.tsamp == 64e-6 and ts.data.dtype == np.float32
        assert np.allclose(ts.data, ref)
    with pytest.raises(ValueError):
        TimeSeries.from_sigproc(os.path.join(REF_DATA, "fake_sigproc_uint8_nosignedkey.tim"))


def _sig_header(**kw):
    h = dict(source_name="X", telescope_id=4, machine_id=10, src_raj=0.0, src_dej=0.0,
             data_type=2, refdm=1.0, fch1=1400.0, nchans=1, nbits=32, tstart=56000.0,
             tsamp=1e-3, nifs=1)
    h.update(kw)
    return h


def test_sigproc_errors(tmp_path):
    from riptide_b200 import TimeSeries
    from riptide_b200.reading import SigprocHeader
    from riptide_b200.reading.writers import write_sigproc

    x = np.arange(64)
    fn = str(tmp_path / "a.tim")
    write_sigproc(fn, x, _sig_header(nchans=4))
    with pytest.raises(ValueError, match="multi-channel"):
        TimeSeries.from_sigproc(fn)
    write_sigproc(fn, x, _sig_header(nbits=16))
    with pytest.raises(ValueError, match="8-bit and 32-bit"):
        TimeSeries.from_sigproc(fn)
    write_sigproc(fn, x, _sig_header(nbits=8))
    with pytest.raises(ValueError, match="signedness"):
        TimeSeries.from_sigproc(fn)
    # a non-standard key needs extra_keys
    write_sigproc(fn, x, _sig_header(num_trusses=3), extra_keys={"num_trusses": int})
    with pytest.raises(KeyError, match="num_trusses"):
        SigprocHeader(fn)
    ts = TimeSeries.from_sigproc(fn, extra_keys={"num_trusses": int})
    assert ts.metadata["num_trusses"] == 3 and np.array_equal(ts.data, x)
    with open(fn, "wb") as f:
        f.write(struct.pack("i", 5) + b"HELLO")
    with pytest.raises(AssertionError):
        SigprocHeader(fn)


def test_presto_errors(tmp_path):
    from riptide_b200.reading import inf2dict

    g, docs = _cases()
    fn = _write_case(tmp_path, 0, docs[0], g)
    text = open(fn).read()
    with pytest.raises(ValueError, match="makedata"):
        inf2dict(text.replace("Parkes", "None (Artificial Data Set)"))
    with pytest.raises(ValueError, match="EM Band"):
        inf2dict(text.replace("=  Radio", "=  Optical"))
    with pytest.raises(ValueError, match="column 40"):
        inf2dict(text.replace(" Telescope used                         =",
                              " Telescope used                        ="))


def test_payload_read_errors(tmp_path):
    from riptide_b200.reading import read_payload

    with pytest.raises(OSError):
        read_payload(str(tmp_path / "missing.dat"), 0, 10, "f32")
    fn = tmp_path / "short.dat"
    np.arange(10, dtype=np.float32).tofile(fn)
    with pytest.raises(OSError, match="fewer"):
        read_payload(str(fn), 0, 11, "f32")
    assert np.array_equal(read_payload(str(fn), 8, None, "f32"), np.arange(2, 10))
    big = tmp_path / "big.dat"
    v = np.random.default_rng(0).integers(0, 256, (5 << 20) + 3).astype(np.uint8)
    v.tofile(big)
    y = read_payload(str(big), 3, v.size - 3, "u8", threads=7)
    assert np.array_equal(y, v[3:].astype(np.float32))


def test_metadata_schema():
    from riptide_b200 import Metadata

    m = Metadata({"dm": 3.0, "tobs": 10.0})
    assert m["source_name"] is None and m["skycoord"] is None
    with pytest.raises(ValueError):
        Metadata({"dm": -1.0})
    with pytest.raises(ValueError):
        Metadata({"tobs": 0.0})
    with pytest.raises(TypeError):
        Metadata({"extra": object()})


# --------------------------------------------------------------------------------- folding
def _fold_cases():
    import importlib.util

    spec = importlib.util.spec_from_file_location("mg", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.FOLD_CASES


def test_fold_oracle_pinned_to_reference():
    g = load_golden("fold.npz")
    for i, (s, period, bins, subints) in enumerate(_fold_cases()):
        y = O.fold(g[f"x{s}"], float(g[f"tsamp{s}"]), period, bins, subints)
        ref = g[f"y{i}"]
        assert y.shape == ref.shape, i
        # the reference build sums with vectorised (reassociated) float32 adds
        assert np.allclose(y, ref, rtol=1e-5, atol=2e-6), i


def test_fold_shape_and_errors():
    from riptide_b200.folding import fold_shape

    g = load_golden("fold.npz")
    for i, (s, period, bins, subints) in enumerate(_fold_cases()):
        n = g[f"x{s}"].size
        assert fold_shape(n, float(g[f"tsamp{s}"]), period, bins, subints) == g[f"y{i}"].shape
    n, tsamp = 10000, 1e-3  # the reference's test_methods series: 10 s at 1 ms
    assert fold_shape(n, tsamp, 1.0, 100) == (10, 100)
    assert fold_shape(n, tsamp, 1.0, 100, 2) == (2, 100)
    assert fold_shape(n, tsamp, 1.0, 100, 10) == (10, 100)
    assert fold_shape(n, tsamp, 1.0, 100, 1) == (100,)
    with pytest.raises(ValueError, match="exceeds the number"):
        fold_shape(n, tsamp, 1.0, 100, 1000000)
    with pytest.raises(ValueError, match="subints"):
        fold_shape(n, tsamp, 1.0, 100, 0)
    with pytest.raises(ValueError, match="Bin width"):
        fold_shape(n, tsamp, 1.0, 1000000)
    with pytest.raises(ValueError, match="Period exceeds"):
        fold_shape(n, tsamp, 1.0e6, 100)
    with pytest.raises(ValueError, match="Bin width"):
        fold_shape(n, tsamp, 1.0e-6, 100)


def test_worker_pool_configuration():
    from riptide_b200 import WorkerPool

    with pytest.raises(ValueError, match="format"):
        WorkerPool({"rmed_width": 5.0, "rmed_minpts": 101}, [{"ffa_search": {}}], fmt="fits")
    with pytest.raises(ValueError, match="unknown ffa_search"):
        WorkerPool({"rmed_width": 5.0, "rmed_minpts": 101},
                   [{"ffa_search": {"period_min": 1.0, "bogus": 1}, "find_peaks": {}}])
    with pytest.raises(ValueError, match="at least one"):
        WorkerPool({"rmed_width": 5.0, "rmed_minpts": 101}, [])


def test_stacked_polyfit_is_np_polyfit():
    """The threshold fits of find_peaks_batched, stacked into one least-squares call, return
    exactly np.polyfit's coefficients (peak_detection.py:89-109 fits one width at a time)."""
    from riptide_b200.peaks import _polyfit_stacked

    rng = np.random.default_rng(11)
    for M in (10, 47, 333):
        X = np.sort(rng.uniform(-5.0, 3.0, (700, M)), axis=1)
        Y = rng.standard_normal((700, M)) * 2.0 + 8.0
        for deg in (2, 2.0, 3):
            C = _polyfit_stacked(X, Y, deg)
            R = np.array([np.polyfit(X[k], Y[k], deg) for k in range(X.shape[0])])
            assert np.array_equal(C, R), (M, deg)


def test_stacked_polyfit_falls_back_when_the_private_call_differs(monkeypatch):
    """The stacked call uses numpy's private LAPACK gufunc; it is checked against np.polyfit
    once, and when it is missing or disagrees every fit is an np.polyfit call."""
    from riptide_b200 import peaks

    assert peaks._stacked_ok()  # numpy of this image: the stacked call is exact
    X = np.sort(np.random.default_rng(12).uniform(-5.0, 3.0, (20, 15)), axis=1)
    Y = np.random.default_rng(13).standard_normal((20, 15))
    R = np.array([np.polyfit(X[k], Y[k], 2) for k in range(20)])
    monkeypatch.setattr(peaks, "_STACKED_OK", None)
    monkeypatch.setattr(peaks, "_ulinalg", None)
    assert not peaks._stacked_ok()
    assert np.array_equal(peaks._polyfit_stacked(X, Y, 2), R)
    monkeypatch.setattr(peaks, "_STACKED_OK", None)
    monkeypatch.setattr(peaks, "_polyfit_lapack", lambda *a: np.zeros((2, 3)))
    assert not peaks._stacked_ok()
    assert np.array_equal(peaks._polyfit_stacked(X, Y, 2), R)


def test_candidate_subints_rule():
    """candidate.py:76-104: subints falls back to None when that many periods exceed the data."""
    from riptide_b200.folding import candidate_subints, fold_shape

    length = 10.0
    assert candidate_subints(1.0, 32, length) is None
    assert candidate_subints(0.25, 32, length) == 32
    assert candidate_subints(0.3125, 32, length) is None  # 32 periods == the data length
    assert candidate_subints(2.0, None, length) is None
    assert candidate_subints(2.0, 1, length) == 1
    # the folded shapes the candidate stage gets for a 10 s series at 1 ms
    assert fold_shape(10000, 1e-3, 1.0, 100, candidate_subints(1.0, 32, length)) == (10, 100)
    assert fold_shape(10000, 1e-3, 0.25, 100, candidate_subints(0.25, 32, length)) == (32, 100)
