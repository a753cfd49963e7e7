"""Generate the golden fixtures in this folder from the REFERENCE implementation itself.

Run in a container where the reference project is mounted (default /root/reference,
override with RIPTIDE_REF_ROOT):

    make -C oracle ref            # the reference's libcpp, built from its own sources
    python tests/golden/make_golden.py
    python tests/golden/make_golden.py dropin    # the libcpp call trace of the glue

What it runs: the reference's compiled ``libcpp`` (oracle/_ref) for the C++ kernels, and the
reference's own Python glue (src/riptide/{search,time_series,running_medians,libffa,
ffautils}.py) imported from the reference tree. The glue imports matplotlib, astropy and
schema, which are not installed here; they are replaced by inert stand-ins that none of
the code paths exercised below call (plotting, sky coordinates, metadata validation).

Inputs are seeded (numpy default_rng); every input is stored beside its output, so the
tests need neither the reference nor this script at run time.
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_ROOT = os.environ.get("RIPTIDE_REF_ROOT", "/root/reference")
sys.path.insert(0, REPO)


def _install_stubs():
    class _Anything:
        def __init__(self, *a, **k):
            self.schema = a[0] if a else None

        def __call__(self, *a, **k):
            return _Anything()

        def __getattr__(self, name):
            return _Anything()

        def validate(self, x):
            return x

    def mod(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        m.__getattr__ = lambda n: _Anything()
        sys.modules[name] = m
        return m

    mpl = mod("matplotlib")
    mpl.pyplot = mod("matplotlib.pyplot")
    ap = mod("astropy")
    ap.units = mod("astropy.units")
    ap.coordinates = mod("astropy.coordinates",
                         SkyCoord=type("SkyCoord", (), {"__init__": lambda self, *a, **k: None}))
    mod("schema", Schema=_Anything, And=_Anything, Or=_Anything, Optional=_Anything)


def import_reference(libcpp=None):
    """Import the reference package `riptide` from REF_ROOT with the compiled libcpp (or the
    given stand-in for it)."""
    from oracle import oracle as O

    libcpp = libcpp if libcpp is not None else O.ref_libcpp()
    if libcpp is None:
        raise SystemExit("reference libcpp missing: run `make -C oracle ref` first")
    _install_stubs()
    pkg = types.ModuleType("riptide")
    pkg.__path__ = [os.path.join(REF_ROOT, "src", "riptide")]
    sys.modules["riptide"] = pkg
    sys.modules["riptide.libcpp"] = libcpp
    pkg.libcpp = libcpp
    import importlib

    mods = {}
    for name in ("timing", "ffautils", "libffa", "running_medians", "time_series", "search",
                 "clustering", "peak_detection", "folding", "reading.presto", "reading.sigproc",
                 "metadata"):
        mods[name] = importlib.import_module("riptide." + name)
    mods["periodogram"] = importlib.import_module("riptide.periodogram")
    return libcpp, mods


class _CallRecorder(types.ModuleType):
    """Stands in for the reference's ``riptide.libcpp`` module: forwards every call to it and
    records (name, positional arguments, outputs)."""

    def __init__(self, lib):
        super().__init__("riptide.libcpp")
        self._lib = lib
        self.calls = []

    def __getattr__(self, name):
        fn = getattr(self._lib, name)

        def call(*args):
            out = fn(*args)
            self.calls.append((name, args, out if isinstance(out, tuple) else (out,)))
            return out

        return call


def make_dropin():
    """dropin_trace.npz: every libcpp call that the reference's own glue makes -- ffa_search
    (search.py:11-93, with TimeSeries.deredden / normalise and fast_running_median),
    libffa.ffa2 / boxcar_snr / downsample and TimeSeries.downsample -- on seeded inputs,
    with its arguments and the reference libcpp's outputs, plus the glue's final outputs.
    Replaying the calls against riptide_b200.libcpp shows that the reference's glue, with
    riptide.libcpp bound to riptide_b200.libcpp, receives the same values."""
    from oracle import oracle as O

    rec = _CallRecorder(O.ref_libcpp())
    _, M = import_reference(libcpp=rec)
    rng = np.random.default_rng(424242)
    ts_cls = M["time_series"].TimeSeries
    finals = {}
    cases = [(1 << 15, 1e-3, dict(period_min=0.5, period_max=5.0)),
             (40001, 5e-4, dict(period_min=0.3, period_max=3.0, bins_min=240, bins_max=260,
                                rmed_width=1.0, rmed_minpts=51)),
             (1 << 14, 1e-3, dict(period_min=0.8, period_max=2.0, deredden=False))]
    for i, (n, tsamp, kw) in enumerate(cases):
        x = M["libffa"].generate_signal(n, 0.77 / tsamp, ducy=0.03, amplitude=18.0)
        x = (x + rng.standard_normal(n) * 0.1 + 2.0).astype(np.float32)
        ts, pg = M["search"].ffa_search(ts_cls(x, tsamp), **kw)
        finals[f"final{i}_z"] = ts.data  # the periodogram is the last call's output
    y = rng.standard_normal((150, 251)).astype(np.float32)
    M["libffa"].ffa2(y)
    M["libffa"].boxcar_snr(y[:40], M["ffautils"].generate_width_trials(251), stdnoise=1.5)
    M["libffa"].downsample(rng.standard_normal(20000).astype(np.float32), 13.37)
    ts_cls(rng.standard_normal(10000).astype(np.float32), 1e-3).downsample(7.5)
    out = dict(finals, n=len(rec.calls))
    for k, (name, args, outs) in enumerate(rec.calls):
        out[f"c{k}_name"] = np.array(name)
        out[f"c{k}_nargs"] = len(args)
        out[f"c{k}_nout"] = len(outs)
        for j, a in enumerate(args):
            if isinstance(a, np.ndarray):
                out[f"c{k}_a{j}"] = a
                out[f"c{k}_t{j}"] = np.array("array")
            else:
                out[f"c{k}_a{j}"] = np.array(a)
                out[f"c{k}_t{j}"] = np.array(type(a).__name__)
        for j, o in enumerate(outs):
            out[f"c{k}_o{j}"] = o
    np.savez_compressed(os.path.join(HERE, "dropin_trace.npz"), **out)
    print("dropin_trace.npz:", [c[0] for c in rec.calls])


def main(sections=None):
    """Write the fixtures of `sections` (all when None): core, fold, readers, workerpool,
    dropin (the last in a process of its own: it imports the glue over a call recorder)."""
    if sections is not None and "dropin" in sections:
        make_dropin()
        return
    libcpp, M = import_reference()
    if sections is None or "fold" in sections:
        make_fold(M)
    if sections is None or "readers" in sections:
        make_readers(M)
    if sections is None or "workerpool" in sections:
        make_workerpool(M)
    if sections is not None and "core" not in sections:
        return
    rng = np.random.default_rng(20240531)
    out = {}

    # --- ffa2: bit-exact target -------------------------------------------------------
    shapes = [(1, 5), (2, 3), (3, 7), (4, 4), (5, 241), (7, 2), (8, 8), (9, 260), (13, 17),
              (16, 33), (31, 250), (64, 64), (100, 241), (257, 13)]
    ffa_in, ffa_out = [], []
    for m, b in shapes:
        x = rng.standard_normal((m, b)).astype(np.float32)
        ffa_in.append(x.ravel())
        ffa_out.append(libcpp.ffa2(x).ravel())
    np.savez_compressed(
        os.path.join(HERE, "ffa2.npz"), shapes=np.array(shapes, dtype=np.int64),
        inputs=np.concatenate(ffa_in), outputs=np.concatenate(ffa_out))

    # --- snr2 ----------------------------------------------------------------------------
    snr_cases = []
    for rows, cols, widths, stdnoise in [
        (50, 240, M["ffautils"].generate_width_trials(240), 1.0),
        (40, 260, M["ffautils"].generate_width_trials(240), 3.25),
        (20, 480, M["ffautils"].generate_width_trials(480), 1.0),
        (10, 64, np.arange(1, 64), 0.5),
        (5, 7, np.array([1, 2, 3, 6]), 2.0),
    ]:
        x = (rng.standard_normal((rows, cols)) * 5 + 0.5).astype(np.float32)
        w = np.asarray(widths, dtype=np.uint64)
        snr_cases.append((x, w, stdnoise, libcpp.snr2(x, w, stdnoise)))
    np.savez_compressed(
        os.path.join(HERE, "snr2.npz"),
        **{f"x{i}": c[0] for i, c in enumerate(snr_cases)},
        **{f"w{i}": c[1] for i, c in enumerate(snr_cases)},
        **{f"s{i}": np.float64(c[2]) for i, c in enumerate(snr_cases)},
        **{f"y{i}": c[3] for i, c in enumerate(snr_cases)},
        n=len(snr_cases))

    # --- downsample --------------------------------------------------------------------
    ds = {}
    x = rng.standard_normal(20011).astype(np.float32) + 0.25
    factors = [1.5, 2.0, 3.0, 7.25, 13.020833333333334, 20.833333333333332, 97.5, 1000.0,
               20011.0 / 7.0, 20011.0]
    for i, f in enumerate(factors):
        ds[f"y{i}"] = libcpp.downsample(x, f)
    np.savez_compressed(os.path.join(HERE, "downsample.npz"), x=x,
                        factors=np.array(factors), **ds, n=len(factors))

    # --- running median: bit-exact target ------------------------------------------------
    x = rng.standard_normal(3001).astype(np.float32)
    x[100:140] = 0.5  # ties
    widths = [1, 3, 5, 7, 11, 25, 37, 101, 999]
    rm = {f"y{w}": libcpp.running_median(x, w) for w in widths}
    np.savez_compressed(os.path.join(HERE, "running_median.npz"), x=x,
                        widths=np.array(widths), **rm)

    # --- periodogram on a small series (reference libcpp) --------------------------------
    x = rng.standard_normal(1 << 14).astype(np.float32)
    pg_cfgs = [
        # tsamp, pmin, pmax, bmin, bmax
        (1e-3, 0.5, 5.0, 240, 260),
        (1e-3, 0.24, 0.6, 240, 260),   # first cycle at f == 1 (no downsampling)
        (4e-4, 0.3, 3.0, 100, 120),
        (5e-4, 0.25, 9.0, 480, 520),
    ]
    pg = {}
    for i, (tsamp, pmin, pmax, bmin, bmax) in enumerate(pg_cfgs):
        w = M["ffautils"].generate_width_trials(bmin).astype(np.uint64)
        p, fb, s = libcpp.periodogram(x, tsamp, w, pmin, pmax, bmin, bmax)
        pg[f"p{i}"], pg[f"fb{i}"], pg[f"s{i}"], pg[f"w{i}"] = p, fb, s, w
    np.savez_compressed(os.path.join(HERE, "periodogram.npz"), x=x,
                        cfgs=np.array(pg_cfgs, dtype=np.float64), **pg, n=len(pg_cfgs))

    # --- ffa_search end to end through the reference's own Python glue ------------------
    TS = M["time_series"].TimeSeries
    ffa_search = M["search"].ffa_search
    fs = {}
    cases = [
        # nsamp, tsamp, period(s), amplitude, kwargs
        (1 << 15, 1e-3, 1.0, 20.0, dict(period_min=0.5, period_max=5.0, rmed_width=4.0)),
        (20000, 5e-4, 0.37, 15.0, dict(period_min=0.2, period_max=2.0, rmed_width=1.0,
                                       rmed_minpts=51)),
        (15000, 1e-3, 1.3, 12.0, dict(period_min=0.8, period_max=2.0, deredden=False)),
    ]
    for i, (nsamp, tsamp, period, amp, kw) in enumerate(cases):
        crng = np.random.default_rng(1000 + i)
        t = np.arange(nsamp) / (period / tsamp)
        kappa = np.log(2.0) / (2.0 * np.sin(np.pi * 0.03 / 2.0) ** 2)
        sig = np.exp(kappa * (np.cos(2 * np.pi * (t - 0.5)) - 1.0))
        sig *= amp / np.sqrt((sig ** 2).sum())
        data = (sig + crng.standard_normal(nsamp) + 0.3 * np.sin(np.arange(nsamp) * 2e-4)
                + 3.0).astype(np.float32)
        ts = TS(data, tsamp)
        tsdr, pgram = ffa_search(ts, **kw)
        fs[f"x{i}"] = data
        fs[f"tsamp{i}"] = np.float64(tsamp)
        fs[f"z{i}"] = tsdr.data
        fs[f"p{i}"], fs[f"fb{i}"], fs[f"s{i}"] = pgram.periods, pgram.foldbins, pgram.snrs
        fs[f"w{i}"] = np.asarray(pgram.widths)
        for k, v in kw.items():
            fs[f"kw{i}_{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "ffa_search.npz"), **fs, n=len(cases))

    # --- glue pieces: deredden / normalise / fast_running_median -------------------------
    x = (rng.standard_normal(30000) + np.linspace(0, 5, 30000)).astype(np.float32)
    g = {"x": x}
    g["norm"] = TS(x, 1e-3).normalise().data
    g["dered_w0.5_m51"] = TS(x, 1e-3).deredden(0.5, minpts=51).data
    g["dered_w4_m101"] = TS(x, 1e-3).deredden(4.0, minpts=101).data
    g["frm_w2001_m101"] = M["running_medians"].fast_running_median(x, 2001, 101)
    g["frm_w37_m41"] = M["running_medians"].fast_running_median(x, 37, 41)
    np.savez_compressed(os.path.join(HERE, "glue.npz"), **g)

    # --- find_peaks on the periodograms above and one longer search --------------------
    fp = {}
    pgrams = []
    for i, (nsamp, tsamp, period, amp, kw) in enumerate(cases):
        pgrams.append((fs[f"p{i}"], fs[f"fb{i}"], fs[f"s{i}"], fs[f"w{i}"], nsamp * tsamp))
    crng = np.random.default_rng(4242)
    nsamp, tsamp = 1 << 15, 2e-3
    t = np.arange(nsamp) * tsamp
    data = crng.standard_normal(nsamp)
    for per, amp in ((0.731, 1.2), (2.9, 0.9)):
        data += amp * np.exp(-0.5 * ((np.mod(t, per) - per / 2) / (0.01 * per)) ** 2)
    tsdr, pgram = ffa_search(TS(data.astype(np.float32), tsamp), period_min=0.5, period_max=5.0)
    pgrams.append((pgram.periods, pgram.foldbins, pgram.snrs, np.asarray(pgram.widths),
                   nsamp * tsamp))
    Pg = M["periodogram"].Periodogram
    for i, (p, fb, s, w, tobs) in enumerate(pgrams):
        pg = Pg(w, p, fb, s, metadata={"tobs": tobs, "dm": None})
        peaks, polycos = M["peak_detection"].find_peaks(pg)
        if i >= len(cases):  # the first periodograms are those of ffa_search.npz
            fp[f"p{i}"], fp[f"fb{i}"], fp[f"s{i}"], fp[f"w{i}"] = p, fb, s, w
        fp[f"tobs{i}"] = np.float64(tobs)
        fp[f"ip{i}"] = np.array([k.ip for k in peaks], dtype=np.int64)
        fp[f"iw{i}"] = np.array([k.iw for k in peaks], dtype=np.int64)
        fp[f"snr{i}"] = np.array([k.snr for k in peaks], dtype=np.float64)
        fp[f"freq{i}"] = np.array([k.freq for k in peaks], dtype=np.float64)
        fp[f"ducy{i}"] = np.array([k.ducy for k in peaks], dtype=np.float64)
        deg = max(len(v) for v in polycos.values())
        pc = np.full((len(w), deg), np.nan)
        for iw, v in polycos.items():
            pc[iw, :len(v)] = v
        fp[f"polycos{i}"] = pc
    np.savez_compressed(os.path.join(HERE, "find_peaks.npz"), **fp, n=len(pgrams),
                        n_from_ffa_search=len(cases))

    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


def make_fold(M):
    """TimeSeries.fold of the reference (folding.py:21-85) on a seeded series, for each case
    (period, bins, subints) of FOLD_CASES."""
    rng = np.random.default_rng(777)
    TS = M["time_series"].TimeSeries
    out = {}
    for s, (nsamp, tsamp) in enumerate(FOLD_SERIES):
        x = (rng.standard_normal(nsamp) + 0.5).astype(np.float32)
        out[f"x{s}"] = x
        out[f"tsamp{s}"] = np.float64(tsamp)
    for i, (s, period, bins, subints) in enumerate(FOLD_CASES):
        ts = TS(out[f"x{s}"], float(out[f"tsamp{s}"]))
        out[f"y{i}"] = np.asarray(ts.fold(period, bins, subints=subints), dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "fold.npz"), **out, n=len(FOLD_CASES))


# (series index, period s, bins, subints or None)
FOLD_SERIES = [(20000, 1e-3), (1 << 16, 64e-6)]
FOLD_CASES = [
    (0, 1.0, 100, None), (0, 1.0, 100, 2), (0, 1.0, 100, 20), (0, 1.0, 100, 1),
    (0, 1.0, 100, 3), (0, 1.0, 100, 7), (0, 0.37, 64, None), (0, 0.37, 64, 13),
    (0, 2.5, 250, 4), (0, 19.9, 128, None), (0, 0.101, 100, None), (0, 7.0, 60, 2),
    (1, 0.0731, 128, None), (1, 0.0731, 128, 16), (1, 1.9, 256, 1), (1, 0.5, 512, 3),
]


def make_readers(M):
    """Files written by riptide_b200.reading.writers, read back by the reference's own readers
    (reading/presto.py, reading/sigproc.py, TimeSeries.from_presto_inf / from_sigproc). The
    file bytes are stored so that the tests pin the writer too."""
    import json
    import tempfile
    import warnings

    from riptide_b200.reading.writers import write_presto, write_sigproc

    TS = M["time_series"].TimeSeries
    out = {}
    docs = []
    rng = np.random.default_rng(31337)
    with tempfile.TemporaryDirectory() as d:
        for i, (kind, items, data) in enumerate(_reader_cases(rng)):
            if kind == "presto":
                base = os.path.join(d, f"case{i}")
                write_presto(base, data, items)
                with warnings.catch_warnings():
                    warnings.simplefilter("ignore")
                    ts = TS.from_presto_inf(base + ".inf")
                inf = M["reading.presto"].PrestoInf(base + ".inf")
                hdr = {k: v for k, v in inf.items()}
                with open(base + ".inf", "rb") as f:
                    out[f"inf{i}"] = np.frombuffer(f.read(), dtype=np.uint8)
                with open(base + ".dat", "rb") as f:
                    out[f"dat{i}"] = np.frombuffer(f.read(), dtype=np.uint8)
            else:
                fn = os.path.join(d, f"case{i}.tim")
                write_sigproc(fn, data, items)
                ts = TS.from_sigproc(fn)
                sh = M["reading.sigproc"].SigprocHeader(fn)
                hdr = dict(sh)
                hdr["_bytesize"] = sh.bytesize
                with open(fn, "rb") as f:
                    out[f"tim{i}"] = np.frombuffer(f.read(), dtype=np.uint8)
            out[f"data{i}"] = ts.data
            out[f"in{i}"] = np.asarray(data)
            docs.append({"kind": kind, "items": items, "header": hdr, "tsamp": ts.tsamp,
                         "dm": ts.metadata.get("dm"), "tobs": ts.metadata.get("tobs")})
    out["json"] = np.frombuffer(json.dumps(docs).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "readers.npz"), **out, n=len(docs))


# The reference's pipeline test data (tests/test_pipeline.py:36-66): three DM trials of a
# 1 s pulsar, 128 s at 256 us, each generated after np.random.seed(0).
WP_TRIALS = [(0.0, 10.0, 0.05), (10.0, 20.0, 0.02), (20.0, 10.0, 0.05)]  # dm, amplitude, ducy
WP_TOBS, WP_TSAMP, WP_PERIOD = 128.0, 256e-6, 1.0
WP_DEREDDEN = {"rmed_width": 5.0, "rmed_minpts": 101}
WP_RANGES = [
    {"name": "medium", "ffa_search": {"period_min": 0.5, "period_max": 4.0, "bins_min": 480,
                                      "bins_max": 520, "fpmin": 8, "wtsp": 1.5},
     "find_peaks": {"smin": 7.0}},
    {"name": "long", "ffa_search": {"period_min": 4.0, "period_max": 120.0, "bins_min": 960,
                                    "bins_max": 1040, "fpmin": 8, "wtsp": 1.5},
     "find_peaks": {"smin": 7.0}},
]


def make_workerpool(M):
    """Peaks of the reference's WorkerPool.process_fname_list (pipeline/worker_pool.py) over
    PRESTO files of the reference's pipeline test signal, with the ranges of its test
    configuration A (tests/pipeline_config_A.yml)."""
    import importlib.util
    import tempfile

    from riptide_b200.reading.writers import write_presto

    pkg = sys.modules["riptide"]
    pkg.TimeSeries = M["time_series"].TimeSeries
    pkg.Metadata = M["metadata"].Metadata
    pkg.ffa_search = M["search"].ffa_search
    pkg.find_peaks = M["peak_detection"].find_peaks
    # the module file alone: the pipeline package's __init__ imports the whole application
    spec = importlib.util.spec_from_file_location(
        "ref_worker_pool", os.path.join(REF_ROOT, "src", "riptide", "pipeline", "worker_pool.py"))
    WP = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(WP)
    TS = M["time_series"].TimeSeries
    out = {}
    with tempfile.TemporaryDirectory() as d:
        fnames = []
        for i, (dm, amp, ducy) in enumerate(WP_TRIALS):
            np.random.seed(0)
            ts = TS.generate(WP_TOBS, WP_TSAMP, WP_PERIOD, amplitude=amp, ducy=ducy, stdnoise=1.0)
            out[f"sum{i}"] = np.float64(ts.data.astype(np.float64).sum())
            base = os.path.join(d, f"fake_DM{dm:.3f}")
            write_presto(base, ts.data, workerpool_inf(os.path.basename(base), ts.nsamp, dm))
            fnames.append(base + ".inf")
        pool = WP.WorkerPool(WP_DEREDDEN, WP_RANGES, processes=1, fmt="presto")
        # process_fname_list without its process pool: the same calls, flattened the same way
        peaks = [p for f in fnames for p in pool.process_fname(f)]
    for key in ("period", "freq", "width", "ducy", "iw", "ip", "snr", "dm"):
        out[key] = np.array([getattr(p, key) for p in peaks])
    np.savez_compressed(os.path.join(HERE, "workerpool.npz"), **out)


def workerpool_inf(basename, nsamp, dm):
    """.inf items of the pipeline test files (tests/presto_generation.py:7-28)."""
    return dict(basename=basename, telescope="Parkes", instrument="Multibeam",
                source_name="Pulsar", raj="00:00:01.0000", decj="-00:00:01.0000",
                observer="Kenji Oba", mjd=59000.0, barycentered=True, nsamp=int(nsamp),
                tsamp=WP_TSAMP, breaks=False, onoff_pairs=[], em_band="Radio", fov_arcsec=981.0,
                dm=float(dm), fbot=1182.1953125, bandwidth=400.0, nchan=1024, cbw=0.390625,
                analyst="Space Sheriff Gavan")


def _reader_cases(rng):
    radio = dict(basename="case", telescope="Parkes", instrument="Multibeam",
                 source_name="J0000+0000", raj="00:00:01.0000", decj="-00:00:01.0000",
                 observer="Nobody", mjd=59000.5, barycentered=True, nsamp=1000, tsamp=6.4e-05,
                 breaks=False, onoff_pairs=[], em_band="Radio", fov_arcsec=981.0, dm=42.42,
                 fbot=1182.1953125, bandwidth=400.0, nchan=1024, cbw=0.390625, analyst="Nobody")
    breaks = dict(radio, breaks=True, onoff_pairs=[(0, 700), (800, 999)], nsamp=1000, dm=0.0)
    xray = {k: v for k, v in radio.items()
            if k not in ("fov_arcsec", "dm", "fbot", "bandwidth", "nchan", "cbw", "analyst")}
    xray.update(em_band="X-ray", fov_arcsec=3.0, central_energy_kev=1.0,
                energy_bandpass_kev=5.0, analyst="Nobody")
    sig = dict(source_name="Fake", telescope_id=4, machine_id=10, src_raj=63642.23,
               src_dej=-454405.0, az_start=0.0, za_start=0.0, data_type=2, refdm=26.31,
               fch1=1581.8046875, barycentric=0, nchans=1, nbits=32, tstart=56771.1303125,
               tsamp=6.4e-05, nifs=1)
    u8 = dict(sig, nbits=8, signed=False, refdm=187.5)
    i8 = dict(sig, nbits=8, signed=True, refdm=3.0)
    return [
        ("presto", radio, rng.standard_normal(1000).astype(np.float32)),
        ("presto", breaks, rng.standard_normal(1000).astype(np.float32)),
        ("presto", xray, rng.poisson(3.0, 1000).astype(np.float32)),
        ("sigproc", sig, rng.standard_normal(777).astype(np.float32)),
        ("sigproc", u8, rng.integers(0, 256, 1001).astype(np.uint8)),
        ("sigproc", i8, rng.integers(-128, 128, 1003).astype(np.int8)),
    ]


if __name__ == "__main__":
    main(sys.argv[1:] or None)
