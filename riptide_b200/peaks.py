"""Peak detection in periodograms (peak_detection.py:38-240 and clustering.py:4-48 of the
reference), for one periodogram or a whole batch on the device.

Per periodogram and width trial, the reference fits a dynamic S/N threshold: the frequency
range is cut into segments of segwidth / T_obs Hz, each segment gives a control point
(median frequency, median S/N + nstd * IQR / 1.349), a degree-`polydeg` polynomial in log f is
fitted to the control points (a constant `smin` below `minseg` segments), and the points
above both the threshold and `smin` are clustered in frequency (radius clrad / T_obs), one
peak per cluster at its highest S/N.

Here the segment statistics (sorts of every segment's S/N and frequencies) and the
thresholding of every periodogram point run on the GPU (rt_peak_segments, rt_peak_select);
the polynomial fits (np.polyfit, a few hundred points each) and the clustering of the
selected points run on the host with the reference's numpy calls, so that the peaks are the
ones the reference finds.
"""
import ctypes
import os
import typing
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _lib, libcpp

try:  # the LAPACK least-squares gufunc behind np.linalg.lstsq (numpy >= 1.x and 2.x)
    from numpy.linalg import _umath_linalg as _ulinalg
except ImportError:  # pragma: no cover
    _ulinalg = None

_POOL = None


def _pool():
    global _POOL
    if _POOL is None:
        _POOL = ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1)))
    return _POOL


_STACKED_OK = None


def _stacked_ok():
    """Whether the stacked LAPACK call reproduces np.polyfit on this numpy. The gufunc is
    private to numpy (its name and signature "ddd->ddid" may change between releases), so it
    is checked once, on a fixed problem, against np.polyfit itself; if it is missing, raises
    or differs in any bit, every fit goes through np.polyfit."""
    global _STACKED_OK
    if _STACKED_OK is None:
        ok = _ulinalg is not None
        if ok:
            try:
                x = np.array([[-0.7, -0.2, 0.1, 0.4, 0.9, 1.3, 2.2], [0.0, 0.5, 1.0, 1.5, 2.0, 2.5, 3.0]])
                y = np.array([[1.0, 2.5, 0.3, 4.0, 3.3, -1.2, 0.7], [3.0, 1.0, 4.0, 1.0, 5.0, 9.0, 2.0]])
                c = _polyfit_lapack(x, y, 2)
                ok = all(np.array_equal(c[k], np.polyfit(x[k], y[k], 2)) for k in range(2))
            except Exception:
                ok = False
        _STACKED_OK = ok
    return _STACKED_OK


def _polyfit_stacked(X, Y, deg):
    """np.polyfit(X[k], Y[k], deg) for every row k of X, Y (K x M), in one stacked call of the
    LAPACK least-squares routine np.polyfit uses: the same Vandermonde matrix, column scaling,
    rcond and driver call per problem, so every coefficient is the one np.polyfit returns.
    Large stacks are split over threads (the gufunc runs without the GIL). Falls back to one
    np.polyfit per row where the stacked call is unavailable (_stacked_ok)."""
    K, M = X.shape
    order = int(deg) + 1
    if not _stacked_ok():
        return np.array([np.polyfit(X[k], Y[k], deg) for k in range(K)]).reshape(K, order)
    return _polyfit_lapack(X, Y, deg)


def _polyfit_lapack(X, Y, deg):
    K, M = X.shape
    order = int(deg) + 1
    lhs = np.empty((K, M, order))
    tmp = lhs[:, :, ::-1]  # np.vander: powers by repeated multiplication
    tmp[:, :, 0] = 1
    if order > 1:
        tmp[:, :, 1:] = (X + 0.0)[:, :, None]
        np.multiply.accumulate(tmp[:, :, 1:], out=tmp[:, :, 1:], axis=2)
    scale = np.sqrt((lhs * lhs).sum(axis=1))
    lhs /= scale[:, None, :]
    rhs = (Y + 0.0)[:, :, None]
    rcond = M * np.finfo(np.float64).eps

    def solve(sl):
        with np.errstate(invalid="ignore", over="ignore", divide="ignore", under="ignore"):
            return _ulinalg.lstsq(lhs[sl], rhs[sl], rcond, signature="ddd->ddid")[0]

    if K >= 512:
        parts = [slice(a, min(K, a + 256)) for a in range(0, K, 256)]
        c = np.concatenate(list(_pool().map(solve, parts)))
    else:
        c = solve(slice(0, K))
    return c[:, :, 0] / scale


class Peak(typing.NamedTuple):
    """A peak of a periodogram (peak_detection.py:14-35)."""

    period: float
    freq: float
    width: int
    ducy: float
    iw: int
    ip: int
    snr: float
    dm: float

    def summary_dict(self):
        attrs = ("period", "freq", "dm", "width", "ducy", "snr")
        return {a: getattr(self, a) for a in attrs}


def _cluster1d(x, r):
    """Friends-of-friends clusters of 1D points within r (clustering.py:4-48)."""
    if not len(x):
        return []
    indices = x.argsort()
    ibreaks = np.where(abs(np.diff(x[indices])) > r)[0]
    if not len(ibreaks):
        return [indices]
    ibounds = np.concatenate(([0], ibreaks + 1, [len(x)]))
    return [indices[a:b] for a, b in zip(ibounds[:-1], ibounds[1:])]


def find_peaks_batched(periods, foldbins, snrs, row_offsets, tobs, widths, dms=None,
                       smin=6.0, segwidth=5.0, nstd=6.0, minseg=10, polydeg=2, clrad=0.1,
                       capacity=1 << 22):
    """Peaks of a batch of periodograms packed by trial (as BatchedSearch.run returns them:
    CUDA tensors periods f64[L], foldbins i32[L], snrs f32[L, nw]; row_offsets[T + 1]).
    `tobs`: per-trial observation time (s). Returns a list, per trial, of (peaks, polycos)
    as find_peaks returns them."""
    torch = libcpp._t()
    lib = _lib.load()
    st = libcpp._stream()
    rows = np.ascontiguousarray(np.asarray(row_offsets, dtype=np.uint64))
    T = rows.size - 1
    nw = int(np.asarray(widths).size)
    tob = np.ascontiguousarray(np.asarray(tobs, dtype=np.float64).reshape(T))
    dms = [None] * T if dms is None else list(dms)
    p = periods.contiguous()
    s = snrs.contiguous()
    rp = rows.ctypes.data_as(_lib._u64p)
    segoff = np.zeros(T + 1, dtype=np.uint64)
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(lib.rt_peak_segments(libcpp._ptr(p), None, nw, rp, T, tob.ctypes.data_as(dp),
                                    float(segwidth), float(nstd),
                                    segoff.ctypes.data_as(_lib._u64p), None, None, st))
    nseg = int(segoff[-1])
    fc = torch.empty(nseg, dtype=torch.float64, device=p.device)
    sc = torch.empty((nseg, nw), dtype=torch.float64, device=p.device)
    _lib.check(lib.rt_peak_segments(libcpp._ptr(p), libcpp._ptr(s), nw, rp, T,
                                    tob.ctypes.data_as(dp), float(segwidth), float(nstd),
                                    segoff.ctypes.data_as(_lib._u64p), libcpp._ptr(fc),
                                    libcpp._ptr(sc), st))
    fc_h, sc_h = fc.cpu().numpy(), sc.cpu().numpy()
    # threshold polynomials (fit_threshold, peak_detection.py:89-109), one fit per width:
    # the fits of all trials with the same number of segments and all their widths in one
    # stacked least-squares call
    ncoef = int(polydeg) + 1
    coef = np.zeros((T, nw, ncoef), dtype=np.float64)
    polycos = [dict() for _ in range(T)]
    nseg_t = np.diff(segoff.astype(np.int64))
    by_nseg = {}
    for t in range(T):
        if nseg_t[t] >= minseg:
            by_nseg.setdefault(int(nseg_t[t]), []).append(t)
        else:
            for iw in range(nw):
                polycos[t][iw] = [smin]
                coef[t, iw, ncoef - 1] = smin
    for M, ts in by_nseg.items():
        X = np.stack([np.log(fc_h[int(segoff[t]):int(segoff[t + 1])]) for t in ts])
        Y = np.stack([sc_h[int(segoff[t]):int(segoff[t + 1])].T for t in ts]).reshape(-1, M)
        C = _polyfit_stacked(np.repeat(X, nw, axis=0), Y, polydeg)
        # np.poly1d(c).coefficients: leading zeros trimmed, [0.] when all are zero
        lead = np.argmax(C != 0, axis=1)
        lead[~(C != 0).any(axis=1)] = ncoef - 1
        coef[ts] = C.reshape(len(ts), nw, ncoef)
        for j, t in enumerate(ts):
            for iw in range(nw):
                polycos[t][iw] = C[j * nw + iw, lead[j * nw + iw]:]
    dcoef = torch.from_numpy(coef).to(p.device)
    sel = torch.empty(capacity, dtype=torch.int64, device=p.device)
    count = ctypes.c_size_t(0)
    _lib.check(lib.rt_peak_select(libcpp._ptr(p), libcpp._ptr(s), nw, rp, T, libcpp._ptr(dcoef),
                                  ncoef, float(smin), libcpp._ptr(sel), capacity,
                                  ctypes.byref(count), st))
    e = torch.sort(sel[:count.value]).values
    r = e // nw
    iws = (e - r * nw).cpu().numpy()
    rows_sel = r.cpu().numpy()
    f_sel = (1.0 / p[r]).cpu().numpy()
    s_sel = s.view(-1)[e].double().cpu().numpy()
    fb_sel = foldbins[r].cpu().numpy()
    trial = np.searchsorted(rows[1:].astype(np.int64), rows_sel, side="right")
    w = np.asarray(widths)
    # group the selected points by (trial, width), rows ascending within a group (the order
    # np.where gives the reference)
    gkey = trial.astype(np.int64) * nw + iws
    order = np.lexsort((rows_sel, gkey))
    gk = gkey[order]
    bounds = np.flatnonzero(np.diff(gk)) + 1
    starts = np.concatenate([[0], bounds]) if gk.size else np.zeros(0, np.int64)
    ends = np.concatenate([bounds, [gk.size]]) if gk.size else np.zeros(0, np.int64)
    per_trial = [[] for _ in range(T)]
    for a, b in zip(starts, ends):
        sl = order[a:b]
        t, iw = int(gk[a] // nw), int(gk[a] % nw)
        ix_all = rows_sel[sl] - int(rows[t])
        fsel, ssel, fbsel = f_sel[sl], s_sel[sl], fb_sel[sl]
        for cl in _cluster1d(fsel, clrad / tob[t]):
            k = cl[ssel[cl].argmax()]
            pf = float(fsel[k])
            per_trial[t].append(Peak(period=float(1.0 / pf), freq=pf, width=int(w[iw]),
                                     ducy=float(float(w[iw]) / fbsel[k]), iw=iw,
                                     ip=int(ix_all[k]), snr=float(ssel[k]), dm=dms[t]))
    # groups come in width order within a trial, as the reference's loop over widths
    return [(sorted(per_trial[t], key=lambda q: q.snr, reverse=True), polycos[t])
            for t in range(T)]


def find_peaks(pgram, smin=6.0, segwidth=5.0, nstd=6.0, minseg=10, polydeg=2, clrad=0.1):
    """Peaks of one Periodogram, as the reference's find_peaks (peak_detection.py:149-240)
    returns them: (list of Peak sorted by decreasing S/N, {iw: polynomial coefficients})."""
    torch = libcpp._t()
    dev = torch.device("cuda")

    def on_dev(a, dtype):
        if libcpp._is_cuda_tensor(a):
            return a.to(dtype)
        return torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dtype)

    p = on_dev(pgram.periods, torch.float64)
    fb = on_dev(np.asarray(pgram.foldbins).astype(np.int64) if not libcpp._is_cuda_tensor(pgram.foldbins)
                else pgram.foldbins, torch.int64)
    s = on_dev(pgram.snrs, torch.float32)
    dm = pgram.metadata.get("dm") if isinstance(pgram.metadata, dict) else None
    res = find_peaks_batched(p, fb, s, [0, p.numel()], [pgram.tobs], pgram.widths, dms=[dm],
                             smin=smin, segwidth=segwidth, nstd=nstd, minseg=minseg,
                             polydeg=polydeg, clrad=clrad)
    return res[0]
