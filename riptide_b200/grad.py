"""Differentiable search: gradients of a loss of the periodogram with respect to the
searched series, so that a front end (for instance a whitening FIR filter) can be trained on
the search's own S/N.

The forward is the batched engine (BatchedSearch). The backward recomputes what it needs
instead of storing the FFA outputs of every transform: for each transform whose periodogram
rows carry a gradient it downsamples the normalised series again, folds it, runs the FFA
(rt_ffa2) and applies the adjoint kernels of the C ABI in reverse order:

    boxcar S/N   rt_snr2_backward    (max over phases routed to its first maximising phase)
    FFA          rt_ffa2_transpose   (the transposed butterfly)
    fold         the rows x bins block is the first rows * bins samples
    downsample   rt_downsample_adjoint
    normalise    rt_normalise_adjoint
    deredden     y = x - fast_running_median(x): the running median's own gradient, through
                 np.interp, the exact median (to its selected element) and the scrunch mean

A gradient that reaches few periodogram rows (a max-S/N loss reaches one row per trial)
costs a handful of transforms; the cost grows with the number of transforms touched.
"""
import ctypes

import numpy as np

from . import _lib, libcpp
from .batched import BatchedSearch


def _transforms(bs):
    n = bs.stats["num_transforms"]
    arr = (_lib.SearchTransform * n)()
    _lib.check(_lib.load().rt_search_plan_transforms(bs._plan, ctypes.cast(arr, ctypes.c_void_p)))
    return [(t.trial, t.cycle, t.bins, t.rows, t.rows_eval, t.out_row, t.factor, t.stdnoise)
            for t in arr]


def _ffa2(x):
    torch = libcpp._t()
    out = torch.empty_like(x)
    _lib.check(_lib.load().rt_ffa2(libcpp._ptr(x), x.shape[0], x.shape[1], libcpp._ptr(out),
                                   libcpp._stream()))
    return out


def snr2_backward(profiles, widths, stdnoise, gsnr):
    """Gradient with respect to `profiles` (CUDA (rows, bins)) of sum(gsnr * snr2(...))."""
    torch = libcpp._t()
    w, wp = _lib.u64_array(widths)
    p = profiles.contiguous()
    g = gsnr.contiguous().float()
    out = torch.empty_like(p)
    _lib.check(_lib.load().rt_snr2_backward(libcpp._ptr(p), p.shape[0], p.shape[1], wp, w.size,
                                            float(stdnoise), libcpp._ptr(g), libcpp._ptr(out),
                                            libcpp._stream()))
    return out


def ffa2_transpose(gout):
    """FFA^T applied to a CUDA (rows, bins) gradient."""
    torch = libcpp._t()
    g = gout.contiguous()
    out = torch.empty_like(g)
    _lib.check(_lib.load().rt_ffa2_transpose(libcpp._ptr(g), g.shape[0], g.shape[1],
                                             libcpp._ptr(out), libcpp._stream()))
    return out


def downsample_adjoint(gout, size, f, gin=None):
    """Adds downsample^T(gout) (factor f, input length `size`) into gin (new if None)."""
    torch = libcpp._t()
    if gin is None:
        gin = torch.zeros(size, dtype=torch.float32, device=gout.device)
    _lib.check(_lib.load().rt_downsample_adjoint(libcpp._ptr(gout.contiguous()), size, float(f),
                                                 libcpp._ptr(gin), libcpp._stream()))
    return gin


def normalise_adjoint(g, z, std):
    torch = libcpp._t()
    out = torch.empty_like(g)
    _lib.check(_lib.load().rt_normalise_adjoint(libcpp._ptr(g.contiguous()), libcpp._ptr(z), g.numel(),
                                                float(std), libcpp._ptr(out), libcpp._stream()))
    return out


def _rmed_adjoint(x, g, width_samples, min_points):
    """(fast_running_median)^T g for series x, one per row of a 2D x (running_medians.py:
    49-85): the gradient that the subtracted running median takes away, through np.interp,
    the exact median of each window (to the element it selects, edge-padded windows) and the
    scrunch mean."""
    torch = libcpp._t()
    one = x.dim() == 1
    if one:
        x, g = x.view(1, -1), g.view(1, -1)
    T, N = x.shape
    dev = x.device
    k = int(max(1, width_samples / float(min_points)))
    w = width_samples if k == 1 else min_points
    if k == 1:
        lores = x.double()
        glo = g.double()
        nl = N
    else:
        nl = N // k
        lores = x[:, :nl * k].reshape(T, nl, k).double().mean(2)
        # np.interp^T from x_lores = j k + (k - 1) / 2 back to every sample
        i = torch.arange(N, device=dev, dtype=torch.float64)
        pos = (i - 0.5 * (k - 1)) / k
        j = torch.floor(pos).clamp(0, nl - 1).long()
        a = (pos - j.double()).clamp(0.0, 1.0)
        a = torch.where(pos < 0, torch.zeros_like(a), a)
        a = torch.where(pos >= nl - 1, torch.zeros_like(a), a)
        j = torch.where(pos >= nl - 1, torch.full_like(j, nl - 1), j)
        gd = g.double()
        rows = (torch.arange(T, device=dev) * nl).view(T, 1)
        glo = torch.zeros(T * nl, dtype=torch.float64, device=dev)
        glo.index_add_(0, (rows + j).view(-1), (gd * (1.0 - a)).view(-1))
        glo.index_add_(0, (rows + (j + 1).clamp(max=nl - 1)).view(-1), (gd * a).view(-1))
        glo = glo.view(T, nl)
    half = w // 2
    padded = torch.cat([lores[:, :1].expand(T, half), lores, lores[:, -1:].expand(T, half)], 1)
    win = padded.unfold(1, w, 1)  # (T, nl, w)
    sel = torch.median(win, dim=2).indices + torch.arange(nl, device=dev) - half
    sel = sel.clamp(0, nl - 1) + (torch.arange(T, device=dev) * nl).view(T, 1)
    gsel = torch.zeros(T * nl, dtype=torch.float64, device=dev)
    gsel.index_add_(0, sel.view(-1), glo.reshape(-1))
    gsel = gsel.view(T, nl)
    if k == 1:
        out = gsel.float()
    else:
        out = torch.zeros((T, N), dtype=torch.float64, device=dev)
        out[:, :nl * k] = (gsel / k).repeat_interleave(k, dim=1)
        out = out.float()
    return out.view(-1) if one else out


class DifferentiableSearch(object):
    """ffa_search over a batch of series (lengths fixed at construction), differentiable with
    respect to the packed input. ``snrs(x)`` returns the packed periodogram S/N (rows x
    widths) as a tensor with autograd support; periods and fold bins do not depend on x."""

    def __init__(self, lengths, tsamp, period_min=1.0, period_max=30.0, bins_min=240,
                 bins_max=260, ducy_max=0.20, wtsp=1.5, deredden=True, rmed_width=4.0,
                 rmed_minpts=101, already_normalised=False):
        self.kw = dict(period_min=period_min, period_max=period_max, bins_min=bins_min,
                       bins_max=bins_max, ducy_max=ducy_max, wtsp=wtsp, deredden=deredden,
                       rmed_width=rmed_width, rmed_minpts=rmed_minpts,
                       already_normalised=already_normalised)
        self.bs = BatchedSearch(lengths, tsamp, **self.kw)
        self.tsamp = float(tsamp)
        self.widths = self.bs.widths
        self.lengths = self.bs.lengths.astype(np.int64)
        self.offsets = self.bs.sample_offsets
        self.row_offsets = self.bs.row_offsets
        self.transforms = _transforms(self.bs)
        self.deredden = bool(deredden)
        self.normalise = not bool(already_normalised)
        self.rmed_width_samples = int(round(rmed_width / self.tsamp))
        self.rmed_minpts = int(rmed_minpts)

    def forward(self, x, keep=False):
        """(periods, foldbins, snrs) of the packed CUDA float32 series x (no autograd). With
        keep, also (z, std): the searched (dereddened, normalised) series and the per-trial
        standard deviation it was normalised by, which the backward uses."""
        torch = libcpp._t()
        outs = self.bs.allocate_outputs(x.device)
        z = torch.empty_like(x) if keep else None
        outs = self.bs.run(x.detach().contiguous(), outs, normalised=z)
        self._runs = getattr(self, "_runs", 0) + 1
        if not keep:
            return outs
        T = self.bs.num_trials
        mean = (ctypes.c_double * T)()
        std = (ctypes.c_double * T)()
        _lib.check(_lib.load().rt_search_normalisation(self.bs._plan, mean, std, libcpp._stream()))
        return outs, (z, np.array(std[:], dtype=np.float64), self._runs)

    def snrs(self, x):
        return _SearchFn.apply(x, self)

    # ------------------------------------------------------------------
    # the sparse-row backward runs when at most this many periodogram rows carry a gradient
    max_sparse_rows = 1 << 16

    def backward(self, x, gsnrs, saved):
        """Gradient with respect to x of sum(gsnrs * snrs(x)); `saved` = (z, std, run) from
        forward(keep=True)."""
        torch = libcpp._t()
        z_all, stds, run = saved
        gs = gsnrs.detach().float().contiguous()
        gz_all = None
        if run == self._runs:  # the plan still holds this run's downsampled series
            gz_all = torch.empty_like(x)
            rc = _lib.load().rt_search_backward_rows(self.bs._plan, libcpp._ptr(z_all),
                                                     libcpp._ptr(gs), libcpp._ptr(gz_all),
                                                     self.max_sparse_rows, libcpp._stream())
            if rc == _lib.RT_EINVAL and b"carry a gradient" in _lib.load().rt_last_error():
                gz_all = None
            else:
                _lib.check(rc)
        if gz_all is None:
            gz_all = self._gz_per_transform(x, gs, z_all)
        return self._through_front(x, gz_all, z_all, stds)

    def _gz_per_transform(self, x, gs, z_all):
        """Gradient with respect to the searched series, one transform at a time (any number of
        rows; the FFA outputs are recomputed from the normalised series)."""
        torch = libcpp._t()
        gz_all = torch.zeros_like(x)
        live = (gs != 0).any(dim=1).cpu().numpy() if gs.numel() else np.zeros(0, bool)
        tr = self._tr_arrays()
        cs = np.concatenate([[0], np.cumsum(live)])
        hit = np.nonzero((tr[:, 4] > 0) & (cs[tr[:, 5] + tr[:, 4]] > cs[tr[:, 5]]))[0]
        groups = {}
        for i in hit:
            (t, c, b, m, re, row0, f, sn) = self.transforms[i]
            groups.setdefault((t, c), []).append((b, m, re, row0, f, sn))
        for (t, c), items in groups.items():
            a, e = int(self.offsets[t]), int(self.offsets[t + 1])
            z = z_all[a:e]
            N = e - a
            f = items[0][4]
            ds = z if f == 1 else libcpp.downsample(z, f)
            gds = torch.zeros_like(ds)
            for (b, m, re, row0, _, sn) in items:
                F = _ffa2(ds[:m * b].view(m, b))
                gF = torch.zeros_like(F)
                gF[:re] = snr2_backward(F[:re], self.widths, sn, gs[row0:row0 + re])
                gds[:m * b] += ffa2_transpose(gF).view(-1)
            if f == 1:
                gz_all[a:e] += gds
            else:
                downsample_adjoint(gds, N, f, gz_all[a:e])
        return gz_all

    def _tr_arrays(self):
        if getattr(self, "_tr", None) is None:
            self._tr = np.array([[t[0], t[1], t[2], t[3], t[4], t[5]] for t in self.transforms],
                                dtype=np.int64).reshape(-1, 6)
        return self._tr

    def _through_front(self, x, gz_all, z_all, stds):
        """From the gradient with respect to the searched series to the one with respect to x:
        normalisation, then deredden."""
        torch = libcpp._t()
        gx = torch.empty_like(x) if self.normalise else gz_all
        if self.normalise:
            for t in range(self.bs.num_trials):
                a, e = int(self.offsets[t]), int(self.offsets[t + 1])
                gx[a:e] = normalise_adjoint(gz_all[a:e], z_all[a:e], float(stds[t]))
        if self.deredden:
            gx = gx - self._rmed_adjoint_batch(x.detach(), gx)
        return gx

    def _rmed_adjoint_batch(self, x, g):
        """_rmed_adjoint over every trial: one batched call when all trials have the same
        length, one call per trial otherwise."""
        torch = libcpp._t()
        L = self.lengths
        if L.size > 1 and np.all(L == L[0]):
            n = int(L[0])
            return _rmed_adjoint(x.view(-1, n), g.view(-1, n), self.rmed_width_samples,
                                 self.rmed_minpts).view(-1)
        out = torch.empty_like(g)
        for t in range(L.size):
            a, e = int(self.offsets[t]), int(self.offsets[t + 1])
            out[a:e] = _rmed_adjoint(x[a:e], g[a:e], self.rmed_width_samples, self.rmed_minpts)
        return out

    def close(self):
        self.bs.close()


class _SearchFn(object):
    """torch.autograd.Function wrapper, created lazily (torch is imported on first use)."""
    _fn = None

    @classmethod
    def apply(cls, x, search):
        if cls._fn is None:
            import torch

            class Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, xin, s):
                    (_, _, snrs), (z, std, run) = s.forward(xin, keep=True)
                    ctx.s = s
                    ctx.std = std
                    ctx.run = run
                    ctx.save_for_backward(xin, z)
                    return snrs

                @staticmethod
                def backward(ctx, g):
                    xin, z = ctx.saved_tensors
                    return ctx.s.backward(xin, g, (z, ctx.std, ctx.run)), None

            cls._fn = Fn
        return cls._fn.apply(x, search)


def benchmark_training_step(ntrials=64, steps=3, warmup=2, taps=257):
    """One training step of the differentiable-search workload: a learnable `taps`-tap FIR
    front end on `ntrials` series of 2^20 samples (100 us; half carry a pulsar), the search,
    loss = mean max-S/N of the injected series - mean over the noise-only ones. Returns a
    dict of CUDA-event times (ms) of the forward (FIR + search + loss) and the backward."""
    import torch

    from . import synth

    cfg = synth.CONFIGS[4]
    data, lengths, infos = synth.make_batch(4, ntrials)
    n = int(lengths[0])
    inj = torch.tensor([len(i["pulsars"]) > 0 for i in infos], device=data.device)
    ds = DifferentiableSearch(lengths, cfg["tsamp"], **cfg["search"])
    h = torch.zeros(taps, device=data.device)
    h[taps // 2] = 1.0
    h.requires_grad_(True)
    rows = torch.from_numpy(ds.row_offsets).to(data.device)
    trial_of_row = torch.repeat_interleave(torch.arange(ntrials, device=data.device),
                                           rows[1:] - rows[:-1])

    # FIR front end ('same' convolution) through FFTs: the weight gradient of a long 1-channel
    # convolution is slow through the direct kernels
    L = 1 << (n + taps - 1).bit_length()
    X = torch.fft.rfft(data.view(ntrials, n), n=L)

    def fir(hh):
        y = torch.fft.irfft(X * torch.fft.rfft(hh, n=L), n=L)
        return y[:, taps // 2: taps // 2 + n].contiguous().view(-1)

    def step():
        y = fir(h)
        s = ds.snrs(y)
        best = torch.full((ntrials,), -1e30, device=data.device).scatter_reduce(
            0, trial_of_row, s.max(dim=1).values, reduce="amax")
        return best[inj].mean() - best[~inj].mean()

    def search_only():
        y = data.detach().clone().requires_grad_(True)
        s = ds.snrs(y)
        best = torch.full((ntrials,), -1e30, device=data.device).scatter_reduce(
            0, trial_of_row, s.max(dim=1).values, reduce="amax")
        return best[inj].mean() - best[~inj].mean()

    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    res = {}
    for name, fn in (("step", step), ("search", search_only)):
        fw = bw = 0.0
        for it in range(warmup + steps):
            h.grad = None
            torch.cuda.synchronize()
            e[0].record()
            loss = fn()
            e[1].record()
            (-loss).backward()
            e[2].record()
            torch.cuda.synchronize()
            if it >= warmup:
                fw += e[0].elapsed_time(e[1])
                bw += e[1].elapsed_time(e[2])
        res[name] = (fw / steps, bw / steps, float(loss.detach()),
                     float(h.grad.norm()) if h.grad is not None else None)
    ds.close()
    return {"workload": cfg["name"], "trials": ntrials,
            "step_forward_ms": res["step"][0], "step_backward_ms": res["step"][1],
            "search_forward_ms": res["search"][0], "search_backward_ms": res["search"][1],
            "search_backward_over_forward": res["search"][1] / res["search"][0],
            "loss": res["step"][2], "fir_grad_norm": res["step"][3]}


if __name__ == "__main__":
    import json
    import sys

    print(json.dumps(benchmark_training_step(*[int(a) for a in sys.argv[1:]])))
