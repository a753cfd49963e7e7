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
    """(fast_running_median)^T g for a series x (running_medians.py:49-85): the gradient that
    the subtracted running median takes away, through np.interp, the exact median of each
    window (to the element it selects, edge-padded windows) and the scrunch mean."""
    torch = libcpp._t()
    N = x.numel()
    k = int(max(1, width_samples / float(min_points)))
    w = width_samples if k == 1 else min_points
    if k == 1:
        lores = x.double()
        glo = g.double()
    else:
        nl = N // k
        lores = x[:nl * k].view(nl, k).double().mean(1)
        # np.interp^T from x_lores = j k + (k - 1) / 2 back to every sample
        i = torch.arange(N, device=x.device, dtype=torch.float64)
        pos = (i - 0.5 * (k - 1)) / k
        j = torch.floor(pos).clamp(0, nl - 1).long()
        a = (pos - j.double()).clamp(0.0, 1.0)
        a = torch.where(pos < 0, torch.zeros_like(a), a)
        a = torch.where(pos >= nl - 1, torch.zeros_like(a), a)
        j = torch.where(pos >= nl - 1, torch.full_like(j, nl - 1), j)
        gd = g.double()
        glo = torch.zeros(nl, dtype=torch.float64, device=x.device)
        glo.index_add_(0, j, gd * (1.0 - a))
        glo.index_add_(0, (j + 1).clamp(max=nl - 1), gd * a)
    n = lores.numel()
    half = w // 2
    padded = torch.cat([lores[:1].expand(half), lores, lores[-1:].expand(half)])
    win = padded.unfold(0, w, 1)  # (n, w)
    sel = torch.median(win, dim=1).indices + torch.arange(n, device=x.device) - half
    sel = sel.clamp(0, n - 1)
    gsel = torch.zeros(n, dtype=torch.float64, device=x.device)
    gsel.index_add_(0, sel, glo)
    if k == 1:
        return gsel.float()
    out = torch.zeros(N, dtype=torch.float64, device=x.device)
    out[:n * k] = (gsel / k).repeat_interleave(k)
    return out.float()


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

    def forward(self, x):
        """(periods, foldbins, snrs) of the packed CUDA float32 series x (no autograd)."""
        torch = libcpp._t()
        outs = self.bs.allocate_outputs(x.device)
        return self.bs.run(x.detach().contiguous(), outs)

    def snrs(self, x):
        return _SearchFn.apply(x, self)

    # ------------------------------------------------------------------
    def _searched(self, xt):
        """(dereddened series, normalised series, std) of one trial, as the forward searches it."""
        torch = libcpp._t()
        y = xt
        if self.deredden:
            y = torch.empty_like(xt)
            _lib.check(_lib.load().rt_deredden(libcpp._ptr(xt), xt.numel(), self.tsamp,
                                               self.kw["rmed_width"], self.rmed_minpts,
                                               libcpp._ptr(y), libcpp._stream()))
        if not self.normalise:
            return y, y, 1.0
        yd = y.double()
        m = yd.mean()
        std = float(torch.sqrt(((yd - m) ** 2).mean()))
        z = ((yd - m) / std).float()
        return y, z, std

    def backward(self, x, gsnrs):
        """Gradient with respect to x of sum(gsnrs * snrs(x))."""
        torch = libcpp._t()
        gx = torch.zeros_like(x)
        gs = gsnrs.detach().float().contiguous()
        live = (gs != 0).any(dim=1).cpu().numpy() if gs.numel() else np.zeros(0, bool)
        by_trial = {}
        for (t, c, b, m, re, row0, f, sn) in self.transforms:
            if re and live[row0:row0 + re].any():
                by_trial.setdefault(t, {}).setdefault(c, []).append((b, m, re, row0, f, sn))
        for t, cycles in by_trial.items():
            a, e = int(self.offsets[t]), int(self.offsets[t + 1])
            xt = x[a:e].detach().contiguous()
            N = e - a
            y, z, std = self._searched(xt)
            gz = torch.zeros(N, dtype=torch.float32, device=x.device)
            for c, items in cycles.items():
                f = items[0][4]
                ds = z if f == 1 else libcpp.downsample(z, f)
                gds = torch.zeros_like(ds)
                for (b, m, re, row0, _, sn) in items:
                    F = _ffa2(ds[:m * b].view(m, b))
                    gF = torch.zeros_like(F)
                    gF[:re] = snr2_backward(F[:re], self.widths, sn, gs[row0:row0 + re])
                    gds[:m * b] += ffa2_transpose(gF).view(-1)
                if f == 1:
                    gz += gds
                else:
                    downsample_adjoint(gds, N, f, gz)
            gy = normalise_adjoint(gz, z, std) if self.normalise else gz
            if self.deredden:
                gy = gy - _rmed_adjoint(xt, gy, self.rmed_width_samples, self.rmed_minpts)
            gx[a:e] = gy
        return gx

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
                    _, _, snrs = s.forward(xin)
                    ctx.s = s
                    ctx.save_for_backward(xin)
                    return snrs

                @staticmethod
                def backward(ctx, g):
                    (xin,) = ctx.saved_tensors
                    return ctx.s.backward(xin, g), None

            cls._fn = Fn
        return cls._fn.apply(x, search)
