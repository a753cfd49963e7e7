"""Differentiable search (riptide_b200.grad): the adjoint kernels against the forward ones
(dot-product identities, finite differences), and the gradient of the whole search against
FP64 finite differences of the oracle pipeline and against a pure-torch FP64 reference
gradient. Tolerances are stated per test."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import riptide_b200.grad as G

    return G


def _dot(a, b):
    return float((a.double() * b.double()).sum())


@pytest.mark.parametrize("m,b", [(1, 7), (2, 240), (3, 250), (37, 251), (108, 260), (1000, 240),
                                 (513, 487)])
def test_ffa_transpose_identity(G, m, b):
    # <FFA x, g> == <x, FFA^T g> (FFA is linear); float32 kernels, FP64 dot products
    import torch

    rng = np.random.default_rng(m * 7 + b)
    x = torch.from_numpy(rng.standard_normal((m, b)).astype(np.float32)).cuda()
    g = torch.from_numpy(rng.standard_normal((m, b)).astype(np.float32)).cuda()
    lhs = _dot(G._ffa2(x), g)
    rhs = _dot(x, G.ffa2_transpose(g))
    assert abs(lhs - rhs) <= 2e-5 * (abs(lhs) + float(x.abs().sum()) * 1e-2)


def test_ffa_transpose_is_exact_for_unit_rows(G):
    # FFA^T of a single unit output element is a set of 0/1 entries (one per input row)
    import torch

    m, b = 97, 250
    for s, c in [(0, 0), (50, 17), (96, 249)]:
        g = torch.zeros((m, b), device="cuda")
        g[s, c] = 1.0
        gt = G.ffa2_transpose(g)
        assert torch.all((gt == 0) | (gt == 1))
        assert int(gt.sum()) == m and torch.all(gt.sum(1) == 1)


@pytest.mark.parametrize("f", [1.5, 13.0, 17.3, 250.1, 4100.7])
def test_downsample_adjoint_identity(G, f):
    import torch

    import riptide_b200 as rb

    rng = np.random.default_rng(int(f * 10))
    N = 100003
    x = torch.from_numpy(rng.standard_normal(N).astype(np.float32)).cuda()
    y = rb.libcpp.downsample(x, f)
    g = torch.from_numpy(rng.standard_normal(y.numel()).astype(np.float32)).cuda()
    lhs = _dot(y, g)
    rhs = _dot(x, G.downsample_adjoint(g, N, f))
    assert abs(lhs - rhs) <= 1e-5 * float(y.abs().sum() + 1)


def test_normalise_adjoint_matches_torch(G):
    import torch

    rng = np.random.default_rng(3)
    y = torch.from_numpy(rng.standard_normal(50000) * 3 + 1.5).cuda()
    g = torch.from_numpy(rng.standard_normal(50000)).cuda()
    yy = y.clone().requires_grad_(True)
    z = (yy - yy.mean()) / torch.sqrt(((yy - yy.mean()) ** 2).mean())
    (z * g).sum().backward()
    std = float(torch.sqrt(((y - y.mean()) ** 2).mean()))
    ours = G.normalise_adjoint(g.float(), z.detach().float(), std)
    assert torch.allclose(ours.double(), yy.grad, rtol=1e-4, atol=1e-6)


@pytest.mark.parametrize("b", [240, 259])
def test_snr_backward_finite_differences(G, b):
    # S/N is piecewise linear in the profile; on profiles with one clear pulse (so that every
    # width has a unique maximising phase), FP64 central differences of the FP64 oracle along
    # a random direction equal the gradient to 1e-4 relative
    import torch

    import riptide_b200 as rb

    rng = np.random.default_rng(b)
    widths = rb.generate_width_trials(240)
    ph = np.arange(b)
    x = np.stack([8.0 * np.exp(-((ph - 30 - 37 * r) / (3.0 + r)) ** 2) +
                  0.05 * rng.standard_normal(b) for r in range(6)]).astype(np.float32)
    v = rng.standard_normal((6, b))
    gs = rng.standard_normal((6, widths.size))
    c = O.C()
    eps = 1e-6
    x64 = x.astype(np.float64)
    fd = ((c.snr2(x64 + eps * v, widths, 1.3, f64=True) -
           c.snr2(x64 - eps * v, widths, 1.3, f64=True)) * gs).sum() / (2 * eps)
    gx = G.snr2_backward(torch.from_numpy(x).cuda(), widths, 1.3,
                         torch.from_numpy(gs.astype(np.float32)).cuda())
    ad = float((gx.double().cpu().numpy() * v).sum())
    assert abs(fd - ad) <= 1e-4 * max(1.0, abs(fd)), (fd, ad)


# ------------------------------------------------------------------------------------------
# whole search
# ------------------------------------------------------------------------------------------
KW = dict(period_min=0.1, period_max=0.4, bins_min=40, bins_max=44, rmed_width=0.05,
          rmed_minpts=11)
TSAMP = 1e-3


def _series(n, seed):
    rng = np.random.default_rng(seed)
    t = np.arange(n) * TSAMP
    pulse = 6.0 * np.exp(-0.5 * ((np.mod(t, 0.213) - 0.1) / 0.004) ** 2)
    return (rng.standard_normal(n) + pulse + 0.3 * np.sin(t * 2.0)).astype(np.float32)


def _search_f64(x, transforms, widths):
    """FP64 forward of the same search: deredden (fast_running_median with an exact median),
    normalise, then per transform downsample / fold / FFA / S/N with the FP64 oracle."""
    import torch

    x = np.asarray(x, dtype=np.float64)
    ws = int(round(KW["rmed_width"] / TSAMP))
    k = int(max(1, ws / float(KW["rmed_minpts"])))
    nl = x.size // k
    lores = x[:nl * k].reshape(nl, k).mean(axis=1)
    w = KW["rmed_minpts"]
    half = w // 2
    padded = np.concatenate([np.full(half, lores[0]), lores, np.full(half, lores[-1])])
    win = np.lib.stride_tricks.sliding_window_view(padded, w)
    rm = np.median(win, axis=1)
    xl = np.arange(nl) * k + 0.5 * (k - 1)
    y = x - np.interp(np.arange(x.size), xl, rm)
    z = (y - y.mean()) / y.std()
    c = O.C()
    out = {}
    for (t, cy, b, m, re, row0, f, sn) in transforms:
        ds = z if f == 1 else c.downsample(z, f, f64=True)
        F = c.ffa2(ds[:m * b].reshape(m, b), f64=True)
        out[row0] = c.snr2(F[:re], widths, float(sn), f64=True)
    return np.concatenate([out[k] for k in sorted(out)])


def test_search_gradient_fp64_finite_differences(G):
    # loss = sum(W * snrs) with a random W on the 12 rows of highest S/N (where each width's
    # best phase is clear, so that the float32 forward and the FP64 pipeline select the same
    # phases); directional derivative of the float32 adjoint against FP64 central
    # differences of the FP64 pipeline: 2e-3 relative
    import torch

    n = 1 << 14
    x = _series(n, 5)
    ds = G.DifferentiableSearch([n], TSAMP, **KW)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    s = ds.snrs(xt)
    rng = np.random.default_rng(9)
    W = torch.zeros_like(s)
    rows = torch.argsort(s.detach().max(dim=1).values, descending=True)[:12]
    W[rows] = torch.from_numpy(rng.standard_normal((12, s.shape[1])).astype(np.float32)).cuda()
    (s * W).sum().backward()
    g = xt.grad.double().cpu().numpy()
    v = rng.standard_normal(n)
    Wn = W.double().cpu().numpy()
    eps = 1e-7  # small enough that no median or phase selection flips within the step
    fp = (Wn * _search_f64(x + eps * v, ds.transforms, ds.widths)).sum()
    fm = (Wn * _search_f64(x - eps * v, ds.transforms, ds.widths)).sum()
    fd = (fp - fm) / (2 * eps)
    ad = float(g @ v)
    assert abs(fd - ad) <= 2e-3 * max(1.0, abs(fd)), (fd, ad)
    ds.close()


def _merge_idx(n):
    mh = n >> 1
    kh = np.float32(mh - 1) / np.float32(n - 1)
    kt = np.float32(n - mh - 1) / np.float32(n - 1)
    s = np.arange(n, dtype=np.float64)
    h = (np.float64(kh) * s + 0.5).astype(np.float32).astype(np.int64)
    t = (np.float64(kt) * s + 0.5).astype(np.float32).astype(np.int64)
    return mh, h, t


def _ffa_torch(x):
    """FP64 torch FFA with the reference's recursion (transforms.hpp:13-61)."""
    import torch

    m, b = x.shape
    if m == 1:
        return x
    mh, h, t = _merge_idx(m)
    head = _ffa_torch(x[:mh])
    tail = _ffa_torch(x[mh:])
    rows = []
    for s in range(m):
        sh = int((s - t[s]) % b)
        rows.append(head[h[s]] + torch.roll(tail[t[s]], -sh))
    return torch.stack(rows)


def _snr_torch(F, widths, sn, b):
    import torch

    C = torch.cumsum(F, dim=1)
    wmax = int(max(widths))
    Ce = torch.cat([C, C[:, :wmax] + C[:, -1:]], dim=1)
    outs = []
    for w in widths:
        w = int(w)
        h = np.sqrt((b - w) / (b * w))
        be = w / (b - w) * h
        d = (Ce[:, w:w + b] - Ce[:, :b]).max(dim=1).values
        outs.append(((h + be) * d - be * C[:, -1]) / sn)
    return torch.stack(outs, dim=1)


def _search_torch(x, transforms, widths):
    import torch

    ws = int(round(KW["rmed_width"] / TSAMP))
    k = int(max(1, ws / float(KW["rmed_minpts"])))
    n = x.numel()
    nl = n // k
    lores = x[:nl * k].view(nl, k).mean(1)
    w = KW["rmed_minpts"]
    half = w // 2
    padded = torch.cat([lores[:1].expand(half), lores, lores[-1:].expand(half)])
    rm = torch.median(padded.unfold(0, w, 1), dim=1).values
    i = torch.arange(n, dtype=torch.float64, device=x.device)
    pos = (i - 0.5 * (k - 1)) / k
    j = torch.floor(pos).clamp(0, nl - 2).long()
    a = (pos - j.double()).clamp(0, 1)
    interp = rm[j] + (rm[j + 1] - rm[j]) * a
    interp = torch.where(pos < 0, rm[0].expand(n), interp)
    interp = torch.where(pos >= nl - 1, rm[-1].expand(n), interp)
    y = x - interp
    z = (y - y.mean()) / torch.sqrt(((y - y.mean()) ** 2).mean())
    out = {}
    P = torch.cat([torch.zeros(1, dtype=z.dtype, device=z.device), torch.cumsum(z, 0)])
    for (t, cy, b, m, re, row0, f, sn) in transforms:
        if f == 1:
            ds = z
        else:
            nd = int(np.floor(n / f))
            kk = np.arange(nd, dtype=np.float64)
            start = kk * f
            end = start + f
            imin = np.floor(start).astype(np.int64)
            imax = np.minimum(np.floor(end), n - 1).astype(np.int64)
            wmin = torch.from_numpy(((imin + 1) - start).astype(np.float32).astype(np.float64)).to(z.device)
            wmax = torch.from_numpy((end - imax).astype(np.float32).astype(np.float64)).to(z.device)
            imin_t = torch.from_numpy(imin).to(z.device)
            imax_t = torch.from_numpy(imax).to(z.device)
            ds = wmin * z[imin_t] + (P[imax_t] - P[imin_t + 1]) + wmax * z[imax_t]
        F = _ffa_torch(ds[:m * b].view(m, b))
        out[row0] = _snr_torch(F[:re], widths, float(sn), b)
    return torch.cat([out[k] for k in sorted(out)])


def test_search_gradient_matches_pure_torch(G):
    # full gradient vector of sum(W * snrs), W random on the rows of six transforms, against
    # torch autograd through an FP64 torch restatement of the same search: relative L2
    # difference below 2e-3
    import torch

    n = 1 << 12
    x = _series(n, 8)
    ds = G.DifferentiableSearch([n], TSAMP, **KW)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    s = ds.snrs(xt)
    rng = np.random.default_rng(4)
    picked = [ds.transforms[i] for i in rng.choice(len(ds.transforms), 6, replace=False)]
    W = torch.zeros_like(s)
    for tr in picked:
        r0, re = tr[5], tr[4]
        W[r0:r0 + re] = torch.from_numpy(rng.standard_normal((re, s.shape[1])).astype(np.float32)).cuda()
    (s * W).sum().backward()
    ours = xt.grad.double()
    x64 = torch.from_numpy(x.astype(np.float64)).cuda().requires_grad_(True)
    ref = _search_torch(x64, picked, ds.widths)
    Wp = torch.cat([W[tr[5]:tr[5] + tr[4]] for tr in sorted(picked, key=lambda t: t[5])])
    (ref * Wp.double()).sum().backward()
    err = float((ours - x64.grad).norm() / x64.grad.norm())
    assert err < 2e-3, err
    ds.close()


def test_search_gradient_batched_trials(G):
    # the trials of a batch are independent: the gradient of a batch loss restricted to one
    # trial equals the gradient of that trial searched alone
    import torch

    lens = [1 << 13, 9000, 1 << 13]
    xs = [_series(n, 20 + i) for i, n in enumerate(lens)]
    dsb = G.DifferentiableSearch(lens, TSAMP, **KW)
    xb = torch.from_numpy(np.concatenate(xs)).cuda().requires_grad_(True)
    dsb.snrs(xb)[:, 3].sum().backward()
    for i, x in enumerate(xs):
        d1 = G.DifferentiableSearch([x.size], TSAMP, **KW)
        x1 = torch.from_numpy(x).cuda().requires_grad_(True)
        d1.snrs(x1)[:, 3].sum().backward()
        a, e = int(dsb.offsets[i]), int(dsb.offsets[i + 1])
        assert torch.allclose(x1.grad, xb.grad[a:e], rtol=1e-5, atol=1e-6)
        d1.close()
    dsb.close()


def test_sparse_row_backward_matches_per_transform(G):
    # the batched sparse-row backward (rows recomputed from the run's downsampled series)
    # and the per-transform path (FFA outputs recomputed with rt_ffa2) give the same gradient
    # with respect to the searched series, to float32 rounding (1e-4 relative L2)
    import torch

    lens = [1 << 13, 9000, 1 << 13]
    x = torch.from_numpy(np.concatenate([_series(n, 40 + i) for i, n in enumerate(lens)])).cuda()
    ds = G.DifferentiableSearch(lens, TSAMP, **KW)
    (p, fb, s), (z, std, run) = ds.forward(x, keep=True)
    rng = np.random.default_rng(2)
    g = torch.zeros_like(s)
    rows = rng.choice(s.shape[0], 40, replace=False)
    g[rows] = torch.from_numpy(rng.standard_normal((40, s.shape[1])).astype(np.float32)).cuda()
    from riptide_b200 import _lib, libcpp

    gz = torch.empty_like(x)
    _lib.check(_lib.load().rt_search_backward_rows(ds.bs._plan, libcpp._ptr(z), libcpp._ptr(g),
                                                   libcpp._ptr(gz), 1 << 16, libcpp._stream()))
    ref = ds._gz_per_transform(x, g, z)
    err = float((gz - ref).norm() / ref.norm())
    assert err < 1e-4, err
    # more rows than allowed: a clear error, nothing written past the limit
    with pytest.raises(ValueError):
        _lib.check(_lib.load().rt_search_backward_rows(ds.bs._plan, libcpp._ptr(z),
                                                       libcpp._ptr(g), libcpp._ptr(gz), 8,
                                                       libcpp._stream()))
    ds.close()
