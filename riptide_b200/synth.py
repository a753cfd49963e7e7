"""Seeded synthetic DM-trial workloads (no survey data is available offline).

Each series: white N(0, 1) noise, optionally a 1/f ("red") component scaled to a given rms
(spectral shaping of white noise in the Fourier domain, DC removed), a 50 Hz sinusoid, and
von Mises pulse trains whose `amplitude` is the expected folded S/N (the reference's
generate_signal convention, libffa.py:15-68). Generated with torch on the requested device;
trial i of a configuration uses the seed config_id * 100000 + i, so every consumer (GPU
search, CPU baseline, tests) can regenerate exactly the same arrays.
"""
import math

import numpy as np

CONFIGS = {
    # id: (description, lengths rule, tsamp, search kwargs)
    1: dict(name="c1 single 2^20 samp, 100 us, P 0.5-5 s, b240-260", tsamp=1e-4,
            search=dict(period_min=0.5, period_max=5.0, bins_min=240, bins_max=260,
                        ducy_max=0.2, wtsp=1.5, rmed_width=4.0, rmed_minpts=101)),
    2: dict(name="c2 single 2^23 samp, 64 us, P 0.2-60 s, b240-260", tsamp=64e-6,
            search=dict(period_min=0.2, period_max=60.0, bins_min=240, bins_max=260,
                        ducy_max=0.2, wtsp=1.5, rmed_width=4.0, rmed_minpts=101)),
    3: dict(name="c3 batched 512 x U[0.9, 1.0]*2^22 samp, 64 us, P 0.2-30 s, b240-260",
            tsamp=64e-6,
            search=dict(period_min=0.2, period_max=30.0, bins_min=240, bins_max=260,
                        ducy_max=0.2, wtsp=1.5, rmed_width=4.0, rmed_minpts=101)),
    4: dict(name="c4 differentiable 64 x 2^20 samp, 100 us, P 0.5-5 s, b240-260, 257-tap FIR",
            tsamp=1e-4,
            search=dict(period_min=0.5, period_max=5.0, bins_min=240, bins_max=260,
                        ducy_max=0.2, wtsp=1.5, rmed_width=4.0, rmed_minpts=101)),
    5: dict(name="c5 batched 1024 x U[0.85, 1.0]*2^23 samp, 64 us, P 0.2-60 s, b480-520",
            tsamp=64e-6,
            search=dict(period_min=0.2, period_max=60.0, bins_min=480, bins_max=520,
                        ducy_max=0.2, wtsp=1.5, rmed_width=4.0, rmed_minpts=101)),
}


def trial_seed(config_id, index):
    return int(config_id) * 100000 + int(index)


def trial_lengths(config_id, ntrials, first_index=0):
    """Per-trial lengths (uniform in the configured range, seeded)."""
    out = []
    for i in range(first_index, first_index + ntrials):
        rng = np.random.default_rng(trial_seed(config_id, i) + 7919)
        if config_id in (1, 4):
            out.append(1 << 20)
        elif config_id == 2:
            out.append(1 << 23)
        elif config_id == 3:
            out.append(int(rng.integers(int(0.9 * (1 << 22)), (1 << 22) + 1)))
        elif config_id == 5:
            out.append(int(rng.integers(int(0.85 * (1 << 23)), (1 << 23) + 1)))
        else:
            raise ValueError(config_id)
    return out


def _pulse(torch, n, period_samples, ducy, amplitude, phi0, device):
    kappa = math.log(2.0) / (2.0 * math.sin(math.pi * ducy / 2.0) ** 2)
    t = torch.arange(n, dtype=torch.float64, device=device)
    ph = (t / period_samples - phi0) * (2 * math.pi)
    sig = torch.exp(kappa * (torch.cos(ph) - 1.0))
    return sig * (amplitude / torch.sqrt((sig * sig).sum()))


def _red(torch, n, rms, gen, device):
    # shaped on the next power-of-two length (one FFT size for every trial), then cut to n
    nf = 1 << max(0, (n - 1).bit_length())
    w = torch.randn(nf, generator=gen, device=device, dtype=torch.float32)
    X = torch.fft.rfft(w)
    f = torch.arange(X.numel(), device=device, dtype=torch.float32)
    f[0] = 1.0
    X = X / torch.sqrt(f)
    X[0] = 0
    r = torch.fft.irfft(X, n=nf)[:n]
    return r * (rms / r.std())


def make_trial(config_id, index, n, tsamp, device="cuda"):
    """One seeded series (torch float32 tensor on `device`) and a dict describing it."""
    import torch

    seed = trial_seed(config_id, index)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    rng = np.random.default_rng(seed)
    x = torch.randn(n, generator=gen, device=device, dtype=torch.float32).double()
    info = {"seed": seed, "pulsars": []}
    if config_id in (2, 3, 5):
        x += _red(torch, n, 0.5, gen, device).double()
    if config_id == 5 and rng.random() < 0.10:
        t = torch.arange(n, device=device, dtype=torch.float64) * tsamp
        x += 0.5 * torch.sin(2 * math.pi * 50.0 * t + rng.random() * 2 * math.pi)
        info["sinusoid_hz"] = 50.0
    pulsars = []
    if config_id == 1:
        pulsars = [(1.0, 0.02, 20.0)]
    elif config_id == 2:
        pulsars = [(0.25, 0.01, 8.0 + 17.0 * rng.random()), (3.7, 0.04, 8.0 + 17.0 * rng.random()),
                   (41.0, 0.08, 8.0 + 17.0 * rng.random())]
    elif config_id == 4 and index % 2 == 0:  # half the series carry a pulsar
        pulsars = [(math.exp(rng.uniform(math.log(0.5), math.log(5.0))),
                    rng.uniform(0.01, 0.05), rng.uniform(8.0, 20.0))]
    elif config_id == 3 and rng.random() < 0.30:
        pulsars = [(math.exp(rng.uniform(math.log(0.2), math.log(30.0))),
                    rng.uniform(0.005, 0.10), rng.uniform(6.0, 30.0))]
    elif config_id == 5 and rng.random() < 0.20:
        pulsars = [(math.exp(rng.uniform(math.log(0.2), math.log(60.0))),
                    rng.uniform(0.005, 0.10), rng.uniform(6.0, 30.0))]
    for period, ducy, amp in pulsars:
        x += _pulse(torch, n, period / tsamp, ducy, amp, rng.random(), device)
        info["pulsars"].append({"period": period, "ducy": ducy, "snr": amp})
    return x.float(), info


def make_batch(config_id, ntrials, first_index=0, device="cuda"):
    """Packed float32 tensor of `ntrials` series, their lengths and descriptions."""
    import torch

    cfg = CONFIGS[config_id]
    lengths = trial_lengths(config_id, ntrials, first_index)
    total = int(sum(lengths))
    out = torch.empty(total, dtype=torch.float32, device=device)
    infos, off = [], 0
    for k, n in enumerate(lengths):
        x, info = make_trial(config_id, first_index + k, n, cfg["tsamp"], device)
        out[off:off + n] = x
        infos.append(info)
        off += n
    return out, lengths, infos
