"""Seeded synthetic extracellular recordings (stand-ins for real data).

Additive model after the reference's synthesis processor
(pyms/synthesis/p_synthesize_timeseries.py:72-89): correlated Gaussian noise
plus a low-frequency (LFP-like) component plus spikes of biphasic units.
    noise   x_t = A n_t, n_t ~ N(0, sigma^2 I), A = I + 0.3 G, G_ij ~ N(0, 1/M)
    lfp     per channel, random-phase spectrum with 1/f amplitude on
            [1, 300] Hz, scaled to the given rms
    units   biphasic 1.5 ms templates, trough depth U(50, 300), spread over
            `sites` adjacent channels with a Gaussian falloff, firing as a
            Poisson process (rate U(1, 20) Hz) with a 1.5 ms refractory period
Returned as (N, M) float32 rows (one row of M channels per timepoint).
`generate_numpy` runs on the host; `generate_torch` builds the same model on
a CUDA device for recordings too large for host generation (its random
streams differ from numpy's).
"""
from __future__ import annotations

import numpy as np


def _template(fs: float) -> np.ndarray:
    n = int(round(1.5e-3 * fs))
    t = np.arange(n) / fs
    trough = -np.exp(-((t - 0.45e-3) / 0.15e-3) ** 2)
    rebound = 0.35 * np.exp(-((t - 0.9e-3) / 0.3e-3) ** 2)
    w = trough + rebound
    return (w / -w.min()).astype(np.float64)  # trough depth 1


def _unit_params(rng, M, K, sites, fs, N):
    units = []
    for _ in range(K):
        width = int(rng.integers(sites[0], sites[1] + 1))
        width = min(width, M)
        c0 = int(rng.integers(0, max(1, M - width + 1)))
        chans = np.arange(c0, c0 + width)
        centre = c0 + (width - 1) / 2
        gains = np.exp(-0.5 * ((chans - centre) / max(1.0, width / 3)) ** 2)
        peak = rng.uniform(50, 300)
        rate = rng.uniform(1, 20)
        isi = rng.exponential(1.0 / rate, size=int(rate * N / fs * 1.5) + 10) + 1.5e-3
        times = np.cumsum(isi)
        times = (times[times < N / fs] * fs).astype(np.int64)
        units.append((chans, gains * peak, times))
    return units


def generate_numpy(M: int, N: int, fs: float = 30000.0, K: int = 20, seed: int = 0, sites=(3, 6),
                   noise_sigma: float = 10.0, lfp_rms: float = 30.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((M, M)) / np.sqrt(M)
    A = np.eye(M) + 0.3 * G
    X = (noise_sigma * rng.standard_normal((N, M)).astype(np.float32)) @ A.T.astype(np.float32)
    X = X.astype(np.float32)
    if lfp_rms > 0 and N > 2:
        f = np.fft.rfftfreq(N, 1.0 / fs)
        amp = np.where((f >= 1) & (f <= 300), 1.0 / np.maximum(f, 1.0), 0.0)
        for m in range(M):
            ph = np.exp(2j * np.pi * rng.random(len(f)))
            s = np.fft.irfft(amp * ph, N)
            r = np.sqrt(np.mean(s ** 2))
            if r > 0:
                X[:, m] += (lfp_rms * s / r).astype(np.float32)
    w = _template(fs)
    T = len(w)
    for chans, gains, times in _unit_params(rng, M, K, sites, fs, N):
        times = times[times + T <= N]
        if len(times) == 0:
            continue
        idx = times[:, None] + np.arange(T)[None, :]
        for c, g in zip(chans, gains):
            np.add.at(X[:, c], idx.ravel(), np.tile((g * w)[None, :], (len(times), 1)).ravel().astype(np.float32))
    return X


def generate_torch(M: int, N: int, fs: float = 30000.0, K: int = 300, seed: int = 0, sites=(6, 12),
                   noise_sigma: float = 10.0, lfp_rms: float = 30.0, device="cuda", chunk: int = 1 << 21):
    """Same model, built on a CUDA device in time blocks of `chunk` samples.
    Returns an (N, M) float32 tensor on `device`."""
    import torch

    rng = np.random.default_rng(seed)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    G = rng.standard_normal((M, M)) / np.sqrt(M)
    A = torch.tensor(np.eye(M) + 0.3 * G, dtype=torch.float32, device=device)
    X = torch.empty((N, M), dtype=torch.float32, device=device)
    with torch.no_grad():
        for t0 in range(0, N, chunk):
            n = min(chunk, N - t0)
            z = torch.randn((n, M), generator=g, device=device, dtype=torch.float32) * noise_sigma
            X[t0:t0 + n] = z @ A.T
        if lfp_rms > 0 and N > 2:
            f = torch.fft.rfftfreq(N, 1.0 / fs, device=device)
            amp = torch.where((f >= 1) & (f <= 300), 1.0 / torch.clamp(f, min=1.0), torch.zeros_like(f))
            nz = torch.nonzero(amp).flatten()
            lo, hi = int(nz[0]), int(nz[-1]) + 1
            for m0 in range(0, M, 16):
                m1 = min(M, m0 + 16)
                spec = torch.zeros((m1 - m0, len(f)), dtype=torch.complex64, device=device)
                ph = torch.rand((m1 - m0, hi - lo), generator=g, device=device) * (2 * np.pi)
                spec[:, lo:hi] = amp[lo:hi] * torch.exp(1j * ph)
                s = torch.fft.irfft(spec, n=N)
                s = s * (lfp_rms / torch.sqrt(torch.mean(s * s, dim=1, keepdim=True)))
                X[:, m0:m1] += s.T
                del spec, s
        w = torch.tensor(_template(fs), dtype=torch.float32, device=device)
        T = len(w)
        for chans, gains, times in _unit_params(rng, M, K, sites, fs, N):
            times = times[times + T <= N]
            if len(times) == 0:
                continue
            idx = (torch.tensor(times, device=device)[:, None] + torch.arange(T, device=device)[None, :]).flatten()
            for c, gn in zip(chans, gains):
                X[:, int(c)].index_add_(0, idx, (float(gn) * w).repeat(len(times)))
    return X
