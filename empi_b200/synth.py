"""Seeded synthetic EEG-like signals for the benchmark and test workloads.

Every workload is a sum of Gabor atoms plus noise.  An atom is
``A * exp(-pi ((t - t0) / s)^2) * cos(2 pi f (t - t0) + phi)``, the waveform
empi subtracts (reference src/gabor.cpp:159-163).  Signals are float32,
sample-major with channels interleaved, the layout empi reads
(reference src/io.cpp:28-34, README.md:151-156).

Workloads (seed = 1000 + index, NumPy PCG64):
  0  SMP    1 ch x 1 epoch x 1280 @128 Hz, 5 atoms, white noise 10 dB,
            energyError 0.01, 50 iterations, energyPercent 99
  1  MMP2  19 ch x 8 epochs x 5120 @256 Hz, 20 shared atoms per epoch with
            N(0,1) channel gains and a common phase, white noise 5 dB per
            channel, energyError 0.01, 100 iterations, energyPercent 99
  2  MMP3  32 ch x 4 epochs x 16384 @512 Hz, 40 atoms per epoch with per-channel
            N(0,1) amplitude and U[0, 2pi) phase, pink noise 0 dB,
            energyError 0.005, 200 iterations
  3  SMP batch: 512 instances at 256 Hz, C ~ U{1..32}, N log-uniform in
            [512, 16384], 3-60 atoms, white noise at SNR ~ U[0, 20] dB,
            energyError 0.01, 150 iterations, energyPercent 99.5
  4  workload 2's shapes with energyError 0.001 and 300 iterations
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Workload:
    """One decomposition job: a list of epochs sharing fs and settings."""

    name: str
    variant: str            # "smp" | "mmp1" | "mmp2" | "mmp3"
    fs: float
    energy_error: float
    iterations: int
    energy_percent: float
    epochs: list            # list of float32 arrays shaped (N, C)

    @property
    def channels(self) -> int:
        return self.epochs[0].shape[1]

    @property
    def samples(self) -> int:
        return self.epochs[0].shape[0]


def gabor(n: int, fs: float, s: float, t0: float, f: float, phi: float, amp: float) -> np.ndarray:
    t = np.arange(n) / fs
    return amp * np.exp(-np.pi * ((t - t0) / s) ** 2) * np.cos(2 * np.pi * f * (t - t0) + phi)


def _atom_params(rng: np.random.Generator, n: int, fs: float, fmax: float):
    s = math.exp(rng.uniform(math.log(0.1), math.log(5.0)))
    t0 = rng.uniform(0.0, n / fs)
    f = rng.uniform(0.0, fmax)
    phi = rng.uniform(0.0, 2 * math.pi)
    amp = rng.lognormal(0.0, 1.0)
    return s, t0, f, phi, amp


def _white(rng, n, power):
    return rng.standard_normal(n) * math.sqrt(power)


def _pink(rng, n, power):
    w = rng.standard_normal(n)
    spec = np.fft.rfft(w)
    k = np.arange(spec.size, dtype=np.float64)
    k[0] = 1.0
    spec = spec / np.sqrt(k)
    spec[0] = 0.0
    x = np.fft.irfft(spec, n)
    x = x / max(np.sqrt(np.mean(x * x)), 1e-30)
    return x * math.sqrt(power)


def _with_noise(rng, sig, snr_db, pink=False):
    p = float(np.mean(sig * sig))
    noise_p = p / (10.0 ** (snr_db / 10.0)) if p > 0 else 1.0
    return sig + (_pink(rng, sig.size, noise_p) if pink else _white(rng, sig.size, noise_p))


def smp_channel(rng, n, fs, n_atoms, snr_db):
    """One config-0-style channel."""
    x = np.zeros(n)
    for _ in range(n_atoms):
        x += gabor(n, fs, *_atom_params(rng, n, fs, fs / 2))
    return _with_noise(rng, x, snr_db)


def workload(index: int, seed: int | None = None, epochs: int | None = None,
             channels: int | None = None, samples: int | None = None,
             iterations: int | None = None) -> Workload:
    """The seeded workload ``index``; optional overrides shrink it for tests."""
    rng = np.random.default_rng(1000 + index if seed is None else seed)
    if index == 0:
        fs, n, c, e = 128.0, samples or 1280, channels or 1, epochs or 1
        eps = [np.stack([smp_channel(rng, n, fs, 5, 10.0) for _ in range(c)], 1) for _ in range(e)]
        return Workload("smp-1x1x1280@128", "smp", fs, 0.01, iterations or 50, 99.0,
                        [x.astype(np.float32) for x in eps])
    if index == 1:
        fs, n, c, e = 256.0, samples or 5120, channels or 19, epochs or 8
        out = []
        for _ in range(e):
            sig = np.zeros((n, c))
            for _ in range(20):
                g = gabor(n, fs, *_atom_params(rng, n, fs, fs / 2))
                sig += g[:, None] * rng.standard_normal(c)[None, :]
            out.append(np.stack([_with_noise(rng, sig[:, k], 5.0) for k in range(c)], 1))
        return Workload("mmp2-19x8x5120@256", "mmp2", fs, 0.01, iterations or 100, 99.0,
                        [x.astype(np.float32) for x in out])
    if index in (2, 4):
        fs, n, c, e = 512.0, samples or 16384, channels or 32, epochs or 4
        out = []
        for _ in range(e):
            sig = np.zeros((n, c))
            for _ in range(40):
                s, t0, f, _, _ = _atom_params(rng, n, fs, fs / 2)
                amps = rng.standard_normal(c)
                phis = rng.uniform(0, 2 * math.pi, c)
                for k in range(c):
                    sig[:, k] += gabor(n, fs, s, t0, f, phis[k], amps[k])
            out.append(np.stack([_with_noise(rng, sig[:, k], 0.0, pink=True) for k in range(c)], 1))
        if index == 2:
            return Workload("mmp3-32x4x16384@512", "mmp3", fs, 0.005, iterations or 200, 100.0,
                            [x.astype(np.float32) for x in out])
        return Workload("mmp3-32x4x16384@512-eps0.001", "mmp3", fs, 0.001, iterations or 300, 100.0,
                        [x.astype(np.float32) for x in out])
    if index == 3:
        fs = 256.0
        count = epochs or 512
        out = []
        for _ in range(count):
            c = channels or int(rng.integers(1, 33))
            n = samples or int(round(math.exp(rng.uniform(math.log(512), math.log(16384)))))
            k = int(rng.integers(3, 61))
            snr = rng.uniform(0.0, 20.0)
            out.append(np.stack([smp_channel(rng, n, fs, k, snr) for _ in range(c)], 1).astype(np.float32))
        return Workload("smp-batch-512@256", "smp", fs, 0.01, iterations or 150, 99.5, out)
    raise ValueError(f"unknown workload {index}")
