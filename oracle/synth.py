"""Seeded synthetic laser Doppler interferograms (TEST INFRASTRUCTURE ONLY).

Stands in for recorded .holo acquisitions, of which the reference ships none.  The model:

* reference wave R = exp(i 2 pi sin(1.5 deg) x / lambda), unit amplitude, tilted along x;
* object O0: circular-Gaussian complex speckle ((N(0,1) + i N(0,1))/sqrt 2) on a centred disk,
  propagated by float64 angular spectrum over ``z_obj`` and normalised to rms 1 in the frame;
* Doppler map f_d: uniform noise -> Gaussian filter (sigma = H/16 px) -> rescaled to
  [0, f_max];
* frames O_t = O0 exp(i 2 pi f_d t / fs) (+ optional rank-2 clutter), I_t = |R + O_t|^2,
  scaled to mean 2048, Poisson shot noise, clipped to [0, 4095] (12-bit values in uint16).

Seeds follow seed = 1000 + config index + 17 * acquisition index.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

try:
    from scipy.ndimage import gaussian_filter as _gauss
except ImportError:  # pragma: no cover
    _gauss = None


@dataclass
class SynthConfig:
    height: int
    width: int
    n_frames: int
    fs: float
    disk_px: int
    z_obj: float
    lam: float = 852e-9
    pitch: float = 12e-6
    tilt_deg: float = 1.5
    f_max: float = 18e3
    scr_db: Optional[float] = None   # signal-to-clutter ratio for the rank-2 clutter (None = off)
    seed: int = 1000


def config_seed(config_index: int, acquisition: int = 0) -> int:
    return 1000 + config_index + 17 * acquisition


def _as_propagate_f64(u: np.ndarray, lam: float, pitch: float, z: float) -> np.ndarray:
    H, W = u.shape
    fx = np.fft.fftfreq(W, d=pitch)
    fy = np.fft.fftfreq(H, d=pitch)
    arg = 1.0 - (lam * fx[None, :]) ** 2 - (lam * fy[:, None]) ** 2
    kz = 2 * math.pi / lam * np.sqrt(np.maximum(arg, 0.0))
    # drop the constant 2 pi z / lambda term: a global phase
    tf = np.exp(1j * z * (kz - 2 * math.pi / lam)) * (arg > 0)
    return np.fft.ifft2(np.fft.fft2(u) * tf)


def _smooth(a: np.ndarray, sigma: float) -> np.ndarray:
    if _gauss is not None:
        return _gauss(a, sigma, mode="wrap")
    # separable FFT Gaussian (periodic) fallback
    H, W = a.shape
    gy = np.exp(-0.5 * (np.fft.fftfreq(H) * 2 * math.pi * sigma) ** 2)
    gx = np.exp(-0.5 * (np.fft.fftfreq(W) * 2 * math.pi * sigma) ** 2)
    return np.real(np.fft.ifft2(np.fft.fft2(a) * gy[:, None] * gx[None, :]))


class Interferograms:
    """Frame generator; ``frames(t0, n)`` returns uint16 [n, H, W] for absolute times t0..t0+n-1."""

    def __init__(self, cfg: SynthConfig):
        self.cfg = cfg
        rng = np.random.default_rng(cfg.seed)
        H, W = cfg.height, cfg.width
        yy, xx = np.mgrid[0:H, 0:W]
        r = np.hypot(xx - W / 2.0, yy - H / 2.0)
        disk = r <= cfg.disk_px / 2.0
        speck = (rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W))) / math.sqrt(2)
        o0 = _as_propagate_f64(speck * disk, cfg.lam, cfg.pitch, cfg.z_obj)
        o0 /= math.sqrt(np.mean(np.abs(o0) ** 2))
        self.o0 = o0
        x = np.arange(W) * cfg.pitch
        self.ref = np.exp(1j * 2 * math.pi * math.sin(math.radians(cfg.tilt_deg)) * x / cfg.lam)[None, :]
        fd = _smooth(rng.uniform(size=(H, W)), max(H, W) / 16.0)
        fd = (fd - fd.min()) / max(fd.max() - fd.min(), 1e-30) * cfg.f_max
        self.fd = fd
        self.clutter = None
        if cfg.scr_db is not None:
            g1 = _smooth(rng.standard_normal((H, W)), max(H, W) / 8.0) + \
                1j * _smooth(rng.standard_normal((H, W)), max(H, W) / 8.0)
            g2 = _smooth(rng.standard_normal((H, W)), max(H, W) / 8.0) + \
                1j * _smooth(rng.standard_normal((H, W)), max(H, W) / 8.0)
            g1 /= math.sqrt(np.mean(np.abs(g1) ** 2))
            g2 /= math.sqrt(np.mean(np.abs(g2) ** 2))
            # slow (< 500 Hz) complex processes a(t), b(t): a few low-frequency tones
            n_tone = 4
            self._tones = [(rng.uniform(0, 500, n_tone), rng.uniform(0, 2 * math.pi, n_tone),
                            rng.uniform(0.5, 1.0, n_tone)) for _ in range(2)]
            scale = 10.0 ** (-cfg.scr_db / 20.0)   # amplitude ratio clutter/signal
            self.clutter = (g1, g2, scale)
        self._noise_seed = cfg.seed * 7919 + 13

    def _slow(self, which: int, t: np.ndarray) -> np.ndarray:
        f, ph, a = self._tones[which]
        s = np.zeros(t.shape, dtype=np.complex128)
        for fi, pi, ai in zip(f, ph, a):
            s += ai * np.exp(1j * (2 * math.pi * fi * t / self.cfg.fs + pi))
        return 1.0 + 0.5 * s / len(f)

    def frames(self, t0: int, n: int) -> np.ndarray:
        cfg = self.cfg
        out = np.empty((n, cfg.height, cfg.width), dtype=np.uint16)
        for i in range(n):
            t = t0 + i
            ot = self.o0 * np.exp(1j * 2 * math.pi * self.fd * t / cfg.fs)
            if self.clutter is not None:
                g1, g2, scale = self.clutter
                tt = np.array([t], dtype=np.float64)
                ot = ot + scale * (self._slow(0, tt)[0] * g1 + self._slow(1, tt)[0] * g2)
            inten = np.abs(self.ref + ot) ** 2
            inten *= 2048.0 / inten.mean()
            rng = np.random.default_rng(self._noise_seed + t)
            noisy = rng.poisson(inten)
            out[i] = np.clip(noisy, 0, 4095).astype(np.uint16)
        return out


# The benchmark workloads (sizes, rates and bands): config0 the small host-path case, config1 the
# full-size 1024^2 12-bit case, config2 the same with a set clutter-to-signal ratio.
def config0(n_frames: int = 32, acquisition: int = 0) -> SynthConfig:
    return SynthConfig(512, 512, n_frames, 37e3, 400, 0.30, seed=config_seed(0, acquisition))


def config1(n_frames: int = 64, acquisition: int = 0, height: int = 1024, width: int = 1024) -> SynthConfig:
    return SynthConfig(height, width, n_frames, 67e3, int(round(900 * width / 1024)), 0.25,
                       seed=config_seed(1, acquisition))


def config2(scr_db: float, n_frames: int = 64, height: int = 1024, width: int = 1024) -> SynthConfig:
    return SynthConfig(height, width, n_frames, 67e3, int(round(900 * width / 1024)), 0.25,
                       scr_db=scr_db, seed=config_seed(2))
