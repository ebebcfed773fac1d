"""Device-side synthetic laser Doppler interferograms (acquisition simulator).

Generates 12-bit frames on the GPU with torch for benchmarks and the streaming simulator:
an off-axis plane reference wave (1.5 degree tilt), a circular-Gaussian speckle object on a
centred disk propagated by an angular spectrum over ``z_obj``, a smooth Doppler map in
[0, f_max] and frames I_t = |R + O0 exp(i 2 pi f_d t / fs)|^2 scaled to mean 2048 with Poisson
shot noise, clipped to [0, 4095].  Frames are returned as uint16 values in an int16 tensor or
packed to the 12-bit stream by the library's hf_pack12.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import torch


@dataclass
class Scene:
    height: int
    width: int
    fs: float
    disk_px: int
    z_obj: float
    lam: float = 852e-9
    pitch: float = 12e-6
    tilt_deg: float = 1.5
    f_max: float = 18e3
    seed: int = 1000
    scr_db: Optional[float] = None  # rank-2 global clutter at this signal-to-clutter ratio (None = off)


class DeviceInterferograms:
    def __init__(self, scene: Scene, device="cuda"):
        self.s = scene
        self.dev = torch.device(device)
        g = torch.Generator(device=self.dev).manual_seed(scene.seed)
        H, W = scene.height, scene.width
        yy, xx = torch.meshgrid(torch.arange(H, device=self.dev, dtype=torch.float64),
                                torch.arange(W, device=self.dev, dtype=torch.float64), indexing="ij")
        disk = (torch.hypot(xx - W / 2.0, yy - H / 2.0) <= scene.disk_px / 2.0).to(torch.float64)
        re = torch.randn((H, W), generator=g, device=self.dev, dtype=torch.float64)
        im = torch.randn((H, W), generator=g, device=self.dev, dtype=torch.float64)
        speck = torch.complex(re, im) / math.sqrt(2.0) * disk
        fx = torch.fft.fftfreq(W, d=scene.pitch, device=self.dev, dtype=torch.float64)
        fy = torch.fft.fftfreq(H, d=scene.pitch, device=self.dev, dtype=torch.float64)
        arg = 1.0 - (scene.lam * fx[None, :]) ** 2 - (scene.lam * fy[:, None]) ** 2
        kz = 2 * math.pi / scene.lam * torch.sqrt(torch.clamp(arg, min=0.0))
        tf = torch.exp(1j * scene.z_obj * (kz - 2 * math.pi / scene.lam)) * (arg > 0)
        o0 = torch.fft.ifft2(torch.fft.fft2(speck) * tf)
        self.o0 = o0 / torch.sqrt(torch.mean(torch.abs(o0) ** 2))
        x = torch.arange(W, device=self.dev, dtype=torch.float64) * scene.pitch
        self.ref = torch.exp(1j * 2 * math.pi * math.sin(math.radians(scene.tilt_deg)) * x / scene.lam)[None, :]
        noise = torch.rand((H, W), generator=g, device=self.dev, dtype=torch.float64)
        sigma = max(H, W) / 16.0
        gy = torch.exp(-0.5 * (torch.fft.fftfreq(H, device=self.dev, dtype=torch.float64) * 2 * math.pi * sigma) ** 2)
        gx = torch.exp(-0.5 * (torch.fft.fftfreq(W, device=self.dev, dtype=torch.float64) * 2 * math.pi * sigma) ** 2)
        fd = torch.fft.ifft2(torch.fft.fft2(noise) * gy[:, None] * gx[None, :]).real
        self.fd = (fd - fd.min()) / torch.clamp(fd.max() - fd.min(), min=1e-30) * scene.f_max
        self._g = torch.Generator(device=self.dev).manual_seed(scene.seed * 7919 + 13)
        self.clutter = None
        if scene.scr_db is not None:
            # rank-2 clutter K_t = a(t) G1 + b(t) G2: smooth complex spatial patterns (sigma = side/8)
            # of unit rms, and slow complex processes a, b made of four tones below 500 Hz
            sc = max(H, W) / 8.0
            cy = torch.exp(-0.5 * (torch.fft.fftfreq(H, device=self.dev, dtype=torch.float64) * 2 * math.pi * sc) ** 2)
            cx = torch.exp(-0.5 * (torch.fft.fftfreq(W, device=self.dev, dtype=torch.float64) * 2 * math.pi * sc) ** 2)

            def smooth_noise():
                n = torch.randn((H, W), generator=g, device=self.dev, dtype=torch.float64)
                return torch.fft.ifft2(torch.fft.fft2(n) * cy[:, None] * cx[None, :]).real

            pats = []
            for _ in range(2):
                p = torch.complex(smooth_noise(), smooth_noise())
                pats.append(p / torch.sqrt(torch.mean(torch.abs(p) ** 2)))
            gt = torch.Generator(device="cpu").manual_seed(scene.seed * 31 + 7)
            tones = [(torch.rand(4, generator=gt, dtype=torch.float64) * 500.0,
                      torch.rand(4, generator=gt, dtype=torch.float64) * 2 * math.pi,
                      0.5 + 0.5 * torch.rand(4, generator=gt, dtype=torch.float64)) for _ in range(2)]
            self.clutter = (pats, tones, 10.0 ** (-scene.scr_db / 20.0))

    def frames(self, t0: int, n: int) -> torch.Tensor:
        """uint16 values in an int16 tensor [n, H, W] for absolute times t0 .. t0+n-1."""
        s = self.s
        out = torch.empty((n, s.height, s.width), dtype=torch.int16, device=self.dev)
        for i in range(n):
            ot = self.o0 * torch.exp(1j * 2 * math.pi * self.fd * ((t0 + i) / s.fs))
            if self.clutter is not None:
                pats, tones, scale = self.clutter
                t = (t0 + i) / s.fs
                for p, (f, ph, a) in zip(pats, tones):
                    tone = sum(float(ai) * complex(math.cos(2 * math.pi * float(fi) * t + float(pi)),
                                                   math.sin(2 * math.pi * float(fi) * t + float(pi)))
                               for fi, pi, ai in zip(f, ph, a))
                    ot = ot + scale * (1.0 + 0.5 * tone / len(f)) * p
            inten = torch.abs(self.ref + ot) ** 2
            inten = (inten * (2048.0 / inten.mean())).to(torch.float32)
            noisy = torch.poisson(inten, generator=self._g)
            out[i] = torch.clamp(noisy, 0, 4095).to(torch.int32).to(torch.int16)
        return out


def config1_scene(height=1024, width=1024, acquisition=0) -> Scene:
    return Scene(height, width, 67e3, int(round(900 * width / 1024)), 0.25, seed=1000 + 1 + 17 * acquisition)


def config2_scene(scr_db: float, height=1024, width=1024) -> Scene:
    """Config 1's scene with a rank-2 global phase/amplitude clutter at `scr_db` dB."""
    return Scene(height, width, 67e3, int(round(900 * width / 1024)), 0.25, seed=1000 + 2, scr_db=scr_db)


def config0_scene(acquisition=0) -> Scene:
    return Scene(512, 512, 37e3, 400, 0.30, seed=1000 + 17 * acquisition)


@dataclass
class Acquisition:
    """One acquisition of the uneven batch: its scene and processing parameters."""
    scene: Scene
    frames: int        # T, window length
    hop: int
    z: float           # propagation distance of the reconstruction
    z_begin: int       # band bins [z_begin, z_end) of the T-point DFT
    z_end: int


def band_bins(f_lo: float, f_hi: float, fs: float, T: int) -> tuple[int, int]:
    """z0 = ceil(f_lo/df), z1 = floor(f_hi/df) + 1 with df = fs/T, clipped to the one-sided range."""
    df = fs / T
    z0 = int(math.ceil(f_lo / df - 1e-9))
    z1 = min(int(math.floor(f_hi / df + 1e-9)) + 1, T // 2 + 1)
    return z0, z1


def config3_acquisitions(n: int = 16, seed: int = 1003) -> list[Acquisition]:
    """Seeded uneven acquisitions: frame sizes from {256^2, 512^2, 768^2, 1024^2, 1536 x 1024 (W x H)},
    window lengths from {32, 64, 128} (hop T/4), z uniform in [0.15, 0.40] m, fs from {37, 67} kHz,
    band 4-33 kHz at 67 kHz and 6-18 kHz at 37 kHz."""
    import random
    rng = random.Random(seed)
    sizes = [(256, 256), (512, 512), (768, 768), (1024, 1024), (1024, 1536)]
    out = []
    for a in range(n):
        H, W = sizes[rng.randrange(len(sizes))]
        T = [32, 64, 128][rng.randrange(3)]
        fs = [37e3, 67e3][rng.randrange(2)]
        z = rng.uniform(0.15, 0.40)
        z0, z1 = band_bins(4e3, 33e3, fs, T) if fs > 50e3 else band_bins(6e3, 18e3, fs, T)
        scene = Scene(H, W, fs, int(round(0.85 * min(H, W))), z, seed=1000 + 3 + 17 * a)
        out.append(Acquisition(scene, T, max(1, T // 4), z, z0, z1))
    return out
