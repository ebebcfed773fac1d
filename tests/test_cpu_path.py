"""The FP32 C++/OpenMP restatement of the path (oracle/cpu_path.cc), which bench.py times as the
CPU baseline and the reference arm, against the FP64 oracle: relative L2 < 1e-4 per moment image
(the plain form's tolerance), for Fresnel and angular-spectrum propagation, with and without the
clutter filter, 12-bit packed and uint16 frames."""
import numpy as np
import pytest

from oracle import cpu_path as CP
from oracle import oracle as O
from oracle import synth as S


@pytest.fixture(scope="module", autouse=True)
def _built():
    CP.build()


@pytest.mark.parametrize("prop,H,W,T,rank,fs,band,packed", [
    ("fresnel", 128, 128, 64, 4, 67e3, (4e3, 33e3), True),
    ("fresnel", 64, 256, 32, 2, 37e3, (6e3, 18e3), False),
    ("angular_spectrum", 128, 128, 32, 0, 37e3, (6e3, 18e3), False),
    ("angular_spectrum", 256, 64, 64, 4, 67e3, (4e3, 33e3), True),
    ("none", 64, 64, 128, 4, 67e3, (4e3, 33e3), True),
])
def test_cpu_restatement_vs_fp64_oracle(prop, H, W, T, rank, fs, band, packed):
    frames = S.Interferograms(S.config1(T, height=H, width=W)).frames(0, T)
    z0, z1 = O.band_bins(band[0], band[1], fs, T)
    cfg = O.PathConfig(H, W, T, T // 4, z0, z1, fs=fs, propagation=prop, z=0.27, clutter_rank=rank)
    exp = O.reconstruct_window(frames, cfg)
    src = O.pack12(frames.reshape(-1)).reshape(T, -1) if packed else frames
    got = CP.window(src, cfg, packed=packed, threads=2)
    for m in range(3):
        assert O.rel_l2(got[m], exp[m]) < 1e-4, (m, O.rel_l2(got[m], exp[m]))


def test_cpu_restatement_rejects_unsupported_shapes():
    cfg = O.PathConfig(96, 96, 32, 8, 6, 16)  # not a power of two
    with pytest.raises(ValueError):
        CP.window(np.zeros((32, 96, 96), np.uint16), cfg, packed=False)
    cfg = O.PathConfig(64, 64, 32, 8, 6, 16, fftshift=True)
    with pytest.raises(ValueError):
        CP.window(np.zeros((32, 64, 64), np.uint16), cfg, packed=False)
