"""GPU parity against the FP64 oracle for every frame size, window length and clutter level the
benchmarks run: 1536 x 1024 frames (configs 3 and 4), the chosen form at T = 32 and T = 128
(configs 3 and 4), config 2 at its full 1024^2 x 64 size, and the config-3 graph launch.

Tolerances are the forms' targets: relative L2 < 1e-4 per moment image for the plain form,
< 1e-3 for the chosen form.  Frames come from the device-side generator the benchmarks use (or
the host generator for config 2), and are copied to the host for the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import synth as S

pytestmark = pytest.mark.gpu

TOL = {0: 1e-4, 1: 1e-3}


def _device_frames(cuda, H, W, n, fs=67e3, z_obj=0.25, seed=1001):
    """uint16 frames [n, H, W] from the benchmarks' device generator, as a host array."""
    from holoflow_b200 import synth as sy
    scene = sy.Scene(H, W, fs, int(round(0.85 * min(H, W))), z_obj, seed=seed)
    fr = sy.DeviceInterferograms(scene, device=cuda).frames(0, n)
    return fr.cpu().numpy().view(np.uint16)


def _run(cuda, frames, cfg, nwin, first=0):
    import torch
    from holoflow_b200 import pipeline as pl
    ring = torch.from_numpy(O.pack12(frames.reshape(-1))).to(cuda)
    p = pl.Pipeline(cfg)
    got = p.run(ring, frames.shape[0], first, nwin).cpu().numpy()
    assert p.status() == 0
    p.close()
    return got


def _oracle(cfg):
    return O.PathConfig(cfg.height, cfg.width, cfg.frames, cfg.hop, cfg.z_begin, cfg.z_end, fs=cfg.fs, z=cfg.z,
                        clutter_rank=cfg.clutter_rank)


def _check_windows(got, frames, cfg, windows, tol, label):
    errs = []
    ocfg = _oracle(cfg)
    for w in windows:
        exp = O.reconstruct_window(frames[w * cfg.hop: w * cfg.hop + cfg.frames], ocfg)
        for m in range(3):
            errs.append(O.rel_l2(got[w, m], exp[m]))
    print(f"{label}: max rel L2 {max(errs):.3e}")
    assert max(errs) < tol, errs


@pytest.mark.parametrize("form,T,hop", [(0, 64, 16), (1, 64, 16), (0, 128, 32), (1, 128, 32), (0, 32, 8), (1, 32, 8)])
def test_frames_1536x1024(cuda, form, T, hop):
    """1536 x 1024 frames (W x H), the largest size of the uneven and streaming workloads: the
    band pass and row FFT at W = 1536 and the column pass at H = 1024, both forms, every (T, hop)
    of those workloads."""
    from holoflow_b200 import pipeline as pl
    H, W, nwin = 1024, 1536, 2
    n = T + hop * (nwin - 1)
    frames = _device_frames(cuda, H, W, n)
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, T)
    cfg = pl.PipelineConfig(height=H, width=W, frames=T, hop=hop, z_begin=z0, z_end=z1, fs=67e3, z=0.27,
                            clutter_rank=4, form=form, max_batch=nwin)
    got = _run(cuda, frames, cfg, nwin)
    _check_windows(got, frames, cfg, range(nwin), TOL[form], f"1536x1024 T={T} form {form}")


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("T,H,fs", [(32, 512, 37e3), (128, 512, 67e3), (32, 1024, 67e3), (128, 1024, 37e3)])
def test_window_lengths_32_and_128(cuda, form, T, H, fs):
    """Windows of 32 and 128 frames (hop T/4), the other lengths of the uneven and streaming
    workloads, at both sampling rates' bands; the chosen form's Gram matrix is then the int8
    tensor-core path for T = 32 / 128 and its band pass the plain tiled DFT."""
    from holoflow_b200 import pipeline as pl
    hop, nwin = T // 4, 3
    n = T + hop * (nwin - 1)
    frames = _device_frames(cuda, H, H, n, fs=fs, seed=1003 + T)
    z0, z1 = O.band_bins(4e3, 33e3, fs, T) if fs > 50e3 else O.band_bins(6e3, 18e3, fs, T)
    cfg = pl.PipelineConfig(height=H, width=H, frames=T, hop=hop, z_begin=z0, z_end=z1, fs=fs, z=0.31,
                            clutter_rank=4, form=form, max_batch=nwin)
    got = _run(cuda, frames, cfg, nwin)
    _check_windows(got, frames, cfg, (0, nwin - 1), TOL[form], f"T={T} {H}^2 form {form}")


@pytest.mark.parametrize("scr_db", [0.0, -20.0, -40.0])
def test_config2_full_size(cuda, scr_db):
    """Config 2 as stated: 1024^2 x 64 frames with a rank-2 global phase/amplitude clutter at SCR
    0, -20 and -40 dB, top-4 clutter removal, both forms; the per-moment error is printed."""
    from holoflow_b200 import pipeline as pl
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, 64)
    frames = S.Interferograms(S.config2(scr_db, 64)).frames(0, 64)
    ocfg = O.PathConfig(1024, 1024, 64, 16, z0, z1, fs=67e3, z=0.25, clutter_rank=4)
    exp = O.reconstruct_window(frames, ocfg)
    for form in (0, 1):
        cfg = pl.PipelineConfig(height=1024, width=1024, frames=64, hop=16, z_begin=z0, z_end=z1, fs=67e3,
                                z=0.25, clutter_rank=4, form=form, max_batch=1)
        got = _run(cuda, frames, cfg, 1)
        errs = [O.rel_l2(got[0, m], exp[m]) for m in range(3)]
        print(f"config2 1024^2 SCR {scr_db:+.0f} dB form {form}: M0/M1/M2 rel L2 "
              + " ".join(f"{e:.3e}" for e in errs))
        assert max(errs) < TOL[form], errs


def test_config3_graph_vs_oracle(cuda):
    """The sixteen uneven acquisitions of the batched workload (sizes 256^2 .. 1536 x 1024,
    T = 32 / 64 / 128, fs 37 / 67 kHz, z 0.15 - 0.40 m) in ONE graph launch, chosen form: each
    acquisition's second window against the FP64 oracle (1e-3); and the plain form's
    per-acquisition launches, which the benchmark compares against, within 1e-4."""
    import torch
    from holoflow_b200 import pipeline as pl
    from holoflow_b200 import synth as sy
    from holoflow_b200.multi import Multi
    acqs = sy.config3_acquisitions()
    WIN = 2
    rings, nfr, outs, hosts = [], [], [], []
    for a in acqs:
        n = a.frames + (WIN - 1) * a.hop
        fr = sy.DeviceInterferograms(a.scene, device=cuda).frames(0, n)
        hosts.append(fr.cpu().numpy().view(np.uint16))
        rings.append(pl.pack12(fr.reshape(-1)))
        nfr.append(n)
        outs.append(torch.full((WIN, 3, a.scene.height, a.scene.width), float("nan"), device=cuda))

    def cfg(a, form):
        return pl.PipelineConfig(height=a.scene.height, width=a.scene.width, frames=a.frames, hop=a.hop,
                                 z_begin=a.z_begin, z_end=a.z_end, fs=a.scene.fs, z=a.z, clutter_rank=4,
                                 form=form, max_batch=WIN)

    m = Multi([cfg(a, 1) for a in acqs])
    m.tune(rings, nfr, [0] * len(acqs), outs, reps=1)
    m.exec(rings, nfr, [0] * len(acqs), outs)
    torch.cuda.synchronize()
    worst = {0: 0.0, 1: 0.0}
    for i, a in enumerate(acqs):
        c1 = cfg(a, 1)
        exp = O.reconstruct_window(hosts[i][a.hop: a.hop + a.frames], _oracle(c1))
        chosen = outs[i].cpu().numpy()[1]
        plain = _run(cuda, hosts[i], cfg(a, 0), WIN)[1]
        for form, got in ((1, chosen), (0, plain)):
            errs = [O.rel_l2(got[k], exp[k]) for k in range(3)]
            worst[form] = max(worst[form], max(errs))
            assert max(errs) < TOL[form], (i, a.scene.height, a.scene.width, a.frames, form, errs)
    print(f"config3: worst rel L2 chosen {worst[1]:.3e} plain {worst[0]:.3e}")
    m.close()
