"""GPU parity of the fused per-window path (hf_pipeline_exec) against the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import synth as S

pytestmark = pytest.mark.gpu


def _run(cuda, frames_u16, cfg_kw, nwin, first=0, fmt="mono12p"):
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    n = frames_u16.shape[0]
    if fmt == "mono12p":
        ring = torch.from_numpy(O.pack12(frames_u16.reshape(-1))).to(cuda)
        dt = hf.HF_MONO12P
    else:
        ring = torch.from_numpy(frames_u16.view(np.int16)).to(cuda)
        dt = hf.HF_U16
    cfg = pl.PipelineConfig(input_dtype=dt, max_batch=nwin, **cfg_kw)
    p = pl.Pipeline(cfg)
    out = p.run(ring, n, first, nwin)
    torch.cuda.synchronize()
    return out.cpu().numpy(), p


def _oracle_cfg(kw):
    prop = {1: "fresnel", 2: "angular_spectrum", 0: "none"}[kw.get("propagation", 1)]
    pad = {"width": kw["pad_w"], "height": kw["pad_h"]} if kw.get("pad_w") else None
    return O.PathConfig(kw["height"], kw["width"], kw["frames"], kw["hop"], kw["z_begin"], kw["z_end"],
                        fs=kw.get("fs", 37e3), propagation=prop, lam=kw.get("lam", 852e-9),
                        pitch=kw.get("pitch", 12e-6), z=kw.get("z", 0.25),
                        clutter_rank=kw.get("clutter_rank", 0), fftshift=bool(kw.get("fftshift", 0)),
                        as_padding=pad)


def _check(got, frames, kw, nwin, tol):
    ocfg = _oracle_cfg(kw)
    for w in range(nwin):
        win = frames[w * kw["hop"]: w * kw["hop"] + kw["frames"]]
        exp = O.reconstruct_window(win, ocfg)
        mask = kw.get("moment_mask", 7)
        exp = exp[[m for m in range(3) if mask & (1 << m)]]
        for m in range(exp.shape[0]):
            err = O.rel_l2(got[w, m], exp[m])
            assert err < tol, (w, m, err)


def test_pipeline_config1_mini_fresnel_svd(cuda):
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, 64)
    kw = dict(height=256, width=256, frames=64, hop=16, z_begin=z0, z_end=z1, fs=67e3, z=0.25,
              clutter_rank=4)
    frames = S.Interferograms(S.config1(64 + 2 * 16, height=256, width=256)).frames(0, 96)
    got, _ = _run(cuda, frames, kw, 3)
    _check(got, frames, kw, 3, 1e-4)


def test_pipeline_config0_angular_spectrum(cuda):
    z0, z1 = O.band_bins(6e3, 18e3, 37e3, 32)
    kw = dict(height=512, width=512, frames=32, hop=32, z_begin=z0, z_end=z1, fs=37e3, z=0.30,
              propagation=2)
    frames = S.Interferograms(S.config0(64)).frames(0, 64)
    got, _ = _run(cuda, frames, kw, 2, fmt="u16")
    _check(got, frames, kw, 2, 1e-4)


@pytest.mark.parametrize("form,tol", [(0, 1e-4), (1, 1e-3)])
def test_pipeline_variants_fftshift_m0_none_padding(cuda, form, tol):
    """Display and propagation variants in both forms (the chosen form runs them through the
    tensor-core segment pass at T = 32)."""
    frames = S.Interferograms(S.config0(48)).frames(0, 48)[:, :128, :128].copy()
    base = dict(height=128, width=128, frames=32, hop=16, z_begin=6, z_end=16, fs=37e3, z=0.3)
    for extra in (dict(fftshift=1), dict(moment_mask=1), dict(propagation=0), dict(clutter_rank=2),
                  dict(propagation=2, pad_w=256, pad_h=256), dict(propagation=2, fftshift=1, moment_mask=5)):
        kw = {**base, **extra}
        got, p = _run(cuda, frames, dict(kw, form=form), 2)
        assert p.status() == 0
        _check(got, frames, kw, 2, tol)


def test_pipeline_ring_wraparound(cuda):
    """Windows that wrap around the end of the device ring equal the unwrapped ones."""
    frames = S.Interferograms(S.config0(64)).frames(0, 64)[:, :128, :128].copy()
    kw = dict(height=128, width=128, frames=32, hop=16, z_begin=6, z_end=16, z=0.3)
    a, _ = _run(cuda, frames, kw, 1, first=16)
    rolled = np.roll(frames, -40, axis=0)  # frame 16 now sits at index 40 (wraps)
    b, _ = _run(cuda, rolled, kw, 1, first=40)
    assert np.array_equal(a, b)


def test_pipeline_full_config1_window(cuda):
    """Config 1 at full size (1024^2, T = 64, hop 16, top-4 clutter removal, Fresnel, 4-33 kHz)."""
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, 64)
    kw = dict(height=1024, width=1024, frames=64, hop=16, z_begin=z0, z_end=z1, fs=67e3, z=0.25,
              clutter_rank=4)
    frames = S.Interferograms(S.config1(64)).frames(0, 64)
    got, _ = _run(cuda, frames, kw, 1)
    _check(got, frames, kw, 1, 1e-4)


def test_pipeline_rejects_bad_desc(cuda):
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    with pytest.raises(hf.HfError) as e:
        pl.Pipeline(pl.PipelineConfig(height=64, width=64, frames=32, hop=8, z_begin=10, z_end=5))
    assert e.value.code == hf.HF_ERR_INVALID


@pytest.mark.parametrize("T,H,W", [(64, 256, 256), (128, 128, 128), (64, 1024, 1024)])
def test_chosen_form_tensor_core_gram(cuda, T, H, W):
    """The chosen form's tcgen05 Gram matrix equals the exact integer Gram of the 12-bit frames."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    frames = S.Interferograms(S.config1(T, height=H, width=W)).frames(0, T)
    ring = torch.from_numpy(O.pack12(frames.reshape(-1))).to(cuda)
    cfg = pl.PipelineConfig(height=H, width=W, frames=T, hop=16, z_begin=4, z_end=min(32, T // 2),
                            fs=67e3, z=0.25, clutter_rank=4, form=hf.HF_FORM_CHOSEN)
    p = pl.Pipeline(cfg)
    p.run(ring, T, 0, 1)
    gram, _ = p.inspect(0)
    assert p.status() == 0
    X = frames.reshape(T, -1).astype(np.float64)
    exact = X @ X.T
    g = gram.cpu().numpy()
    # 12-bit samples: exact int8 split on the tensor core, so the Gram matrix is exact
    assert np.array_equal(g, exact)
    assert np.array_equal(g, g.T)


@pytest.mark.parametrize("hop,nwin,dtype,first,H", [
    (16, 8, "mono12p", 0, 128), (16, 5, "mono12p", 37, 128), (8, 2, "mono12p", 3, 128),
    (24, 3, "mono12p", 11, 128), (32, 6, "mono12p", 50, 128), (16, 7, "u8", 9, 128),
    (8, 4, "u8", 0, 128), (16, 8, "mono12p", 5, 512)])
def test_chosen_form_grouped_gram(cuda, hop, nwin, dtype, first, H):
    """Batches of overlapping 64-frame windows on an 8-frame hop grid share each staged frame
    between the windows of a group of four; every window's Gram matrix stays the exact integer
    Gram of its own frames, for full and partial groups, 12- and 8-bit samples, and windows that
    wrap around the end of the frame ring."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    T, W = 64, H
    n = T + hop * (nwin - 1)
    rng = np.random.default_rng(hop * 100 + nwin)
    top = 4096 if dtype == "mono12p" else 256
    frames = rng.integers(0, top, size=(n, H * W)).astype(np.uint16)
    frames[0, :] = top - 1  # saturated and zero frames exercise the extreme fields
    frames[1, :] = 0
    # ring slot (first + f) % n holds window frame f
    slots = (first + np.arange(n)) % n
    ring_np = np.empty_like(frames)
    ring_np[slots] = frames
    if dtype == "mono12p":
        ring = torch.from_numpy(O.pack12(ring_np.reshape(-1))).to(cuda)
        in_dtype = hf.HF_MONO12P
    else:
        ring = torch.from_numpy(ring_np.astype(np.uint8).reshape(-1)).to(cuda)
        in_dtype = hf.HF_U8
    cfg = pl.PipelineConfig(height=H, width=W, frames=T, hop=hop, z_begin=4, z_end=32, fs=67e3, z=0.25,
                            clutter_rank=4, form=hf.HF_FORM_CHOSEN, max_batch=nwin, input_dtype=in_dtype)
    p = pl.Pipeline(cfg)
    p.run(ring, n, first, nwin)
    assert p.status() == 0
    for w in range(nwin):
        gram, _ = p.inspect(w)
        X = frames[w * hop:w * hop + T].astype(np.float64)
        assert np.array_equal(gram.cpu().numpy(), X @ X.T), w


@pytest.mark.parametrize("H,W,nwin", [(256, 256, 3), (512, 512, 2), (768, 768, 2), (1024, 1024, 2)])
def test_chosen_form_fresnel_vs_oracle(cuda, H, W, nwin):
    """Chosen form (int8 tensor-core Gram, f16 tensor-core band DFT fused with lens + row FFT):
    M0/M1/M2 within the 1e-3 relative-L2 target of the float64 oracle, and the device status word
    stays clear."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, 64)
    n = 64 + 16 * (nwin - 1)
    frames = S.Interferograms(S.config1(n, height=H, width=W)).frames(0, n)
    ring = torch.from_numpy(O.pack12(frames.reshape(-1))).to(cuda)
    cfg = pl.PipelineConfig(height=H, width=W, frames=64, hop=16, z_begin=z0, z_end=z1, fs=67e3, z=0.25,
                            clutter_rank=4, form=hf.HF_FORM_CHOSEN, max_batch=nwin)
    p = pl.Pipeline(cfg)
    got = p.run(ring, n, 0, nwin).cpu().numpy()
    assert p.status() == 0
    ocfg = O.PathConfig(H, W, 64, 16, z0, z1, fs=67e3, z=0.25, clutter_rank=4)
    for w in range(nwin):
        exp = O.reconstruct_window(frames[16 * w:16 * w + 64], ocfg)
        for m in range(3):
            err = O.rel_l2(got[w, m], exp[m])
            assert err < 1e-3, (w, m, err)


@pytest.mark.parametrize("form", [0, 1])
def test_camera_stream_lookahead_matches_exec(cuda, form):
    """Windows reconstructed through a camera stream (pushes from host memory, batches of varying
    size, the next batch's filter prepared ahead on a side stream) equal hf_pipeline_exec of each
    window alone: bit for bit in the chosen form (exact integer Gram matrices); within 1e-5 in the
    plain form, whose FP32 covariance splits its partial sums by a grid sized from the batch."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    H = W = 256
    nwin = 9
    n = 64 + 16 * (nwin - 1)
    frames = S.Interferograms(S.config1(n, height=H, width=W)).frames(0, n)
    packed = O.pack12(frames.reshape(-1)).reshape(n, -1)
    cfg = pl.PipelineConfig(height=H, width=W, frames=64, hop=16, z_begin=4, z_end=32, fs=67e3, z=0.25,
                            clutter_rank=4, form=form, max_batch=3)
    ref = pl.Pipeline(cfg)
    ring = torch.from_numpy(packed.reshape(-1).copy()).to(cuda)
    expect = [ref.run(ring, n, 16 * w, 1).cpu().numpy()[0] for w in range(nwin)]
    p = pl.Pipeline(cfg)
    cam = pl.CameraStream(p, n)
    host = torch.from_numpy(packed.copy()).pin_memory()
    cam.push(host, n)
    out = torch.empty((3, *p.out_shape), dtype=torch.float32, pin_memory=True)
    got = []
    for mw in (2, 2, 1, 3, 3):      # matching and mismatching lookahead batches
        k = cam.process(mw, out)
        torch.cuda.synchronize()
        got += [out[i].numpy().copy() for i in range(k)]
    assert len(got) == nwin and cam.ready() == 0
    for w in range(nwin):
        if form == 1:
            assert np.array_equal(got[w], expect[w]), w
        else:
            assert O.rel_l2(got[w], expect[w]) < 1e-5, w
    assert p.status() == 0


def test_camera_stream_push_stream_and_async_output(cuda):
    """Pushes on their own CUDA stream, two steps ahead of the reconstruction, with images copied
    to the host asynchronously into alternating buffers, and a ring just large enough that pushes
    overwrite slots that recent processes read: every window equals hf_pipeline_exec of it alone."""
    import torch
    from holoflow_b200 import pipeline as pl
    H = W = 256
    B, hop, T = 2, 16, 64
    nsteps = 7
    n = (T - hop) + (nsteps + 2) * B * hop
    frames = S.Interferograms(S.config1(n, height=H, width=W)).frames(0, n)
    packed = O.pack12(frames.reshape(-1)).reshape(n, -1)
    cfg = pl.PipelineConfig(height=H, width=W, frames=T, hop=hop, z_begin=4, z_end=32, fs=67e3, z=0.25,
                            clutter_rank=4, form=1, max_batch=B)
    ref = pl.Pipeline(cfg)
    ring = torch.from_numpy(packed.reshape(-1).copy()).to(cuda)
    expect = [ref.run(ring, n, hop * w, 1).cpu().numpy()[0] for w in range(nsteps * B)]
    p = pl.Pipeline(cfg)
    cam = pl.CameraStream(p, (T - hop) + 4 * B * hop)
    host = torch.from_numpy(packed.copy()).pin_memory()
    h2d = torch.cuda.Stream(device=cuda)
    main = torch.cuda.current_stream()
    outs = [torch.empty((B, *p.out_shape), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    pos = 0

    def push(k):
        nonlocal pos
        cam.push(host[pos:pos + k], k, stream=h2d)
        pos += k

    push(T - hop)
    push(B * hop)
    push(B * hop)
    got = []
    for s in range(nsteps):
        push(B * hop)
        k = cam.process(B, outs[s % 2], stream=main, async_copy=True)
        assert k == B
        cam.output_wait(host_block=True)
        got += [outs[s % 2][i].numpy().copy() for i in range(B)]
    torch.cuda.synchronize()
    for w in range(nsteps * B):
        assert np.array_equal(got[w], expect[w]), w
    assert p.status() == 0


@pytest.mark.parametrize("scr_db", [0.0, -20.0, -40.0])
def test_config2_clutter_error_vs_fp64_oracle(cuda, scr_db):
    """Config 2: config 1 with a rank-2 global phase/amplitude clutter at SCR 0, -20, -40 dB,
    top-4 clutter removal, 256 x 256 crop of the scene size.  Relative L2 error of each moment image
    against the FP64 oracle: < 1e-4 in the plain form, < 1e-3 in the chosen form."""
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, 64)
    kw = dict(height=256, width=256, frames=64, hop=16, z_begin=z0, z_end=z1, fs=67e3, z=0.25, clutter_rank=4)
    frames = S.Interferograms(S.config2(scr_db, 64 + 16, height=256, width=256)).frames(0, 80)
    ocfg = _oracle_cfg(kw)
    exp = [O.reconstruct_window(frames[16 * w: 16 * w + 64], ocfg) for w in range(2)]
    for form, tol in ((0, 1e-4), (1, 1e-3)):
        got, _ = _run(cuda, frames, {**kw, "form": form}, 2)
        errs = [O.rel_l2(got[w, m], exp[w][m]) for w in range(2) for m in range(3)]
        print(f"config2 SCR {scr_db:+.0f} dB form {form}: max rel L2 {max(errs):.3e}")
        assert max(errs) < tol, errs


@pytest.mark.parametrize("form,prop,H", [(0, "fresnel", 256), (1, "fresnel", 256), (1, "fresnel", 1024),
                                         (0, "angular_spectrum", 128)])
def test_two_sided_fft_time_method(cuda, form, prop, H):
    """The reference's FFT time method (graph_builder.cc:270-287): the band [z0, z1) and the
    negative band [T - z1, T - z0) concatenated, 2 Nz planes propagated, moments weighted
    [f0 .. f1) then [f0 - fs .. f1 - fs) (590-594); against the float64 oracle within the form's
    tolerance (1e-4 plain, 1e-3 chosen)."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    W = H
    nwin = 2
    n = 64 + 16 * (nwin - 1)
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, 64) if prop == "fresnel" else (6, 16)
    frames = S.Interferograms(S.config1(n, height=H, width=W)).frames(0, n)
    ring = torch.from_numpy(O.pack12(frames.reshape(-1))).to(cuda)
    cfg = pl.PipelineConfig(height=H, width=W, frames=64, hop=16, z_begin=z0, z_end=z1, fs=67e3, z=0.25,
                            clutter_rank=4, form=form, max_batch=nwin, time_method=hf.HF_TIME_FFT,
                            propagation=hf.HF_PROP_FRESNEL if prop == "fresnel" else hf.HF_PROP_ANGULAR_SPECTRUM)
    p = pl.Pipeline(cfg)
    got = p.run(ring, n, 0, nwin).cpu().numpy()
    assert p.status() == 0
    ocfg = O.PathConfig(H, W, 64, 16, z0, z1, fs=67e3, z=0.25, clutter_rank=4, propagation=prop,
                        time_method="fft")
    tol = 1e-4 if form == 0 else 1e-3
    for w in range(nwin):
        exp = O.reconstruct_window(frames[16 * w:16 * w + 64], ocfg)
        for m in range(3):
            err = O.rel_l2(got[w, m], exp[m])
            assert err < tol, (w, m, err)
    # the negative band's weights are negative: M1 differs from the one-sided method's
    one = pl.Pipeline(pl.PipelineConfig(**{**cfg.__dict__, "time_method": hf.HF_TIME_RFFT}))
    got1 = one.run(ring, n, 0, nwin).cpu().numpy()
    assert O.rel_l2(got1[0, 1], got[0, 1]) > 0.1


@pytest.mark.parametrize("T,hop,H,W,prop,fmt,lo,hi,fs", [
    (32, 32, 128, 256, 2, "u16", 6e3, 18e3, 37e3),        # config-0 shape class: T = 32, angular spectrum
    (128, 32, 64, 384, 1, "mono12p", 4e3, 33e3, 67e3),    # T = 128: 56 bins (N = 112), 3 tiles
    (64, 16, 64, 1536, 1, "mono12p", 4e3, 33e3, 67e3),    # 12 tiles: segments of 8 and 4
    (32, 8, 96, 1280, 0, "u16", 6e3, 18e3, 37e3),         # no propagation, 10 tiles in one segment
])
def test_chosen_form_segment_band_pass(cuda, T, hop, H, W, prop, fmt, lo, hi, fs):
    """Shapes the fused row pass does not take run the tensor-core band DFT in row segments (raw
    planes, lens in the row pass); the moments match the FP64 oracle within the chosen form's
    tolerance, and the plain form's FP32 band DFT within its own."""
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    nwin = 3
    n = T + hop * (nwin - 1)
    z0, z1 = O.band_bins(lo, hi, fs, T)
    frames = S.Interferograms(S.SynthConfig(H, W, n, fs, int(0.8 * min(H, W)), 0.25, seed=1077)).frames(0, n)
    kw = dict(height=H, width=W, frames=T, hop=hop, z_begin=z0, z_end=z1, fs=fs, z=0.25, clutter_rank=4,
              propagation=prop)
    for form, tol, kind in ((hf.HF_FORM_CHOSEN, 1e-3, hf.HF_BAND_TC_SEGMENTS), (hf.HF_FORM_PLAIN, 1e-4, hf.HF_BAND_FP32)):
        got, p = _run(cuda, frames, dict(kw, form=form), nwin, fmt=fmt)
        assert p.band_pass() == kind
        assert p.status() == 0
        _check(got, frames, kw, nwin, tol)

