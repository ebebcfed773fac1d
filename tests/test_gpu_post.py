"""Post-moment display chain on the GPU against the oracle's restatements of the reference
(holonp/src/fftshift.cu, holotask/src/syncs/flatfield.cu, pct_clip.cu, asyncs/slide_avg.cu).

Tolerances: fftshift, the percentile clip and the sliding average are exact (index moves, an exact
radix select, and the reference's own float32 operation order); the flatfield compares float32
kernels to a float64 oracle at 2e-5 of the image's largest magnitude."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import synth as S

pytestmark = pytest.mark.gpu


def _post():
    from holoflow_b200 import post
    return post


def image(rng, shape):
    """A moment-like image: smooth background, structure and noise, positive."""
    H, W = shape[-2:]
    y, x = np.mgrid[0:H, 0:W] / max(H, W)
    base = 1000.0 * (1.0 + 0.5 * np.sin(3.0 * x) * np.cos(2.0 * y)) + 200.0 * np.exp(-((x - 0.4) ** 2 + (y - 0.6) ** 2) / 0.01)
    return (base + 30.0 * rng.standard_normal(shape)).astype(np.float32)


@pytest.mark.parametrize("shape,axes,dtype", [((1024, 1024), None, np.float32), ((3, 7, 5), (-2, -1), np.float32),
                                             ((2, 6, 9), (0, 2), np.uint8), ((4, 5), (1,), np.complex64),
                                             ((5, 3, 8), None, np.uint16)])
def test_fftshift_matches_reference_rule(cuda, shape, axes, dtype):
    import torch
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(shape) * 100).astype(dtype) if dtype != np.complex64 else \
        (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    t = torch.from_numpy(x).to(cuda)
    got = _post().fftshift(t, axes).cpu().numpy()
    assert np.array_equal(got, O.fftshift_ref(x, None if axes is None else [a % x.ndim for a in axes]))


@pytest.mark.parametrize("shape,sigma", [((1, 512, 512), (3.0, 3.0)), ((2, 1024, 1024), (7.5, 4.0)),
                                         ((1, 300, 200), (10.0, 2.0)), ((1, 512, 512), (20.0, 20.0)),
                                         ((2, 1024, 1024), (18.7, 25.0))])
def test_flatfield_spatial_and_fourier_paths(cuda, shape, sigma):
    import torch
    rng = np.random.default_rng(2)
    x = image(rng, shape)
    sy, sx = sigma
    ff = _post().Flatfield(shape, sy, sx)
    fourier = O.flatfield_uses_fourier(shape[-2], shape[-1], sy, sx)
    assert ff.fourier == fourier
    got = ff(torch.from_numpy(x).to(cuda)).cpu().numpy()
    exp = O.flatfield_fourier(x, sy, sx) if fourier else O.flatfield_spatial(x, sy, sx)
    err = np.abs(got - exp).max() / np.abs(x).max()
    assert err < 2e-5, err


@pytest.mark.parametrize("shape,pcts,roi", [((1, 1024, 1024), (0.5, 99.5), (0.5, 0.5, 0.5, 0.5)),
                                            ((3, 256, 320), (10.0, 90.0), (0.4, 0.6, 0.3, 0.45)),
                                            ((2, 128, 128), (0.0, 100.0), (0.5, 0.5, 1.0, 1.0))])
def test_pct_clip_exact_against_sorted_ranks(cuda, shape, pcts, roi):
    import torch
    rng = np.random.default_rng(3)
    x = (rng.standard_normal(shape) * 50).astype(np.float32)
    x.reshape(-1)[::97] = 0.0
    x.reshape(-1)[1::89] = -0.0
    x.reshape(-1)[2::61] = x.reshape(-1)[5]  # ties
    mask = O.ellipse_mask(*shape, *roi, 0.0)
    exp, lo, hi = O.pct_clip(x, pcts[0], pcts[1], mask)
    pc = _post().PctClip(shape, pcts[0], pcts[1], roi=(*roi, 0.0))
    assert pc.roi_count == int(mask.sum())
    bounds = torch.empty(2, dtype=torch.float32, device=cuda)
    for _ in range(2):  # the selection state is rebuilt on every call
        got = pc(torch.from_numpy(x).to(cuda), bounds=bounds)
        assert np.array_equal(bounds.cpu().numpy(), np.array([lo, hi], dtype=np.float32))
        assert np.array_equal(got.cpu().numpy(), exp)


def test_pct_clip_rotated_roi_and_empty_roi(cuda):
    import torch
    import holoflow_b200 as hf
    post = _post()
    rng = np.random.default_rng(4)
    x = rng.standard_normal((1, 200, 300)).astype(np.float32)
    pc = post.PctClip((1, 200, 300), 5.0, 95.0, roi=(0.5, 0.5, 0.4, 0.2, 30.0))
    got = pc(torch.from_numpy(x).to(cuda)).cpu().numpy()
    lo, hi = got.min(), got.max()
    # the two bounds are values of the image, and ~5 % of the region's pixels lie on each side
    assert lo in x and hi in x and (x < lo).mean() > 0.01 and (x > hi).mean() > 0.01
    with pytest.raises(hf.HfError, match="no pixels in ROI"):
        post.PctClip((1, 4, 4), 5.0, 95.0, roi=(0.01, 0.01, 0.01, 0.01, 0.0))


@pytest.mark.parametrize("window,discard", [(1, 0), (3, 1), (4, 0)])
def test_sliding_average_float32_sequence(cuda, window, discard):
    import torch
    rng = np.random.default_rng(5)
    imgs = [image(rng, (256, 256)) for _ in range(9)]
    exp = O.slide_avg(imgs, window, discard)
    sa = _post().SlidingAverage(256 * 256, window, discard)
    got = []
    for im in imgs:
        r = sa.push(torch.from_numpy(im).to(cuda))
        if r is not None:
            got.append(r.cpu().numpy())
    assert len(got) == len(exp) == 9 - discard - window + 1
    for g, e in zip(got, exp):
        assert np.array_equal(g, e)


def test_display_chain_nodes_end_to_end(cuda):
    """FFTShiftNp -> Flatfield -> PctClip -> Conversion(U8, Scaled) driven as nodes, as the
    reference's graph wires them (graph_builder.cc:633-676), against the oracle chain."""
    import torch
    from holoflow_b200 import nodes as N
    rng = np.random.default_rng(6)
    x = image(rng, (1, 512, 512))
    dev = torch.from_numpy(x).to(cuda)
    (s,) = N.run_sync_factory("FFTShiftNp", {"axes": [-2, -1]}, [dev])
    (f,) = N.run_sync_factory("Flatfield", {"sigma_y": 4.0, "sigma_x": 4.0}, [s])
    roi = {"cx": 0.5, "cy": 0.5, "rx": 0.5, "ry": 0.5, "angle": 0.0}
    (c,) = N.run_sync_factory("PctClip", {"min_pct": 1.0, "max_pct": 99.0, "roi": roi}, [f])
    e = O.flatfield_spatial(O.fftshift_ref(x, [1, 2]), 4.0, 4.0)
    got_f = f.cpu().numpy()
    assert np.abs(got_f - e).max() / np.abs(x).max() < 2e-5
    # the clip is exact on the device's own flatfield output
    mask = O.ellipse_mask(1, 512, 512, 0.5, 0.5, 0.5, 0.5, 0.0)
    exp_c, _, _ = O.pct_clip(got_f, 1.0, 99.0, mask)
    assert np.array_equal(c.cpu().numpy(), exp_c)
    (u8,) = N.run_sync_factory("Conversion", {"target": "U8", "strategy": "Scaled"}, [c])
    u = u8.cpu().numpy()
    assert u.dtype == np.uint8 and u.min() == 0 and u.max() == 255


@pytest.mark.parametrize("real,shape,radii", [(False, (3, 256, 256), (4, 60, 6, 10)), (True, (2, 512, 512), (0, 100, 0, 20)),
                                              (False, (1, 1024, 1024), (10, 300, 20, 40)), (True, (1, 128, 256), (3, 40, 5, 0))])
def test_filter2d_complex_and_real(cuda, real, shape, radii):
    """Filter2D against the oracle: the annulus in natural frequency order, (g, g) on complex
    planes as the reference's complex path, (g, 0) on the real half spectrum; unnormalized."""
    import torch
    rng = np.random.default_rng(7)
    x = rng.standard_normal(shape).astype(np.float32)
    if not real:
        x = (x + 1j * rng.standard_normal(shape)).astype(np.complex64)
    f = _post().Filter2D(shape, real, *radii)
    got = f(torch.from_numpy(x).to(cuda)).cpu().numpy()
    exp = O.filter2d(x, *radii)
    assert O.rel_l2(got, exp) < 1e-5


@pytest.mark.parametrize("form", [0, 1])
def test_pipeline_filter2d_before_fresnel(cuda, form):
    """With the filter on and Fresnel propagation, the band planes go through Filter2D before
    the lens (graph_builder.cc:124-126), in both forms, against the oracle."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    H = W = 256
    nwin, n = 2, 80
    z0, z1 = O.band_bins(4e3, 33e3, 67e3, 64)
    frames = S.Interferograms(S.config1(n, height=H, width=W)).frames(0, n)
    ring = torch.from_numpy(O.pack12(frames.reshape(-1))).to(cuda)
    flt = dict(r_inner=4, r_outer=90, s_inner=6, s_outer=20)
    cfg = pl.PipelineConfig(height=H, width=W, frames=64, hop=16, z_begin=z0, z_end=z1, fs=67e3, z=0.25,
                            clutter_rank=4, form=form, max_batch=nwin, as_filter=1, **flt)
    p = pl.Pipeline(cfg)
    got = p.run(ring, n, 0, nwin).cpu().numpy()
    assert p.status() == 0
    ocfg = O.PathConfig(H, W, 64, 16, z0, z1, fs=67e3, z=0.25, clutter_rank=4, filter2d=flt)
    tol = 1e-4 if form == 0 else 1e-3
    for w in range(nwin):
        exp = O.reconstruct_window(frames[16 * w:16 * w + 64], ocfg)
        for m in range(3):
            assert O.rel_l2(got[w, m], exp[m]) < tol, (w, m)
