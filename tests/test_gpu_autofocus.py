"""Shack-Hartmann autofocus on the GPU against the oracle (oracle/shack.py), which restates
short_time_fresnel_diffraction.cu, cross_correlation2.cu, shack_hartmann_slopes.cu,
zernike_from_slopes.cc, zernike_phase.cu, correct_phase.cu and wrap2pi.cu.

Tolerances: the short-time Fresnel transforms are float32 FFTs of lengths up to 1024 against
float64 (relative L2 1e-5); correlation maps 2e-5 absolute on textured images (the cross power
is unit-magnitude in every bin, so bins at rounding level would carry noise phases); peak offsets
2e-3 pixel; the device Zernike fit equals the host fit bit for bit and the float64
fit to 2e-5 (the reference's bound); the autofocus chain's coefficients to 1e-3 relative."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from oracle import shack as SH

pytestmark = pytest.mark.gpu

LAM, DX, Z = 852e-9, 20e-6, 0.25


def _af():
    from holoflow_b200 import autofocus
    return autofocus


def cfield(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.mark.parametrize("shape,win,stride,ref,output", [
    ((2, 510, 510), (102, 102), (102, 102), "global", "magnitude"),   # nb = 5: 2 x 3 x 17
    ((1, 512, 512), (170, 170), (170, 170), "global", "complex"),     # nb = 3: 2 x 5 x 17
    ((3, 219, 219), (73, 73), (73, 73), "local", "complex"),          # prime side
    ((1, 256, 320), (64, 80), (32, 40), "local", "magnitude"),        # overlapping, non-square
    ((2, 1024, 1024), (204, 204), (204, 204), "global", "magnitude"),  # 4 x 3 x 17
    ((1, 96, 1024), (96, 1024), (96, 1024), "global", "complex"),     # one window, longest rows
])
def test_stfd_matches_oracle(cuda, shape, win, stride, ref, output):
    import torch
    rng = np.random.default_rng(1)
    x = cfield(rng, shape)
    op = _af().ShortTimeFresnel(shape, win, stride, LAM, DX, DX, Z, phase_ref=ref, output=output)
    got = op(torch.from_numpy(x).to(cuda)).cpu().numpy()
    exp = SH.stfd(x, win[0], win[1], stride[0], stride[1], LAM, DX, DX, Z, ref, output == "magnitude")
    assert got.shape == exp.shape
    assert O.rel_l2(got, exp) < 1e-5


def test_stfd_real_input_window_lens_and_set_z(cuda):
    import torch
    rng = np.random.default_rng(2)
    x = rng.standard_normal((2, 120, 150)).astype(np.float32)
    op = _af().ShortTimeFresnel(x.shape, (40, 50), (40, 50), LAM, DX, DX, Z, phase_ref="local", output="complex",
                                skip_phase_shift=False, real_input=True)
    exp = SH.stfd(x, 40, 50, 40, 50, LAM, DX, DX, Z, "local", False, skip_phase_shift=False)
    assert O.rel_l2(op(torch.from_numpy(x).to(cuda)).cpu().numpy(), exp) < 1e-5
    op.set_z(0.4)
    exp = SH.stfd(x, 40, 50, 40, 50, LAM, DX, DX, 0.4, "local", False, skip_phase_shift=False)
    assert O.rel_l2(op(torch.from_numpy(x).to(cuda)).cpu().numpy(), exp) < 1e-5


@pytest.mark.parametrize("nb,side,nz", [(5, 510, 8), (3, 512, 4), (7, 511, 2)])
def test_subaperture_mean_magnitude_with_shift(cuda, nb, side, nz):
    """The fused Mean over the band and the per-sub-aperture fftshift (graph_builder.cc:345-347)."""
    import torch
    rng = np.random.default_rng(3)
    x = cfield(rng, (nz, side, side))
    s = side // nb
    op = _af().ShortTimeFresnel(x.shape, (s, s), (s, s), LAM, DX, DX, Z, phase_ref="global",
                                output="mean_magnitude", fftshift_windows=True)
    got = op(torch.from_numpy(x).to(cuda)).cpu().numpy()
    exp = SH.subaperture_m0(x, nb, LAM, DX, Z)
    assert O.rel_l2(got, exp) < 1e-5


def translated(sy, sx, h, w, shifts):
    def pattern(x, y):
        def g(cx, cy, s, a):
            return a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * s * s))
        return g(0.43 * w, 0.48 * h, 3.4, 1.0) + g(0.62 * w, 0.36 * h, 2.1, 0.55) + g(0.31 * w, 0.66 * h, 1.7, 0.27)
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    return np.stack([pattern(x - dx, y - dy) for dx, dy in shifts]).reshape(sy, sx, h, w).astype(np.float32)


@pytest.mark.parametrize("case", ["integer", "subpixel"])
def test_slopes_known_answers(cuda, case):
    """The reference's slope tests (shack_hartmann_test.cu:563-654) on the device, and the offsets
    against the oracle.  (The maps of these smooth images are not compared: the unit-magnitude
    cross power gives every spectral bin the same weight, and the bins where the Gaussians' spectra
    have decayed to float32 rounding carry phases that are rounding noise in any float32
    implementation; test_correlation_maps_textured compares maps where the spectrum is not.)"""
    import torch
    if case == "integer":
        shifts = [(-2, 1), (-1, 0), (0, -1), (-1, 1), (0, 0), (1, -1), (0, 1), (1, 0), (2, -1)]
        sy = sx = 3
        h = w = 32
        skip = False
    else:
        shifts = [(0.0, 0.0)] * 25
        shifts[6], shifts[18], shifts[2], shifts[22] = (0.35, -0.42), (-0.35, 0.42), (-0.60, -0.25), (0.60, 0.25)
        sy = sx = 5
        h = w = 48
        skip = True
    img = translated(sy, sx, h, w, shifts)
    kw = dict(lam=float(w), dx=1.0, dy=w / h, z=2.0)
    roi = (0.5, 0.5, 10.0, 10.0, 0.0)
    op = _af().ShackHartmannSlopes(sy, sx, h, w, roi=roi, skip_outside_pupil=skip, **kw)
    got = op(torch.from_numpy(img).to(cuda)).cpu().numpy().reshape(-1, 2)
    exp = SH.shack_hartmann_slopes(img, roi=roi, skip_outside=skip, **kw)
    # the noise-phase bins move each map by ~1e-2 of its peak, the parabolic refinement by ~3e-3 px
    assert np.abs(got - exp.reshape(-1, 2)).max() < 1e-2
    act = op.active()
    if case == "integer":
        assert all(act)
        assert np.abs(got - np.array(shifts, float)).max() < 0.03
    else:
        assert abs(got[np.array(act), 0].sum()) < 2e-6 and abs(got[np.array(act), 1].sum()) < 2e-6
        assert all(got[i, 0] == 0.0 and got[i, 1] == 0.0 for i in range(25) if not act[i])
        assert abs(got[6, 0] - 0.35) < 0.13 and abs(got[6, 1] + 0.42) < 0.13


@pytest.mark.parametrize("sy,h,w", [(3, 32, 32), (5, 34, 51), (3, 17, 40)])
def test_correlation_maps_textured(cuda, sy, h, w):
    """Maps and offsets on textured images (every spectral bin well above rounding): sample i is
    the centre image rolled by an integer offset, so each map is one sharp peak there."""
    import torch
    rng = np.random.default_rng(6)
    base = rng.standard_normal((h, w)).astype(np.float32)
    offs = [(int(rng.integers(-3, 4)), int(rng.integers(-3, 4))) for _ in range(sy * sy)]
    offs[(sy // 2) * sy + sy // 2] = (0, 0)
    img = np.stack([np.roll(base, (dy, dx), axis=(0, 1)) for dx, dy in offs]).reshape(sy, sy, h, w)
    kw = dict(lam=float(w), dx=1.0, dy=w / h, z=2.0)
    roi = (0.5, 0.5, 10.0, 10.0, 0.0)
    op = _af().ShackHartmannSlopes(sy, sy, h, w, roi=roi, skip_outside_pupil=False, **kw)
    maps = torch.empty((sy, sy, h, w), dtype=torch.float32, device=cuda)
    got = op(torch.from_numpy(img).to(cuda), maps=maps).cpu().numpy().reshape(-1, 2)
    exp, emaps = SH.shack_hartmann_slopes(img, roi=roi, skip_outside=False, return_maps=True, **kw)
    assert np.abs(maps.cpu().numpy() - emaps).max() < 2e-5
    assert np.abs(got - exp.reshape(-1, 2)).max() < 2e-3


def test_zernike_fit_device_equals_host_and_oracle(cuda):
    import torch
    from tests.test_shack_oracle import FIT_GEO, ideal_slopes
    inj = [0.18, -0.11, 0.07, 0.04, -0.03, 0.05, -0.02]
    s = sum(ideal_slopes(m, inj[m - 4]) for m in range(4, 11)).astype(np.float32)
    idx = list(range(2, 11))
    fit = _af().ZernikeFit(5, 5, (10, 10), (10, 10), 0.5, 1.0, 1.0, idx)
    assert fit.pupil_radius == 25.0
    dev = fit(torch.from_numpy(s.reshape(-1)).to(cuda)).cpu().numpy()
    host = np.array(fit.host(s.reshape(-1)), np.float32)
    assert np.array_equal(dev, host)
    exp = SH.zernike_from_slopes(s, idx, 0.5, SH.geometry(**FIT_GEO))
    assert np.abs(dev - exp).max() < 2e-5
    assert dev[0] == 0.0 and dev[1] == 0.0


def test_zernike_phase_correct_phase_wrap(cuda):
    import torch
    af = _af()
    idx = [2, 4, 5, 7, 10]
    c = np.array([0.3, -1.2, 0.4, 0.25, -0.6], np.float32)
    ph = af.zernike_phase(torch.from_numpy(c).to(cuda), idx, 96, 130)
    exp = SH.zernike_phase(c.astype(np.float64), idx, 96, 130)
    assert np.abs(ph.cpu().numpy() - exp).max() < 1e-5
    rng = np.random.default_rng(4)
    x = cfield(rng, (3, 96, 130))
    got = af.correct_phase(torch.from_numpy(x).to(cuda), ph).cpu().numpy()
    assert O.rel_l2(got, SH.correct_phase(x, ph.cpu().numpy().astype(np.float64))) < 1e-6
    xr = rng.standard_normal((2, 96, 130)).astype(np.float32)
    got = af.correct_phase(torch.from_numpy(xr).to(cuda), ph).cpu().numpy()
    assert O.rel_l2(got, SH.correct_phase(xr, ph.cpu().numpy().astype(np.float64))) < 1e-6
    v = (rng.standard_normal(10000) * 20).astype(np.float32)
    assert np.array_equal(af.wrap2pi(torch.from_numpy(v).to(cuda)).cpu().numpy(), SH.wrap2pi(v))


def aberrated_planes(nz, side, a4, seed=5):
    """Band planes whose one-FFT Fresnel image is a few point scatterers seen through a defocus
    aberration a4 Z4 (radians) over the pupil: planes = conj(lens) IFFT(points) exp(i a4 Z4)."""
    rng = np.random.default_rng(seed)
    lens = SH.stfd_input_lens(side, side, side, side, LAM, Z, DX, DX, "global")
    y, x = (np.mgrid[0:side, 0:side] - (side - 1) / 2.0) / (side / 2.0)
    ab = np.exp(1j * a4 * SH.zernike_value(4, x, y))
    out = np.empty((nz, side, side), np.complex64)
    for k in range(nz):
        pts = np.zeros((side, side), np.complex128)
        for _ in range(6):
            pts[rng.integers(side // 4, 3 * side // 4), rng.integers(side // 4, 3 * side // 4)] = np.exp(
                2j * math.pi * rng.random()) * (1.0 + rng.random())
        out[k] = np.conj(lens) * np.fft.ifft2(pts) * ab * side
    return out


@pytest.mark.parametrize("nb,side,n_iter", [(5, 510, 1), (3, 512, 2)])
def test_autofocus_chain_matches_oracle_and_recovers_defocus(cuda, nb, side, n_iter):
    """The whole pass chain against the oracle; the injected defocus comes back as A4 and a second
    measurement of the corrected planes finds almost none left."""
    import torch
    af = _af()
    a4 = 4.0
    planes = aberrated_planes(4, side, a4)
    idx = [4, 5, 6]
    cfg = SH.AutofocusConfig(nb, LAM, DX, Z, idx)
    op = af.Autofocus(4, side, side, nb, LAM, DX, Z, indexes=idx, n_iter=n_iter)
    dev = torch.from_numpy(planes).to(cuda)
    corrected = op(dev)
    m0, sl, coeff = op.m0().cpu().numpy(), op.slopes().cpu().numpy(), op.coefficients().cpu().numpy()
    cur, total_c, total_ph = planes.astype(np.complex128), np.zeros(len(idx)), 0.0
    for _ in range(n_iter):
        em0, esl, ec, eph, cur = SH.autofocus(cur, cfg)
        total_c, total_ph = total_c + ec, total_ph + eph
    assert O.rel_l2(m0, em0) < 1e-4
    spp = LAM / ((side // nb) * DX)
    assert np.abs(sl - esl).max() / spp < 2e-3
    assert np.abs(coeff - total_c).max() < 1e-3 * max(1.0, np.abs(total_c).max())
    assert O.rel_l2(op.phase().cpu().numpy(), total_ph) < 1e-3
    assert O.rel_l2(corrected.cpu().numpy(), cur) < 1e-3
    # physics: the fit sees the injected defocus, and the corrected planes carry little of it
    assert abs(coeff[0] - a4) < 0.35 * a4
    again = af.Autofocus(4, side, side, nb, LAM, DX, Z, indexes=idx)
    again(corrected)
    assert abs(again.coefficients().cpu().numpy()[0]) < 0.35 * abs(coeff[0])


def test_autofocus_without_orders_passes_planes_through(cuda):
    import torch
    planes = aberrated_planes(2, 255, 2.0)
    op = _af().Autofocus(2, 255, 255, 5, LAM, DX, Z, indexes=[])
    dev = torch.from_numpy(planes).to(cuda)
    out = op(dev)
    assert torch.equal(out, dev)
    assert op.slopes().shape == (5, 5, 2)


def test_validation_messages(cuda):
    import holoflow_b200 as hf
    af = _af()
    with pytest.raises(hf.HfError, match="autofocus_nb_subaps must be odd"):
        af.Autofocus(2, 64, 64, 4, LAM, DX, Z)
    with pytest.raises(hf.HfError, match="too large for the current frame size"):
        af.Autofocus(2, 64, 64, 65, LAM, DX, Z)
    with pytest.raises(hf.HfError, match="only Noll indexes 2..10"):
        af.ZernikeFit(5, 5, (10, 10), (10, 10), 0.5, 1.0, 1.0, [11])
    with pytest.raises(hf.HfError, match="indexes must be unique"):
        af.ZernikeFit(5, 5, (10, 10), (10, 10), 0.5, 1.0, 1.0, [4, 4])
    with pytest.raises(hf.HfError, match="dx must equal dy"):
        af.ShortTimeFresnel((1, 64, 64), (32, 32), (32, 32), LAM, DX, 2 * DX, Z)
    with pytest.raises(hf.HfError, match="must be odd for an unambiguous center"):
        af.ShackHartmannSlopes(4, 5, 32, 32, LAM, DX, DX, Z)
    with pytest.raises(hf.HfError, match="window sides must be in 2..1024"):
        af.ShortTimeFresnel((1, 2048, 2048), (2048, 2048), (2048, 2048), LAM, DX, DX, Z)


def test_full_pairwise_known_answers(cuda):
    """FullPairwise slope recovery (shack_hartmann_slopes_full_pairwise.cuh) on the device: the
    reference's star-graph / batch-size and periodic-peak tests (shack_hartmann_test.cu:656-739),
    and the oracle's restatement."""
    import torch
    shifts = [(-2, 1), (-1, 0), (0, -1), (-1, 1), (0, 0), (1, -1), (0, 1), (1, 0), (2, -1)]
    img = translated(3, 3, 40, 40, shifts)
    kw = dict(lam=40.0, dx=1.0, dy=1.0, z=2.0)
    roi = (0.5, 0.5, 10.0, 10.0, 0.0)
    dev = torch.from_numpy(img).to(cuda)
    single = _af().ShackHartmannSlopes(3, 3, 40, 40, roi=roi, skip_outside_pupil=False, **kw)(dev).cpu().numpy()
    single = single.reshape(-1, 2)
    exp = SH.full_pairwise_slopes(img, roi=roi, skip_outside=False, **kw).reshape(-1, 2)
    edges = 9 * 8 // 2
    base = None
    for batch in (1, 5, 32, edges + 11):
        op = _af().ShackHartmannSlopes(3, 3, 40, 40, roi=roi, skip_outside_pupil=False, mode="full_pairwise",
                                       pair_batch_size=batch, **kw)
        got = op(dev).cpu().numpy().reshape(-1, 2)
        if base is None:
            base = got
        assert np.abs(got - base).max() < 2e-6, batch          # batch-invariant
        assert np.abs(got - np.array(shifts, float)).max() < 0.035
        assert np.abs(got - single).max() < 0.025              # star vs complete graph
        assert abs(got[:, 0].sum()) < 4e-6 and abs(got[:, 1].sum()) < 4e-6
        assert np.abs(got - exp).max() < 1e-2                  # against the oracle
    # periodic-peak and sub-pixel conventions on a 1 x 3 grid (an even-sized grid is allowed too)
    sh = [(-9.0, 7.0), (-0.40, 0.35), (9.0, -7.0)]
    img = translated(1, 3, 48, 48, sh)
    op = _af().ShackHartmannSlopes(1, 3, 48, 48, roi=roi, skip_outside_pupil=False, mode="full_pairwise",
                                   pair_batch_size=2, lam=48.0, dx=1.0, dy=1.0, z=2.0)
    s = op(torch.from_numpy(img).to(cuda)).cpu().numpy().reshape(-1)
    mx, my = sum(v[0] for v in sh) / 3.0, sum(v[1] for v in sh) / 3.0
    for i, (dx, dy) in enumerate(sh):
        assert abs(s[2 * i] - (dx - mx)) < 0.08 and abs(s[2 * i + 1] - (dy - my)) < 0.08
    assert abs((s[0] - s[4]) + 18.0) < 0.2 and abs((s[1] - s[5]) - 14.0) < 0.2
    op2 = _af().ShackHartmannSlopes(2, 2, 32, 32, roi=roi, skip_outside_pupil=False, mode="full_pairwise", **kw)
    assert op2(torch.zeros((2, 2, 32, 32), device=cuda)).shape == (2, 2, 2)
    with pytest.raises(Exception, match="at least two active subapertures"):
        _af().ShackHartmannSlopes(1, 1, 32, 32, roi=roi, skip_outside_pupil=False, mode="full_pairwise", **kw)


@pytest.mark.parametrize("sy,h,w,skip", [(5, 34, 51, True), (3, 64, 64, False)])
def test_full_pairwise_textured_vs_oracle(cuda, sy, h, w, skip):
    """FullPairwise slopes on textured sub-aperture images (sharp peaks) against the oracle."""
    import torch
    rng = np.random.default_rng(7 + sy)
    base = rng.standard_normal((h, w)).astype(np.float32)
    offs = [(int(rng.integers(-3, 4)), int(rng.integers(-3, 4))) for _ in range(sy * sy)]
    img = np.stack([np.roll(base, (dy, dx), axis=(0, 1)) for dx, dy in offs]).reshape(sy, sy, h, w)
    kw = dict(lam=float(w), dx=1.0, dy=w / h, z=2.0)
    roi = (0.5, 0.5, 10.0, 10.0, 0.0)
    op = _af().ShackHartmannSlopes(sy, sy, h, w, roi=roi, skip_outside_pupil=skip, mode="full_pairwise",
                                   pair_batch_size=7, **kw)
    got = op(torch.from_numpy(img).to(cuda)).cpu().numpy().reshape(-1, 2)
    exp = SH.full_pairwise_slopes(img, roi=roi, skip_outside=skip, **kw).reshape(-1, 2)
    assert np.abs(got - exp).max() < 2e-3


def test_full_pairwise_slopes_node(cuda):
    """The ShackHartmannSlopes node in "full_pairwise" mode gives the binding's slopes; map output
    is refused as in the reference (shack_hartmann_slopes.cu:343-345)."""
    import torch
    from holoflow_b200 import nodes as N
    rng = np.random.default_rng(3)
    base = rng.standard_normal((40, 40)).astype(np.float32)
    img = np.stack([np.roll(base, (int(rng.integers(-2, 3)), int(rng.integers(-2, 3))), axis=(0, 1))
                    for _ in range(9)]).reshape(1, 3, 3, 40, 40)
    dev = torch.from_numpy(img).to(cuda)
    sl = {"lambda": 40.0, "dx": 1.0, "dy": 1.0, "z": 2.0, "subaperture_height": 40, "subaperture_width": 40,
          "stride_y": 40, "stride_x": 40, "mode": "full_pairwise", "pair_batch_size": 4,
          "skip_subapertures_outside_pupil": False,
          "correlation_roi": {"cx": 0.5, "cy": 0.5, "rx": 10.0, "ry": 10.0, "angle": 0.0}}
    (slopes,) = N.run_sync_factory("ShackHartmannSlopes", sl, [dev])
    op = _af().ShackHartmannSlopes(3, 3, 40, 40, roi=(0.5, 0.5, 10.0, 10.0, 0.0), skip_outside_pupil=False,
                                   mode="full_pairwise", pair_batch_size=4, lam=40.0, dx=1.0, dy=1.0, z=2.0)
    assert torch.equal(slopes.reshape(3, 3, 2), op(dev[0]))
    with pytest.raises(Exception, match="FullPairwise correlation-map output is not supported"):
        N.run_sync_factory("ShackHartmannSlopes", {**sl, "output_xcorr_maps": True}, [dev])


def test_autofocus_as_nodes(cuda):
    """ShortTimeFresnelDiffraction -> Mean -> FFTShiftNp -> ShackHartmannSlopes -> (host)
    ZernikeFromSlopes -> ZernikePhase -> CorrectPhase, driven as the reference's graph wires them
    (graph_builder.cc:336-451), against the oracle chain."""
    import torch
    from holoflow_b200 import nodes as N
    nb, side, nz = 5, 510, 4
    s = side // nb
    planes = aberrated_planes(nz, side, 3.0, seed=8)
    dev = torch.from_numpy(planes).to(cuda)
    stfd = {"lambda": LAM, "dx": DX, "dy": DX, "z": Z, "win_h": s, "win_w": s, "stride_y": s, "stride_x": s,
            "phase_ref": "GLOBAL", "output_magnitude": True}
    (mag,) = N.run_sync_factory("ShortTimeFresnelDiffraction", stfd, [dev.reshape(1, nz, side, side)])
    assert tuple(mag.shape) == (1, nz, nb, nb, s, s)
    (m0,) = N.run_sync_factory("Mean", {"axes": [1], "keepdims": False}, [mag])
    (m0,) = N.run_sync_factory("FFTShiftNp", {"axes": [-2, -1]}, [m0])
    assert O.rel_l2(m0.cpu().numpy()[0], SH.subaperture_m0(planes, nb, LAM, DX, Z)) < 1e-5
    sl = {"lambda": LAM, "dx": DX, "dy": DX, "z": Z, "subaperture_height": s, "subaperture_width": s, "stride_y": s,
          "stride_x": s, "correlation_roi": {"cx": 0.5, "cy": 0.5, "rx": 0.5, "ry": 0.5, "angle": 0.0}}
    (slopes,) = N.run_sync_factory("ShackHartmannSlopes", sl, [m0])
    idx = [4, 5, 6]
    fit = {"indexes": idx, "lambda": LAM, "dx": DX, "dy": DX, "subaperture_height": s, "subaperture_width": s,
           "stride_y": s, "stride_x": s}
    (coeffs,) = N.run_sync_factory("ZernikeFromSlopes", fit, [slopes.cpu()])
    (dcoeffs,) = N.run_sync_factory("ZernikeFromSlopes", fit, [slopes])
    assert torch.equal(coeffs, dcoeffs.cpu())  # host and device fits agree bit for bit
    _, esl, ec, eph, ecor = SH.autofocus(planes.astype(np.complex128), SH.AutofocusConfig(nb, LAM, DX, Z, idx))
    spp = LAM / (s * DX)
    assert np.abs(slopes.cpu().numpy()[0] - esl).max() / spp < 2e-3
    assert np.abs(coeffs.numpy().reshape(-1) - ec).max() < 1e-3 * max(1.0, np.abs(ec).max())
    zp = {"indexes": idx, "ny": side, "nx": side, "output": "Device"}
    (phase,) = N.run_sync_factory("ZernikePhase", zp, [dcoeffs.reshape(-1)])
    (host_phase,) = N.run_sync_factory("ZernikePhase", dict(zp, output="Host"), [coeffs.reshape(-1)])
    assert np.abs(phase.cpu().numpy() - host_phase.numpy()).max() < 1e-5
    (cor,) = N.run_sync_factory("CorrectPhase", {}, [dev, phase])
    assert O.rel_l2(cor.cpu().numpy(), ecor) < 1e-3
    (w,) = N.run_sync_factory("Wrap2Pi", {}, [phase])
    assert np.array_equal(w.cpu().numpy(), SH.wrap2pi(phase.cpu().numpy()))


def doppler_frames(T, side, k0, a4, seed=9):
    """float32 frames x_t = Re(A exp(2 pi i k0 t / T)): the band DFT at bin k0 is (T / 2) A, with
    A = conj(Fresnel lens) IFFT(point scatterers) exp(i a4 Z4), so the Fresnel image of the band
    is the scatterers seen through a defocus aberration."""
    rng = np.random.default_rng(seed)
    lens = O.fresnel_lens(side, side, LAM, Z, DX)
    y, x = (np.mgrid[0:side, 0:side] - (side - 1) / 2.0) / (side / 2.0)
    pts = np.zeros((side, side), np.complex128)
    for _ in range(8):
        pts[rng.integers(side // 4, 3 * side // 4), rng.integers(side // 4, 3 * side // 4)] = np.exp(
            2j * math.pi * rng.random()) * (1.0 + rng.random())
    A = np.conj(lens) * np.fft.ifft2(pts) * np.exp(1j * a4 * SH.zernike_value(4, x, y)) * side * 100.0
    t = np.arange(T)[:, None, None]
    return np.real(A[None] * np.exp(2j * math.pi * k0 * t / T)).astype(np.float32)


@pytest.mark.parametrize("form,n_iter", [(0, 1), (1, 1), (1, 2)])
def test_pipeline_with_autofocus(cuda, form, n_iter):
    """The fused pipeline with autofocus on (graph_builder.cc:139-153): each window's band planes
    are measured and corrected before the Fresnel lens; moments and coefficients against the
    oracle, and the correction sharpens the image."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    T, side, k0, a4, nb = 32, 256, 5, 4.0, 5
    frames = doppler_frames(T, side, k0, a4)
    ring = torch.from_numpy(frames).to(cuda)
    base = dict(height=side, width=side, frames=T, hop=T, z_begin=3, z_end=9, input_dtype=hf.HF_F32, lam=LAM,
                pitch=DX, z=Z, form=form, max_batch=1)
    af = dict(autofocus_nb_subaps=nb, autofocus_orders=(4, 5, 6), autofocus_n_iter=n_iter)
    p = pl.Pipeline(pl.PipelineConfig(**base, **af))
    got = p.run(ring, T, 0, 1).cpu().numpy()[0]
    assert p.status() == 0
    coeff = p.autofocus_coefficients(0).cpu().numpy()
    ocfg = O.PathConfig(side, side, T, T, 3, 9, lam=LAM, pitch=DX, z=Z,
                        autofocus=dict(nb=nb, orders=[4, 5, 6], n_iter=n_iter))
    exp = O.reconstruct_window(frames.astype(np.float64), ocfg)
    _, ecoeff = O.autofocus_planes(O.band_planes(frames.astype(np.float64), ocfg), ocfg)
    assert np.abs(coeff - ecoeff).max() < 1e-3 * max(1.0, np.abs(ecoeff).max())
    tol = 1e-4 if form == 0 else 1e-3
    for m in range(3):
        assert O.rel_l2(got[m], exp[m]) < tol, m
    assert abs(coeff[0] - a4) < 0.35 * a4
    # the corrected image is sharper: more of M0's energy in its brightest pixels
    plain = pl.Pipeline(pl.PipelineConfig(**base)).run(ring, T, 0, 1).cpu().numpy()[0, 0]
    def peak_share(img):
        v = np.sort(img.ravel())[::-1]
        return v[:64].sum() / v.sum()
    assert peak_share(got[0]) > 1.2 * peak_share(plain)


def test_pipeline_with_autofocus_tensor_core_band(cuda):
    """uint16 frames in the chosen form: the tensor-core band pass stores the raw band planes
    for the autofocus (its lens and row FFT move to the per-window row pass)."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    T, side, k0, a4, nb = 64, 256, 9, 4.0, 5
    fr = doppler_frames(T, side, k0, a4)
    frames = np.clip(np.rint(2048.0 + fr * (1800.0 / np.abs(fr).max())), 0, 4095).astype(np.uint16)
    ring = torch.from_numpy(frames.view(np.int16)).to(cuda)
    cfg = pl.PipelineConfig(height=side, width=side, frames=T, hop=T, z_begin=6, z_end=13, input_dtype=hf.HF_U16,
                            lam=LAM, pitch=DX, z=Z, form=1, max_batch=1, autofocus_nb_subaps=nb,
                            autofocus_orders=(4, 5, 6))
    p = pl.Pipeline(cfg)
    got = p.run(ring, T, 0, 1).cpu().numpy()[0]
    assert p.status() == 0
    coeff = p.autofocus_coefficients(0).cpu().numpy()
    ocfg = O.PathConfig(side, side, T, T, 6, 13, lam=LAM, pitch=DX, z=Z, autofocus=dict(nb=nb, orders=[4, 5, 6]))
    exp = O.reconstruct_window(frames.astype(np.float64), ocfg)
    _, ecoeff = O.autofocus_planes(O.band_planes(frames.astype(np.float64), ocfg), ocfg)
    assert np.abs(coeff - ecoeff).max() < 1e-3 * max(1.0, np.abs(ecoeff).max())
    for m in range(3):
        assert O.rel_l2(got[m], exp[m]) < 1e-3, m
    assert abs(coeff[0] - a4) < 0.35 * a4


def test_doppler_moments_node_with_autofocus(cuda):
    """The DopplerMoments node with the reference's autofocus settings names runs the same plan as
    PipelineConfig(autofocus_*): identical moments."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import nodes as N
    from holoflow_b200 import pipeline as pl
    T, side = 32, 256
    frames = doppler_frames(T, side, 5, 4.0)
    dev = torch.from_numpy(frames).to(cuda)
    s = {"time_z_begin": 3, "time_z_end": 9, "propagation": "fresnel", "lambda": LAM, "dx": DX, "z": Z,
         "input_format": "f32", "form": "chosen", "autofocus_enabled": True, "autofocus_nb_subaps": 5,
         "autofocus_zernike_orders": [4, 5, 6]}
    (got,) = N.run_sync_factory("DopplerMoments", s, [dev.reshape(1, T, side, side)])
    cfg = pl.PipelineConfig(height=side, width=side, frames=T, hop=T, z_begin=3, z_end=9, input_dtype=hf.HF_F32,
                            lam=LAM, pitch=DX, z=Z, form=1, max_batch=1, autofocus_nb_subaps=5,
                            autofocus_orders=(4, 5, 6))
    exp = pl.Pipeline(cfg).run(dev, T, 0, 1)
    assert torch.equal(got, exp)


@pytest.mark.parametrize("form", [0, 1])
def test_pipeline_with_autofocus_flatfield(cuda, form):
    """pp_flatfield on the sub-aperture images (graph_builder.cc:348-352), sigma from the cutoff
    period and the one-FFT Fresnel output pitch, in the fused pipeline and the standalone pass."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import autofocus as af
    from holoflow_b200 import pipeline as pl
    T, side, per = 32, 256, 2e-3
    frames = doppler_frames(T, side, 5, 4.0)
    ring = torch.from_numpy(frames).to(cuda)
    cfg = pl.PipelineConfig(height=side, width=side, frames=T, hop=T, z_begin=3, z_end=9, input_dtype=hf.HF_F32,
                            lam=LAM, pitch=DX, z=Z, form=form, max_batch=1, autofocus_nb_subaps=5,
                            autofocus_orders=(4, 5, 6), autofocus_flatfield_period=per)
    p = pl.Pipeline(cfg)
    got = p.run(ring, T, 0, 1).cpu().numpy()[0]
    coeff = p.autofocus_coefficients(0).cpu().numpy()
    ocfg = O.PathConfig(side, side, T, T, 3, 9, lam=LAM, pitch=DX, z=Z,
                        autofocus=dict(nb=5, orders=[4, 5, 6], flatfield_period=per))
    planes = O.band_planes(frames.astype(np.float64), ocfg)
    _, ecoeff = O.autofocus_planes(planes, ocfg)
    assert np.abs(coeff - ecoeff).max() < 1e-3 * max(1.0, np.abs(ecoeff).max())
    exp = O.reconstruct_window(frames.astype(np.float64), ocfg)
    for m in range(3):
        assert O.rel_l2(got[m], exp[m]) < (1e-4 if form == 0 else 1e-3), m
    # the standalone pass: the flattened sub-aperture images against the oracle
    op = af.Autofocus(planes.shape[0], side, side, 5, LAM, DX, Z, indexes=[4, 5, 6], flatfield_period=per)
    op(torch.from_numpy(planes.astype(np.complex64)).to(cuda))
    acfg = SH.AutofocusConfig(5, LAM, DX, Z, [4, 5, 6], flatfield_period=per)
    em0 = SH.subaperture_flatfield(SH.subaperture_m0(planes, 5, LAM, DX, Z), acfg)
    assert O.rel_l2(op.m0().cpu().numpy(), em0) < 5e-5  # the high-pass leaves a smaller norm


def drifting_doppler_frames(n_frames, T, side, k0, a4_0, a4_rate, seed=9):
    """Frames x_t = Re(A(t) exp(2 pi i k0 t / T)) whose defocus drifts, a4(t) = a4_0 + a4_rate t:
    every window sees a slightly different aberration, so a sliding average differs from one window."""
    rng = np.random.default_rng(seed)
    lens = O.fresnel_lens(side, side, LAM, Z, DX)
    y, x = (np.mgrid[0:side, 0:side] - (side - 1) / 2.0) / (side / 2.0)
    pts = np.zeros((side, side), np.complex128)
    for _ in range(8):
        pts[rng.integers(side // 4, 3 * side // 4), rng.integers(side // 4, 3 * side // 4)] = np.exp(
            2j * math.pi * rng.random()) * (1.0 + rng.random())
    base = np.conj(lens) * np.fft.ifft2(pts) * side * 100.0
    z4 = SH.zernike_value(4, x, y)
    out = np.empty((n_frames, side, side), np.float32)
    for t in range(n_frames):
        out[t] = np.real(base * np.exp(1j * (a4_0 + a4_rate * t) * z4) * np.exp(2j * math.pi * k0 * t / T))
    return out


@pytest.mark.parametrize("form,n,pairwise", [(0, 3, False), (1, 3, False), (1, 5, False), (1, 3, True)])
def test_pipeline_sliding_correction_of_the_delayed_window(cuda, form, n, pairwise):
    """pp_accumulation = n (graph_builder.cc:128-153, 348): window w's sub-aperture images are
    averaged causally over the last n windows and the fit corrects window w - (n - 1) / 2, which
    the plan keeps across calls (the dual reader's delayed window); the first (n - 1) / 2 outputs
    are zero images.  Two calls (3 + 4 windows) against the oracle's sequence, optionally with the
    full-pairwise slopes."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    T, hop, side, nb = 32, 8, 256, 5
    nwin = 7
    frames = drifting_doppler_frames(T + hop * (nwin - 1), T, side, 5, 3.0, 0.02)
    ring = torch.from_numpy(frames).to(cuda)
    cfg = pl.PipelineConfig(height=side, width=side, frames=T, hop=hop, z_begin=3, z_end=9, input_dtype=hf.HF_F32,
                            lam=LAM, pitch=DX, z=Z, form=form, max_batch=4, autofocus_nb_subaps=nb,
                            autofocus_orders=(4, 5, 6), autofocus_pp_accumulation=n,
                            autofocus_full_pairwise=int(pairwise))
    p = pl.Pipeline(cfg)
    got = np.concatenate([p.run(ring, frames.shape[0], 0, 3).cpu().numpy(),
                          p.run(ring, frames.shape[0], 3 * hop, 4).cpu().numpy()])
    assert p.status() == 0
    ocfg = O.PathConfig(side, side, T, hop, 3, 9, lam=LAM, pitch=DX, z=Z,
                        autofocus=dict(nb=nb, orders=[4, 5, 6], pp_accumulation=n, full_pairwise=pairwise))
    exp = O.reconstruct_sequence([frames[w * hop: w * hop + T].astype(np.float64) for w in range(nwin)], ocfg)
    d = (n - 1) // 2
    tol = 1e-4 if form == 0 else 1e-3
    for w in range(nwin):
        if w < d:
            assert not got[w].any(), w
            continue
        for m in range(3):
            assert O.rel_l2(got[w, m], exp[w][m]) < tol, (w, m, O.rel_l2(got[w, m], exp[w][m]))
    # a new sequence starts over: the first d outputs are zero again and the rest repeat
    p.autofocus_reset()
    again = p.run(ring, frames.shape[0], 0, 3).cpu().numpy()
    assert np.array_equal(again, got[:3])


def test_pipeline_sliding_correction_validation(cuda):
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    cfg = dict(height=256, width=256, frames=32, hop=8, z_begin=3, z_end=9, input_dtype=hf.HF_F32, lam=LAM, pitch=DX,
               z=Z, max_batch=2, autofocus_nb_subaps=5, autofocus_orders=(4,))
    with pytest.raises(hf.HfError, match="only supports one autofocus iteration"):
        pl.Pipeline(pl.PipelineConfig(**cfg, autofocus_pp_accumulation=3, autofocus_n_iter=2))
