"""Pins the autofocus oracle to the reference's known-answer tests
(test/holotask/shack_hartmann_test.cu): integer and sub-pixel translations recovered as slopes,
the active-sample gauge, and injected Zernike modes recovered without leakage.  CPU only."""
import math

import numpy as np
import pytest

from oracle import shack as SH


def pattern(x, y, w, h):
    """Three Gaussians (shack_hartmann_test.cu:69-80)."""
    def g(cx, cy, s, a):
        return a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * s * s))
    return g(0.43 * w, 0.48 * h, 3.4, 1.0) + g(0.62 * w, 0.36 * h, 2.1, 0.55) + g(0.31 * w, 0.66 * h, 1.7, 0.27)


def translated(sy, sx, h, w, shifts):
    """translated_subapertures (shack_hartmann_test.cu:82-98): sample i is the pattern moved by
    shifts[i] = (dx, dy)."""
    img = np.zeros((sy * sx, h, w))
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    for i, (dx, dy) in enumerate(shifts):
        img[i] = pattern(x - dx, y - dy, w, h)
    return img.reshape(sy, sx, h, w).astype(np.float32)


def slope_args(h, w):
    """slope_settings (shack_hartmann_test.cu:100-117): one pixel of shift is one unit of slope."""
    return dict(lam=float(w), dx=1.0, dy=w / h, z=2.0, roi=(0.5, 0.5, 10.0, 10.0, 0.0))


def active_5x5(sy, sx):
    x, y = (sx - 2.0) / 2.5, (sy - 2.0) / 2.5
    return x * x + y * y <= 1.0


def test_integer_translations_and_centre_peak():
    """RecoversSignedIntegerTranslationsAndRawMaps (shack_hartmann_test.cu:563-615)."""
    shifts = [(-2, 1), (-1, 0), (0, -1), (-1, 1), (0, 0), (1, -1), (0, 1), (1, 0), (2, -1)]
    img = translated(3, 3, 32, 32, shifts)
    slopes, maps = SH.shack_hartmann_slopes(img, skip_outside=False, return_maps=True, **slope_args(32, 32))
    for i, (dx, dy) in enumerate(shifts):
        assert abs(slopes.reshape(-1, 2)[i, 0] - dx) < 0.03
        assert abs(slopes.reshape(-1, 2)[i, 1] - dy) < 0.03
    cx, cy = SH.peak_shift(maps[1, 1])
    assert abs(cx) < 1e-6 and abs(cy) < 1e-6


def test_subpixel_refinement_and_active_gauge():
    """PreservesSubpixelRefinementAndActiveGauge (shack_hartmann_test.cu:617-654)."""
    shifts = [(0.0, 0.0)] * 25
    shifts[6], shifts[18] = (0.35, -0.42), (-0.35, 0.42)
    shifts[2], shifts[22] = (-0.60, -0.25), (0.60, 0.25)
    img = translated(5, 5, 48, 48, shifts)
    s = SH.shack_hartmann_slopes(img, skip_outside=True, **slope_args(48, 48)).reshape(-1)
    sx = sy = 0.0
    for iy in range(5):
        for ix in range(5):
            i = iy * 5 + ix
            if active_5x5(iy, ix):
                sx += s[2 * i]
                sy += s[2 * i + 1]
            else:
                assert s[2 * i] == 0.0 and s[2 * i + 1] == 0.0
    assert abs(sx) < 2e-6 and abs(sy) < 2e-6
    assert abs(s[12] - 0.35) < 0.13 and abs(s[13] + 0.42) < 0.13
    assert abs(s[36] + 0.35) < 0.13 and abs(s[37] - 0.42) < 0.13


def ideal_slopes(mode, coeff_m):
    """ideal_slopes (shack_hartmann_test.cu:330-362): mean-removed derivatives over the active
    5 x 5 samples, divided by the 25-pixel pupil radius."""
    vals, act = np.zeros((25, 2)), np.zeros(25, bool)
    for iy in range(5):
        for ix in range(5):
            if active_5x5(iy, ix):
                i = iy * 5 + ix
                act[i] = True
                dx, dy = SH.zernike_derivative(mode, (ix - 2.0) / 2.5, (iy - 2.0) / 2.5)
                vals[i] = (dx / 25.0, dy / 25.0)
    out = np.zeros((25, 2))
    out[act] = coeff_m * (vals[act] - vals[act].mean(0))
    return out


FIT_GEO = dict(sy=5, sx=5, sub_h=10, sub_w=10, stride_y=10, stride_x=10, dy=1.0, dx=1.0, skip_outside=True)


@pytest.mark.parametrize("injected", range(4, 11))
def test_each_observable_mode_without_leakage(injected):
    """RecoversEachObservableModeWithoutTipTiltOrLeakage (shack_hartmann_test.cu:740-759)."""
    geo = SH.geometry(**FIT_GEO)
    idx = list(range(2, 11))
    c = SH.zernike_from_slopes(ideal_slopes(injected, 0.7), idx, 0.5, geo)
    expected = 0.7 * 2.0 * math.pi / 0.5
    assert c[0] == 0.0 and c[1] == 0.0
    for mode in range(4, 11):
        want = expected if mode == injected else 0.0
        assert abs(c[mode - 2] - want) < 2e-5, (injected, mode)


def test_combined_modes_match_injection():
    """ObservableCoefficientsAndPhaseMatchCenterGauge (shack_hartmann_test.cu:761-801)."""
    inj = [0.18, -0.11, 0.07, 0.04, -0.03, 0.05, -0.02]
    s = sum(ideal_slopes(m, inj[m - 4]) for m in range(4, 11))
    c = SH.zernike_from_slopes(s, list(range(2, 11)), 0.5, SH.geometry(**FIT_GEO))
    rpm = 2.0 * math.pi / 0.5
    for m in range(7):
        assert abs(c[m + 2] - inj[m] * rpm) < 5e-5


def test_geometry_pupil_and_active_set():
    geo = SH.geometry(**FIT_GEO)
    assert geo.pupil_radius == 25.0
    assert [bool(a) for a in geo.active] == [active_5x5(i // 5, i % 5) for i in range(25)]


def test_stfd_single_window_is_fresnel_and_grid_counts():
    """A window covering the whole field with the global frame is the one-FFT Fresnel transform
    of the field; the window counts follow (H - h) / stride + 1."""
    rng = np.random.default_rng(0)
    f = rng.standard_normal((2, 24, 30)) + 1j * rng.standard_normal((2, 24, 30))
    out = SH.stfd(f, 24, 30, 24, 30, 850e-9, 12e-6, 12e-6, 0.3, "global", output_magnitude=False)
    lens = SH.stfd_input_lens(24, 30, 24, 30, 850e-9, 0.3, 12e-6, 12e-6, "global")
    assert np.allclose(out[:, 0, 0], np.fft.fft2(f * lens))
    assert SH.stfd_grid(100, 90, 20, 30, 20, 15) == (5, 5)


def test_wrap_and_defocus():
    w = SH.wrap2pi(np.array([-1.0, 7.0, 0.5], np.float32))
    assert np.all((w >= 0) & (w < 2 * math.pi + 1e-6))
    d_inv, z_new, dz = SH.defocus_z(0.0, 850e-9, 0.3, 3e-3)
    assert d_inv == 0.0 and z_new == pytest.approx(0.3) and dz == pytest.approx(0.0, abs=1e-9)


# ---- FullPairwise (graph-Laplacian) slope recovery --------------------------------------------
def test_full_pairwise_matches_star_graph_signs_gauge():
    """MatchesStarGraphSignsGaugeAndBatchSizes (shack_hartmann_test.cu:656-710): integer
    translations recovered within 0.035 px, within 0.025 px of the single-reference mode, zero sum."""
    shifts = [(-2, 1), (-1, 0), (0, -1), (-1, 1), (0, 0), (1, -1), (0, 1), (1, 0), (2, -1)]
    img = translated(3, 3, 40, 40, shifts)
    single = SH.shack_hartmann_slopes(img, skip_outside=False, **slope_args(40, 40)).reshape(-1, 2)
    full = SH.full_pairwise_slopes(img, skip_outside=False, **slope_args(40, 40)).reshape(-1, 2)
    for i, (dx, dy) in enumerate(shifts):
        assert abs(full[i, 0] - dx) < 0.035 and abs(full[i, 1] - dy) < 0.035
        assert abs(full[i, 0] - single[i, 0]) < 0.025 and abs(full[i, 1] - single[i, 1]) < 0.025
    assert abs(full[:, 0].sum()) < 4e-6 and abs(full[:, 1].sum()) < 4e-6


def test_full_pairwise_subpixel_and_periodic_peaks():
    """PreservesSubpixelAndPeriodicPeakConventions (shack_hartmann_test.cu:712-739): translations
    up to the unambiguous periodic interval (an 18-pixel endpoint-to-endpoint edge) and sub-pixel
    shifts, compared in the zero-mean gauge."""
    shifts = [(-9.0, 7.0), (-0.40, 0.35), (9.0, -7.0)]
    img = translated(1, 3, 48, 48, shifts)
    s = SH.full_pairwise_slopes(img, skip_outside=False, **slope_args(48, 48)).reshape(-1)
    mx = sum(v[0] for v in shifts) / 3.0
    my = sum(v[1] for v in shifts) / 3.0
    for i, (dx, dy) in enumerate(shifts):
        assert abs(s[2 * i] - (dx - mx)) < 0.08 and abs(s[2 * i + 1] - (dy - my)) < 0.08
    assert abs((s[0] - s[4]) + 18.0) < 0.2 and abs((s[1] - s[5]) - 14.0) < 0.2


def test_full_pairwise_noiseless_defocus_matches_single_reference():
    """NoiselessDefocusMatchesSingleReferenceAndZernikeFit (shack_hartmann_test.cu:803-850): a
    defocus wavefront's sub-aperture shifts on the active 5 x 5 samples; both modes agree to
    0.025 px and inactive samples are 0."""
    h = w = 48
    radius = 0.5 * 5 * w
    coeff_m = radius / (4.0 * math.sqrt(3.0) * 0.4)
    shifts = [(0.0, 0.0)] * 25
    for iy in range(5):
        for ix in range(5):
            xn, yn = (ix - 2.0) / 2.5, (iy - 2.0) / 2.5
            dzx, dzy = SH.zernike_derivative(4, xn, yn)
            shifts[iy * 5] = (coeff_m * dzx / radius, coeff_m * dzy / radius)  # as the test writes it
    img = translated(5, 5, h, w, shifts)
    single = SH.shack_hartmann_slopes(img, skip_outside=True, **slope_args(h, w)).reshape(-1, 2)
    full = SH.full_pairwise_slopes(img, skip_outside=True, **slope_args(h, w)).reshape(-1, 2)
    for iy in range(5):
        for ix in range(5):
            i = iy * 5 + ix
            if active_5x5(iy, ix):
                assert abs(full[i, 0] - single[i, 0]) < 0.025 and abs(full[i, 1] - single[i, 1]) < 0.025
            else:
                assert full[i, 0] == 0.0 and full[i, 1] == 0.0


def test_causal_sliding_average():
    """CausalSlidingAverage (causal_sliding_average.cu:35-90): the first outputs average what has
    arrived (divisor min(k + 1, n)), then the last n; float32 running sum."""
    avg = SH.CausalSlidingAverage(3)
    got = [float(avg(np.array([v], np.float32))[0]) for v in (1.0, 2.0, 3.0, 4.0, 8.0)]
    assert got == [1.0, 1.5, 2.0, 3.0, 5.0]
