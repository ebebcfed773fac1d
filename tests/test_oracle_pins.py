"""Pins the CPU oracle to the reference's own known-answer tests for this path (restated from
test/holotask/angular_spectrum_test.cu, test/holotask/pca_test.cu,
test/holotask/fresnel_diffraction_test.cu and the holonp NumPy-oracle tests), plus the 12-bit
layout's exhaustive known answers.  CPU only."""
import math

import numpy as np
import pytest

from oracle import oracle as O

LAM, DX = 852e-9, 20e-6


# --------------------------------------------------------------------------------------------
# 12-bit packing: every value in both pixel phases, and hand-computed bytes
# --------------------------------------------------------------------------------------------
def test_pack12_all_values_both_phases():
    v = np.arange(4096, dtype=np.uint16)
    even = np.stack([v, np.zeros_like(v)], 1).reshape(-1)
    odd = np.stack([np.zeros_like(v), v], 1).reshape(-1)
    for seq in (even, odd, np.concatenate([v, v[::-1]])):
        assert np.array_equal(O.unpack12(O.pack12(seq)), seq)


def test_pack12_known_bytes():
    # p0 = 0xABC, p1 = 0x123 -> b0 = 0xBC, b1 = 0x3A (p0[11:8] = 0xA | p1[3:0] = 0x3 << 4), b2 = 0x12
    assert list(O.pack12(np.array([0xABC, 0x123]))) == [0xBC, 0x3A, 0x12]
    assert list(O.pack12(np.array([4095, 0]))) == [0xFF, 0x0F, 0x00]
    assert list(O.pack12(np.array([0, 4095]))) == [0x00, 0xF0, 0xFF]


def test_pack12_rejects_bad_input():
    with pytest.raises(ValueError):
        O.pack12(np.array([1, 2, 3]))
    with pytest.raises(ValueError):
        O.pack12(np.array([4096, 0]))


# --------------------------------------------------------------------------------------------
# AngularSpectrum known answers (angular_spectrum_test.cu:146-283)
# --------------------------------------------------------------------------------------------
def test_as_zero_distance_real_input_scales_by_hw():
    x = np.array([[1.0, 2.0], [3.0, 4.0]], np.float32)
    out = O.angular_spectrum(x, LAM, DX, DX, 0.0)
    np.testing.assert_allclose(out, np.array([[4, 8], [12, 16]], complex), atol=1e-3)


def test_as_centres_real_input_in_zero_padded_output():
    x = np.array([[1.0, 2.0], [3.0, 4.0]], np.float32)
    out = O.angular_spectrum(x, LAM, DX, DX, 0.0, padding={"width": 4, "height": 4})
    exp = np.zeros((4, 4), complex)
    exp[1:3, 1:3] = [[16, 32], [48, 64]]
    np.testing.assert_allclose(out, exp, atol=1e-3)


def test_as_centres_batched_complex_input():
    vals = np.arange(1, 9, dtype=np.float32)
    x = (vals + 1j * vals).astype(np.complex64).reshape(2, 2, 2)
    out = O.angular_spectrum(x, LAM, DX, DX, 0.0, padding={"width": 4, "height": 4})
    for b in range(2):
        for y in range(4):
            for xx in range(4):
                if 1 <= xx <= 2 and 1 <= y <= 2:
                    idx = b * 4 + (y - 1) * 2 + xx - 1
                    assert abs(out[b, y, xx] - (idx + 1) * 16 * (1 + 1j)) < 1e-3
                else:
                    assert abs(out[b, y, xx]) < 1e-3


def test_as_centres_batched_real_input():
    x = np.arange(1, 9, dtype=np.float32).reshape(2, 2, 2)
    out = O.angular_spectrum(x, LAM, DX, DX, 0.0, padding={"width": 4, "height": 4})
    for b in range(2):
        for y in range(1, 3):
            for xx in range(1, 3):
                idx = b * 4 + (y - 1) * 2 + xx - 1
                assert abs(out[b, y, xx] - (idx + 1) * 16) < 1e-3
    assert np.abs(out.imag).max() < 1e-3


def test_as_all_pass_filter_preserves_transfer_function():
    x = np.zeros((4, 4), np.complex64)
    x[1, 1] = 1.0
    a = O.angular_spectrum(x, LAM, DX, DX, 0.01)
    b = O.angular_spectrum(x, LAM, DX, DX, 0.01,
                           filt={"r_inner": 0, "r_outer": 100, "s_inner": 0, "s_outer": 0})
    np.testing.assert_allclose(a, b, atol=1e-3)


def test_as_rejects_bad_padding():
    x = np.zeros((4, 4), np.float32)
    with pytest.raises(ValueError):
        O.angular_spectrum(x, LAM, DX, DX, 0.0, padding={"width": 2, "height": 4})
    with pytest.raises(ValueError):
        O.angular_spectrum(np.zeros((2, 2)), LAM, DX, DX, 0.0, padding={"width": 3, "height": 4})


# --------------------------------------------------------------------------------------------
# PCA known answers (pca_test.cu:134-253)
# --------------------------------------------------------------------------------------------
def _two_by_two(scale=1.0):
    return np.array([scale * math.sqrt(2), 0.0, scale / math.sqrt(2), scale * math.sqrt(1.5)],
                    np.float32).reshape(2, 1, 2)


def test_pca_energies_are_ascending_eigenvalues():
    out = O.pca(_two_by_two(), 0, 2).reshape(2, 2)
    assert abs(out[0] @ out[0] - 1.0) < 2e-2
    assert abs(out[1] @ out[1] - 3.0) < 2e-2
    assert abs(out[0] @ out[1]) < 2e-2


def test_pca_nonzero_begin_over_33_batches():
    x = np.stack([_two_by_two(2.0 if b == 32 else 1.0) for b in range(33)])
    out = O.pca(x, 1, 2).reshape(33, 2)
    for b in range(32):
        assert abs(out[b] @ out[b] - 3.0) < 2e-2
    assert abs(out[32] @ out[32] - 12.0) < 5e-2


def test_pca_batches_scale():
    x = np.stack([_two_by_two(b + 1.0) for b in range(3)])
    out = O.pca(x, 0, 2).reshape(3, 2, 2)
    for b in range(3):
        s2 = (b + 1.0) ** 2
        assert abs(out[b, 0] @ out[b, 0] - s2) < 2e-2 * s2
        assert abs(out[b, 1] @ out[b, 1] - 3 * s2) < 2e-2 * s2


@pytest.mark.parametrize("depth", [256, 512])
def test_pca_large_depth_diagonal(depth):
    x = np.zeros((depth, depth), np.float32)
    x[np.arange(depth), np.arange(depth)] = np.sqrt(np.arange(1, depth + 1))
    out = O.pca(x.reshape(depth, 1, depth), depth - 1, depth).reshape(-1)
    assert abs(out @ out - depth) < 5e-2 * depth


def test_pca_recomputes_on_new_input():
    out = O.pca(np.array([3.0, 0.0, 0.0, 1.0], np.float32).reshape(2, 1, 2), 0, 2).reshape(2, 2)
    assert abs(out[0] @ out[0] - 1.0) < 2e-2
    assert abs(out[1] @ out[1] - 9.0) < 3e-2


# --------------------------------------------------------------------------------------------
# Fresnel (fresnel_diffraction_test.cu:112-161): magnitude == |complex|
# --------------------------------------------------------------------------------------------
def test_fresnel_magnitude_matches_complex_modulus():
    i = np.arange(2 * 3 * 32 * 48)
    x = ((i % 7) - 3.0 + 1j * ((i % 5) - 2.0)).reshape(2, 3, 32, 48)
    c = O.fresnel(x, LAM, DX, DX, 0.01, skip_phase_shift=False)
    m = O.fresnel(x, LAM, DX, DX, 0.01, output_magnitude=True)
    np.testing.assert_allclose(m, np.abs(c), rtol=1e-4, atol=1e-4)


def test_fresnel_lens_f32_matches_f64_formula():
    a = O.fresnel_lens(48, 32, LAM, 0.01, DX, "f32")
    b = O.fresnel_lens(48, 32, LAM, 0.01, DX, "f64")
    assert np.abs(np.angle(a / b)).max() < 1e-3


def test_fresnel_rejects_anisotropic_pitch():
    with pytest.raises(ValueError):
        O.fresnel(np.zeros((4, 4)), LAM, DX, 2 * DX, 0.01)


# --------------------------------------------------------------------------------------------
# holonp conventions (fft_test.cu / rfft_test.cu / mean_test.cu check against NumPy)
# --------------------------------------------------------------------------------------------
@pytest.mark.parametrize("norm", ["backward", "forward", "ortho"])
def test_fft_axis_norms_match_numpy(rng, norm):
    x = rng.standard_normal((2, 8, 3, 5))
    np.testing.assert_allclose(O.fft_axis(x, 1, norm), np.fft.fft(x, axis=1, norm=norm), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(O.rfft_axis(x, 1, norm), np.fft.rfft(x, axis=1, norm=norm), rtol=1e-12, atol=1e-12)


def test_band_dft_is_rfft_slice(rng):
    x = rng.integers(0, 4096, (32, 6, 5)).astype(np.float64)
    np.testing.assert_allclose(O.band_dft(x, 6, 16), np.fft.rfft(x, axis=0)[6:16], rtol=1e-12, atol=1e-9)


def test_mean_and_mean_abs(rng):
    x = rng.standard_normal((1, 5, 4, 3)) + 1j * rng.standard_normal((1, 5, 4, 3))
    np.testing.assert_allclose(O.mean(x, [-3]), x.mean(axis=-3, keepdims=True))
    np.testing.assert_allclose(O.mean_abs(x, [-3]), np.abs(x).mean(axis=-3, keepdims=True))


def test_freq_weights_follow_graph_builder():
    w = O.freq_weights(32, 6, 16, 37e3)
    df = 37e3 / 32
    np.testing.assert_array_equal(w, (6 * df + df * np.arange(10)).astype(np.float32))
    w2 = O.freq_weights(32, 6, 16, 37e3, method="fft")
    assert w2.shape == (20,) and np.isclose(w2[10], 6 * df - 37e3)
    assert O.arange_len(0, 0, 1) == 0


def test_band_bins_of_the_workloads():
    assert O.band_bins(4e3, 33e3, 67e3, 64) == (4, 32)
    assert O.band_bins(6e3, 18e3, 37e3, 32) == (6, 16)


def test_conversion_scaled_rounding():
    x = np.array([0.0, 0.5, 1.0, 0.25], np.float32)
    assert list(O.convert(x, "F32", "U8", "Scaled")) == [0, 128, 255, 64]
    with pytest.raises(ValueError):
        O.convert(x, "U16", "F32", "Real")  # no U16 -> F32 Real entry (conversion.cu:138-150)
