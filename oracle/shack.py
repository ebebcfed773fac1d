"""CPU oracle for the Shack-Hartmann autofocus stage (TEST INFRASTRUCTURE ONLY).

This module is the checker for the autofocus kernels.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline legs of ``bench.py`` may import it; the product never calls into it.

It restates in NumPy the reference's autofocus chain (graph_builder.cc:307-501):

- ShortTimeFresnelDiffraction (holotask/src/syncs/short_time_fresnel_diffraction.cu): windows of
  the field times a quadratic input phase (global or local frame), unnormalised 2D forward FFT,
  magnitude or complex output.
- Mean over the band axis, fftshift of every sub-aperture (graph_builder.cc:345-347).
- ShackHartmannSlopes in single-reference mode (shack_hartmann_slopes.cu,
  cross_correlation2.cu, phase_correlation.cuh): ROI mean removal and cosine taper, phase
  correlation against the centre sub-aperture, first-maximum peak with parabolic sub-pixel
  refinement, zero-mean slopes over the active sub-apertures.
- The sub-aperture geometry (shack_hartmann_geometry.cc), ZernikeFromSlopes
  (zernike_from_slopes.cc), ZernikePhase (zernike_phase.cu), CorrectPhase (correct_phase.cu),
  Wrap2Pi (wrap2pi.cu) and the defocus-to-distance estimate (zernike_defocus_z_prop.cc).

Floating point: float64 unless a float32 expression is part of the reference's observable result
(the input lens phase argument, the geometry).  Parity pins: the reference's known-answer tests in
test/holotask/shack_hartmann_test.cu (integer and sub-pixel translations, injected Zernike modes)
are restated in tests/test_shack_oracle.py and hold for this module.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

F32 = np.float32
PI_F32 = F32(math.pi)

SQRT3, SQRT6, SQRT8 = math.sqrt(3.0), math.sqrt(6.0), math.sqrt(8.0)


# ------------------------------------------------------------------------------------------------
# Short-time Fresnel diffraction
# ------------------------------------------------------------------------------------------------

def stfd_input_lens_phase(field_h: int, field_w: int, win_h: int, win_w: int, lam: float, z: float,
                          dx: float, dy: float, phase_ref: str = "global") -> np.ndarray:
    """float32 phase of stft_input_phase_kernel (short_time_fresnel_diffraction.cu:320-333) with the
    origins of input_lens_geometry (:342-369): the largest dimension of the frame (the whole field
    for "global", one window for "local") sets the centre."""
    if phase_ref == "global":
        w, h = field_w, field_h
    else:
        w, h = win_w, win_h
    size = max(w, h)
    off_x, off_y = (size - w) // 2, (size - h) // 2
    x_origin = F32((off_x - size / 2.0)) * F32(dx)
    y_origin = F32((off_y - size / 2.0)) * F32(dy)
    pi_over_lz = PI_F32 / (F32(lam) * F32(z))
    x = np.arange(w, dtype=F32) * F32(dx) + x_origin
    y = np.arange(h, dtype=F32) * F32(dy) + y_origin
    return (pi_over_lz * ((x * x)[None, :] + (y * y)[:, None])).astype(F32)


def stfd_input_lens(field_h, field_w, win_h, win_w, lam, z, dx, dy, phase_ref="global"):
    return np.exp(1j * stfd_input_lens_phase(field_h, field_w, win_h, win_w, lam, z, dx, dy,
                                             phase_ref).astype(np.float64))


def stfd_window_lens(win_h: int, win_w: int, lam: float, z: float, dx: float) -> np.ndarray:
    """stft_win_lens_kernel (short_time_fresnel_diffraction.cu:405-420): output-plane quadratic
    phase of one window, pixel pitch dx on both axes, the phase argument in float32."""
    size = max(win_w, win_h)
    x = (np.arange(win_w) + (size - win_w) // 2 - size / 2.0).astype(F32) * F32(dx)
    y = (np.arange(win_h) + (size - win_h) // 2 - size / 2.0).astype(F32) * F32(dx)
    k = PI_F32 / (F32(lam) * F32(z))
    ph = (k * ((x * x)[None, :] + (y * y)[:, None])).astype(F32)
    return np.exp(1j * ph.astype(np.float64))


def stfd_grid(H: int, W: int, win_h: int, win_w: int, stride_y: int, stride_x: int):
    """Window counts of ShortTimeFresnelDiffractionFactory::infer (:621-622)."""
    return (H - win_h) // stride_y + 1, (W - win_w) // stride_x + 1


def stfd(field: np.ndarray, win_h: int, win_w: int, stride_y: int, stride_x: int, lam: float,
         dx: float, dy: float, z: float, phase_ref: str = "global", output_magnitude: bool = True,
         skip_phase_shift: bool = True) -> np.ndarray:
    """ShortTimeFresnelDiffraction::execute (:564-598).  field [..., H, W] (real or complex) ->
    [..., ny, nx, win_h, win_w]: each window times the input lens (global: the lens at the
    window's pixels; local: the window's own lens), unnormalised 2D FFT, then |.| or the complex
    spectrum (times the window lens when skip_phase_shift is false)."""
    field = np.asarray(field)
    H, W = field.shape[-2:]
    ny, nx = stfd_grid(H, W, win_h, win_w, stride_y, stride_x)
    lens = stfd_input_lens(H, W, win_h, win_w, lam, z, dx, dy, phase_ref)
    out = np.empty(field.shape[:-2] + (ny, nx, win_h, win_w), dtype=np.complex128)
    for gy in range(ny):
        for gx in range(nx):
            y0, x0 = gy * stride_y, gx * stride_x
            win = field[..., y0:y0 + win_h, x0:x0 + win_w].astype(np.complex128)
            lw = lens[y0:y0 + win_h, x0:x0 + win_w] if phase_ref == "global" else lens
            out[..., gy, gx, :, :] = np.fft.fft2(win * lw, axes=(-2, -1))
    if output_magnitude:
        return np.abs(out)
    if not skip_phase_shift:
        out = out * stfd_window_lens(win_h, win_w, lam, z, dx)
    return out


def subaperture_m0(planes: np.ndarray, nb: int, lam: float, dx: float, z: float,
                   shift: bool = True) -> np.ndarray:
    """graph_builder.cc:329-347 for one spectrum: sub-apertures of W/nb x H/nb pixels with
    stride = size, global input phase, |.|, mean over the band axis, fftshift of each
    sub-aperture.  planes [Nz, H, W] complex -> [nb, nb, sh, sw]."""
    Nz, H, W = planes.shape
    sh, sw = H // nb, W // nb
    mag = stfd(planes, sh, sw, sh, sw, lam, dx, dx, z, "global", True)
    m0 = mag.mean(axis=0)
    if shift:
        m0 = np.fft.fftshift(m0, axes=(-2, -1))
    return m0


# ------------------------------------------------------------------------------------------------
# Phase correlation and slopes
# ------------------------------------------------------------------------------------------------

def ellipse_sq_distance(h: int, w: int, cx: float, cy: float, rx: float, ry: float,
                        angle: float = 0.0) -> np.ndarray:
    """phase_correlation.cuh:27-44 in float64: normalised pixel centres, rotated frame."""
    xn = (np.arange(w) + 0.5) / w
    yn = (np.arange(h) + 0.5) / h
    dx = xn[None, :] - cx
    dy = yn[:, None] - cy
    th = angle * math.pi / 180.0
    c, s = math.cos(th), math.sin(th)
    xr = c * dx + s * dy
    yr = -s * dx + c * dy
    return xr * xr / (rx * rx) + yr * yr / (ry * ry)


def phase_correlation_prep(img: np.ndarray, roi) -> np.ndarray:
    """compute_means_kernel + subtract_and_pack_kernel (cross_correlation2.cu:352-429): mean over
    the ROI, then (v - mean) * 0.5 (1 + cos(pi sqrt(d))) inside it and 0 outside."""
    h, w = img.shape[-2:]
    d = ellipse_sq_distance(h, w, *roi)
    inside = d <= 1.0
    mean = img[..., inside].mean(axis=-1) if inside.any() else np.zeros(img.shape[:-2])
    taper = 0.5 * (1.0 + np.cos(math.pi * np.sqrt(np.where(inside, d, 0.0))))
    return np.where(inside, (img - np.asarray(mean)[..., None, None]) * taper, 0.0)


def phase_correlation_maps(images: np.ndarray, reference: np.ndarray, roi) -> np.ndarray:
    """CrossCorrelation2::execute (cross_correlation2.cu:526-605) with backward norm: forward FFT
    of both prepared images, cross power normalised to unit magnitude (zero below 1e-12), inverse
    FFT, real part / (h w)."""
    a = np.fft.fft2(phase_correlation_prep(images, roi), axes=(-2, -1))
    b = np.fft.fft2(phase_correlation_prep(reference, roi), axes=(-2, -1))
    p = a * np.conj(b)
    mag = np.abs(p)
    p = np.where(mag <= 1e-12, 0.0, p / np.where(mag <= 1e-12, 1.0, mag))
    return np.real(np.fft.ifft2(p, axes=(-2, -1)))


def parabolic(vm: float, v0: float, vp: float) -> float:
    """parabolic_peak_offset (phase_correlation.cuh:58-62)."""
    den = vm - 2.0 * v0 + vp
    return 0.0 if abs(den) <= 1e-9 else 0.5 * (vm - vp) / den


def peak_shift(m: np.ndarray) -> tuple:
    """recover_phase_correlation_peaks (shack_hartmann_slopes.cu:124-158): first maximum in
    row-major order, parabolic refinement on the circular neighbours, signed circular
    coordinates.  Returns (dx, dy)."""
    h, w = m.shape
    flat = int(np.argmax(m))  # numpy returns the first occurrence of the maximum
    py, px = divmod(flat, w)
    dxs = parabolic(m[py, (px + w - 1) % w], m[py, px], m[py, (px + 1) % w])
    dys = parabolic(m[(py + h - 1) % h, px], m[py, px], m[(py + 1) % h, px])

    def signed(p, n):
        return float(p) if p < (n + 1) // 2 else float(p) - float(n)
    return signed(px, w) + dxs, signed(py, h) + dys


@dataclass
class Geometry:
    pupil_radius: float
    x_n: np.ndarray  # [sy*sx] float32
    y_n: np.ndarray
    active: np.ndarray  # [sy*sx] bool


def geometry(sy: int, sx: int, sub_h: int, sub_w: int, stride_y: int, stride_x: int, dy: float,
             dx: float, skip_outside: bool = True) -> Geometry:
    """make_shack_hartmann_geometry (shack_hartmann_geometry.cc:20-57) in float32."""
    pitch_x, pitch_y = F32(stride_x) * F32(dx), F32(stride_y) * F32(dy)
    aw = F32((sx - 1) * stride_x + sub_w) * F32(dx)
    ah = F32((sy - 1) * stride_y + sub_h) * F32(dy)
    r = F32(0.5) * min(aw, ah)
    cx, cy = (F32(sx) - F32(1)) * F32(0.5), (F32(sy) - F32(1)) * F32(0.5)
    xs, ys, act = [], [], []
    for iy in range(sy):
        for ix in range(sx):
            xm = (F32(ix) - cx) * pitch_x
            ym = (F32(iy) - cy) * pitch_y
            xn, yn = xm / r, ym / r
            xs.append(xn)
            ys.append(yn)
            act.append((not skip_outside) or bool(xn * xn + yn * yn <= F32(1)))
    return Geometry(float(r), np.array(xs, F32), np.array(ys, F32), np.array(act, bool))


def zero_mean_slopes(shifts: np.ndarray, active: np.ndarray, center: int, spp_x: float,
                     spp_y: float) -> np.ndarray:
    """recover_zero_mean_slopes (shack_hartmann_slopes.cu:160-192): shifts relative to the centre,
    scaled to slopes, mean over the active samples removed; inactive samples are 0."""
    s = (shifts - shifts[center]) * np.array([spp_x, spp_y])
    out = np.zeros_like(s)
    if active.any():
        out[active] = s[active] - s[active].mean(axis=0)
    return out


def shack_hartmann_slopes(images: np.ndarray, lam: float, dx: float, dy: float, z: float,
                          roi=(0.5, 0.5, 0.5, 0.5, 0.0), skip_outside: bool = True,
                          return_maps: bool = False):
    """ShackHartmannSlopes::execute, single-reference mode (shack_hartmann_slopes.cu:240-281).
    images [sy, sx, h, w] -> slopes [sy, sx, 2] (and the correlation maps)."""
    sy, sx, h, w = images.shape
    center = (sy // 2) * sx + sx // 2
    flat = images.reshape(sy * sx, h, w).astype(np.float64)
    maps = phase_correlation_maps(flat, flat[center], roi)
    shifts = np.array([peak_shift(m) for m in maps])
    geo = geometry(sy, sx, h, w, h, w, dy, dx, skip_outside)
    spp_x = (lam * z / (w * dx)) / z
    spp_y = (lam * z / (h * dy)) / z
    slopes = zero_mean_slopes(shifts, geo.active, center, spp_x, spp_y).reshape(sy, sx, 2)
    return (slopes, maps.reshape(sy, sx, h, w)) if return_maps else slopes


def full_pairwise_slopes(images: np.ndarray, lam: float, dx: float, dy: float, z: float,
                         roi=(0.5, 0.5, 0.5, 0.5, 0.0), skip_outside: bool = True) -> np.ndarray:
    """ShackHartmannSlopes, FullPairwise mode (the graph-Laplacian recovery,
    shack_hartmann_slopes_full_pairwise.cuh:69-241).  Every pair (i, j), i < j, of ACTIVE
    sub-apertures is phase-correlated (moving i against reference j: normalised i conj(j),
    phase_correlation.cuh:54-62); the peak shift of the pair, scaled to slopes, is added to rhs[i]
    and subtracted from rhs[j] (accumulate_complete_graph_rhs); the complete-graph Laplacian solve
    in the zero-mean gauge is slope_i = rhs_i / N - mean_k(rhs_k / N) (solve_complete_graph_and_
    scatter); inactive samples are 0.  images [sy, sx, h, w] -> slopes [sy, sx, 2]."""
    sy, sx, h, w = images.shape
    flat = images.reshape(sy * sx, h, w).astype(np.float64)
    geo = geometry(sy, sx, h, w, h, w, dy, dx, skip_outside)
    act = np.flatnonzero(geo.active)
    n = len(act)
    spec = np.fft.fft2(phase_correlation_prep(flat[act], roi), axes=(-2, -1))
    spp_x = (lam * z / (w * dx)) / z
    spp_y = (lam * z / (h * dy)) / z
    rhs = np.zeros((n, 2))
    for i in range(n):
        for j in range(i + 1, n):
            p = spec[i] * np.conj(spec[j])
            mag = np.abs(p)
            p = np.where(mag <= 1e-12, 0.0, p / np.where(mag <= 1e-12, 1.0, mag))
            # the unnormalised inverse times 1 / (h w): numpy's normalised inverse
            ddx, ddy = peak_shift(np.real(np.fft.ifft2(p)))
            rhs[i] += (ddx * spp_x, ddy * spp_y)
            rhs[j] -= (ddx * spp_x, ddy * spp_y)
    out = np.zeros((sy * sx, 2))
    if n:
        mean = (rhs / n).sum(axis=0) / n
        out[act] = rhs / n - mean
    return out.reshape(sy, sx, 2)


# ------------------------------------------------------------------------------------------------
# Zernike modes
# ------------------------------------------------------------------------------------------------

def zernike_value(noll: int, x, y):
    """eval_zernike_noll_value (zernike_phase.cu:88-113), Noll 2..10."""
    if noll == 2:
        return 2.0 * x
    if noll == 3:
        return 2.0 * y
    if noll == 4:
        return SQRT3 * (2.0 * (x * x + y * y) - 1.0)
    if noll == 5:
        return 2.0 * SQRT6 * x * y
    if noll == 6:
        return SQRT6 * (x * x - y * y)
    if noll == 7:
        return SQRT8 * y * (3.0 * x * x - y * y)
    if noll == 8:
        return SQRT8 * y * (3.0 * x * x + 3.0 * y * y - 2.0)
    if noll == 9:
        return SQRT8 * x * (3.0 * x * x + 3.0 * y * y - 2.0)
    if noll == 10:
        return SQRT8 * x * (x * x - 3.0 * y * y)
    raise ValueError("Noll index out of 2..10")


def zernike_derivative(noll: int, x, y):
    """eval_zernike_noll_derivative (zernike_from_slopes.cc:95-123): (dZ/dx, dZ/dy)."""
    if noll == 2:
        return 2.0 + 0 * x, 0 * x
    if noll == 3:
        return 0 * x, 2.0 + 0 * x
    if noll == 4:
        return 4.0 * SQRT3 * x, 4.0 * SQRT3 * y
    if noll == 5:
        return 2.0 * SQRT6 * y, 2.0 * SQRT6 * x
    if noll == 6:
        return 2.0 * SQRT6 * x, -2.0 * SQRT6 * y
    if noll == 7:
        return 6.0 * SQRT8 * x * y, 3.0 * SQRT8 * (x * x - y * y)
    if noll == 8:
        return 6.0 * SQRT8 * x * y, SQRT8 * (3.0 * x * x + 9.0 * y * y - 2.0)
    if noll == 9:
        return SQRT8 * (9.0 * x * x + 3.0 * y * y - 2.0), 6.0 * SQRT8 * x * y
    if noll == 10:
        return 3.0 * SQRT8 * (x * x - y * y), -6.0 * SQRT8 * x * y
    raise ValueError("Noll index out of 2..10")


def zernike_from_slopes(slopes: np.ndarray, indexes: Sequence[int], lam: float, geo: Geometry
                        ) -> np.ndarray:
    """ZernikeFromSlopes::execute (zernike_from_slopes.cc:205-277) in float64: tip and tilt
    (Noll 2, 3) are not observable from zero-mean slopes and stay 0; the other modes are the
    least-squares fit of the mean-removed derivatives (divided by the pupil radius) to the slopes,
    with a 1e-9 ridge, converted to radians (2 pi / lambda)."""
    s = np.asarray(slopes, np.float64).reshape(-1, 2)
    obs = [i for i, n in enumerate(indexes) if n not in (2, 3)]
    act = geo.active
    xn, yn = geo.x_n.astype(np.float64)[act], geo.y_n.astype(np.float64)[act]
    gx = np.stack([zernike_derivative(indexes[i], xn, yn)[0] for i in obs], 1) / geo.pupil_radius
    gy = np.stack([zernike_derivative(indexes[i], xn, yn)[1] for i in obs], 1) / geo.pupil_radius
    gx -= gx.mean(0)
    gy -= gy.mean(0)
    gtg = gx.T @ gx + gy.T @ gy + 1e-9 * np.eye(len(obs))
    gts = gx.T @ s[act, 0] + gy.T @ s[act, 1]
    c = np.linalg.solve(gtg, gts) if obs else np.zeros(0)
    out = np.zeros(len(indexes))
    out[obs] = c * 2.0 * math.pi / lam
    return out


def zernike_phase(coeffs: Sequence[float], indexes: Sequence[int], ny: int, nx: int) -> np.ndarray:
    """zernike_phase_kernel (zernike_phase.cu:151-180): pupil centred on the grid, radius half the
    smaller side, every pixel evaluated (no pupil mask)."""
    cy, cx = (ny - 1) * 0.5, (nx - 1) * 0.5
    r = 0.5 * min(ny, nx)
    x = ((np.arange(nx) - cx) / r)[None, :]
    y = ((np.arange(ny) - cy) / r)[:, None]
    ph = np.zeros((ny, nx))
    for c, n in zip(coeffs, indexes):
        ph = ph + c * zernike_value(n, x, y)
    return ph


def correct_phase(field: np.ndarray, phase: np.ndarray) -> np.ndarray:
    """correct_phase_cf32_kernel (correct_phase.cu:93-106): E exp(-i phi), phase broadcast over
    the leading axes."""
    return field * np.exp(-1j * phase)


def wrap2pi(x: np.ndarray) -> np.ndarray:
    """wrap2pi_kernel (wrap2pi.cu:60-70) in float32: fmod by 2 pi, negatives shifted up."""
    two_pi = F32(2.0) * PI_F32
    v = np.fmod(np.asarray(x, F32), two_pi)
    return np.where(v < 0, v + two_pi, v).astype(F32)


def defocus_z(a4: float, lam: float, z_curr: float, pupil_radius: float) -> tuple:
    """estimate_z_prop_from_a4 (zernike_defocus_z_prop.cc:84-97): (delta 1/z, new z, delta z in
    mm) from the defocus coefficient in radians."""
    d_inv = (2.0 * math.sqrt(3.0) * lam * a4) / (math.pi * pupil_radius * pupil_radius)
    z_new = 1.0 / (1.0 / z_curr - d_inv)
    return d_inv, z_new, 1000.0 * (z_new - z_curr)


# ------------------------------------------------------------------------------------------------
# One autofocus pass
# ------------------------------------------------------------------------------------------------

@dataclass
class AutofocusConfig:
    nb_subaps: int
    lam: float
    dx: float
    z: float
    indexes: Sequence[int] = (4,)
    roi_radius: float = 0.5
    skip_outside: bool = True
    flatfield_period: float = 0.0  # pp_flatfield cutoff period [m]; 0 = off
    full_pairwise: bool = False    # autofocus_use_graph_laplacian (graph_builder.cc:359-361)


def subaperture_flatfield(m0: np.ndarray, cfg: AutofocusConfig) -> np.ndarray:
    """graph_builder.cc:348-352: the flatfield of every sub-aperture image with sigma =
    0.187 period / pitch, the pitch being the one-FFT Fresnel output pitch lambda |z| / (n d)
    of a sub-aperture (graph_builder.cc:32-66), all in float32."""
    from . import oracle as O
    nb, _, sh, sw = m0.shape
    dy_out = F32(cfg.lam) * abs(F32(cfg.z)) / (F32(sh) * F32(cfg.dx))
    dx_out = F32(cfg.lam) * abs(F32(cfg.z)) / (F32(sw) * F32(cfg.dx))
    sy = float(F32(0.187) * F32(cfg.flatfield_period) / dy_out)
    sx = float(F32(0.187) * F32(cfg.flatfield_period) / dx_out)
    flat = m0.reshape(nb * nb, sh, sw)
    out = O.flatfield_fourier(flat, sy, sx) if O.flatfield_uses_fourier(sh, sw, sy, sx) else \
        O.flatfield_spatial(flat, sy, sx)
    return np.asarray(out, np.float64).reshape(m0.shape)


class CausalSlidingAverage:
    """CausalSlidingAverage (causal_sliding_average.cu:35-90): a float32 history of the last n
    inputs (starting at zero) and a float32 running sum, sum += x - x_(k-n); the output is the sum
    divided by min(k + 1, n), so the first outputs average the inputs seen so far."""

    def __init__(self, n: int):
        self.n, self.count, self.hist, self.sum = n, 0, None, None

    def __call__(self, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, np.float32)
        if self.hist is None:
            self.hist = np.zeros((self.n,) + x.shape, np.float32)
            self.sum = np.zeros(x.shape, np.float32)
        slot = self.count % self.n
        self.sum = ((self.sum + x).astype(np.float32) - self.hist[slot]).astype(np.float32)
        self.hist[slot] = x
        out = self.sum / np.float32(min(self.count + 1, self.n))
        self.count += 1
        return out.astype(np.float64)


def autofocus(planes: np.ndarray, cfg: AutofocusConfig, delayed: Optional[np.ndarray] = None,
              average: Optional[CausalSlidingAverage] = None):
    """build_shack_hartmann (graph_builder.cc:307-501) for one spectrum: sub-aperture M0 (causally
    averaged over the last pp_accumulation spectra when `average` is given, graph_builder.cc:348),
    optional flatfield, slopes (single-reference, or full-pairwise when cfg.full_pairwise), Zernike
    fit, phase over the full field, and the corrected planes -- `delayed` when given (the dual
    reader's delayed window, graph_builder.cc:128-143).  Returns (m0, slopes, coefficients, phase,
    corrected)."""
    Nz, H, W = planes.shape
    nb = cfg.nb_subaps
    sh, sw = H // nb, W // nb
    m0 = subaperture_m0(planes, nb, cfg.lam, cfg.dx, cfg.z)
    if average is not None:
        m0 = average(m0)
    if cfg.flatfield_period > 0.0:
        m0 = subaperture_flatfield(m0, cfg)
    roi = (0.5, 0.5, cfg.roi_radius, cfg.roi_radius, 0.0)
    if cfg.full_pairwise:
        slopes = full_pairwise_slopes(m0, cfg.lam, cfg.dx, cfg.dx, cfg.z, roi, cfg.skip_outside)
    else:
        slopes = shack_hartmann_slopes(m0, cfg.lam, cfg.dx, cfg.dx, cfg.z, roi, cfg.skip_outside)
    geo = geometry(nb, nb, sh, sw, sh, sw, cfg.dx, cfg.dx, cfg.skip_outside)
    coeffs = zernike_from_slopes(slopes, cfg.indexes, cfg.lam, geo)
    phase = zernike_phase(coeffs, cfg.indexes, H, W)
    src = planes if delayed is None else delayed
    return m0, slopes, coeffs, phase, correct_phase(src, phase)
