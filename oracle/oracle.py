"""CPU oracle for the laser Doppler reconstruction path (TEST INFRASTRUCTURE ONLY).

This module is the checker.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` may import it; the product (the CUDA library
and its host layer) never calls into it.

It restates, in NumPy float64 (plus float32 where the reference computes in
float32 and the rounding is part of its observable behaviour), every stage of
Holoflow's per-window Doppler path.  Each function cites the reference source
it follows (paths relative to the Holoflow source tree).

Parity pins: the reference's own known-answer tests for this path
(test/holotask/angular_spectrum_test.cu, test/holotask/pca_test.cu,
test/holotask/fresnel_diffraction_test.cu, and the holonp NumPy-oracle tests
for fft/rfft/mean) are restated in tests/test_oracle_pins.py and must hold for
this module.  Fresnel absolute values, the 12-bit unpack, MeanAbs and the
end-to-end moments have no reference fixture: for those stages parity is
unpinned and the oracle's own definition (documented per function) is the
contract.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

try:  # multithreaded FFTs when scipy is present (it is in the image)
    import scipy.fft as _sfft

    def _fft2(x, axes=(-2, -1), inverse=False, workers=-1):
        f = _sfft.ifft2 if inverse else _sfft.fft2
        y = f(x, axes=axes, workers=workers)
        if inverse:  # unnormalised inverse, as cuFFT's CUFFT_INVERSE
            y = y * (x.shape[axes[0]] * x.shape[axes[1]])
        return y

    def _fft(x, axis, workers=-1):
        return _sfft.fft(x, axis=axis, workers=workers)

except ImportError:  # pragma: no cover
    def _fft2(x, axes=(-2, -1), inverse=False, workers=None):
        if inverse:
            return np.fft.ifft2(x, axes=axes) * (x.shape[axes[0]] * x.shape[axes[1]])
        return np.fft.fft2(x, axes=axes)

    def _fft(x, axis, workers=None):
        return np.fft.fft(x, axis=axis)


F32 = np.float32
PI_F32 = F32(math.pi)  # CUDART_PI_F rounded to float32


# -------------------------------------------------------------------------------------------------
# a1: 12-bit packed frames ("Mono12p", little-endian, 2 pixels in 3 bytes)
# -------------------------------------------------------------------------------------------------
# The reference has no 12-bit path (sources/holofile.cc:247-250 accepts 8/16 bpp only), so the
# layout is defined here and pinned by tests/test_oracle_pins.py over all 4096 values x both
# pixel phases:  byte0 = p0[7:0];  byte1 = p0[11:8] | p1[3:0] << 4;  byte2 = p1[11:4].

def pack12(values: np.ndarray) -> np.ndarray:
    """Pack uint16 values (< 4096, even count) into the Mono12p byte stream."""
    v = np.asarray(values, dtype=np.uint16).reshape(-1)
    if v.size % 2:
        raise ValueError("pack12 needs an even number of pixels")
    if v.size and int(v.max()) > 4095:
        raise ValueError("pack12 values must be < 4096")
    p0 = v[0::2].astype(np.uint32)
    p1 = v[1::2].astype(np.uint32)
    out = np.empty((v.size // 2, 3), dtype=np.uint8)
    out[:, 0] = p0 & 0xFF
    out[:, 1] = ((p0 >> 8) & 0xF) | ((p1 & 0xF) << 4)
    out[:, 2] = (p1 >> 4) & 0xFF
    return out.reshape(-1)


def unpack12(packed: np.ndarray, npix: Optional[int] = None) -> np.ndarray:
    """Inverse of :func:`pack12`; returns uint16."""
    b = np.asarray(packed, dtype=np.uint8).reshape(-1)
    if b.size % 3:
        raise ValueError("packed stream length must be a multiple of 3")
    t = b.reshape(-1, 3).astype(np.uint16)
    out = np.empty(t.shape[0] * 2, dtype=np.uint16)
    out[0::2] = t[:, 0] | ((t[:, 1] & 0xF) << 8)
    out[1::2] = (t[:, 1] >> 4) | (t[:, 2] << 4)
    return out if npix is None else out[:npix]


# -------------------------------------------------------------------------------------------------
# a2: Conversion (holotask/src/syncs/conversion.cu:138-150 table, 156-216 kernels)
# -------------------------------------------------------------------------------------------------
CONVERSIONS = {
    ("U8", "F32", "Real"): "F32",
    ("U8", "CF32", "Real"): "CF32",
    ("U16", "CF32", "Real"): "CF32",
    ("F32", "U8", "Scaled"): "U8",
    ("F32", "U16", "Scaled"): "U16",
    ("F32", "CF32", "Real"): "CF32",
    ("CF32", "F32", "Modulus"): "F32",
    ("CF32", "F32", "Argument"): "F32",
}


def convert(x: np.ndarray, src: str, target: str, strategy: str) -> np.ndarray:
    """Element-wise dtype conversion with the reference's exact rounding.

    Scaled conversions follow conversion.cu:177-197: scale = 255/(max-min) computed in float32,
    val = int((x - min) * scale + 0.5) (truncation toward zero), clamped to the target range.
    """
    key = (src, target, strategy)
    if key not in CONVERSIONS:
        raise ValueError(f"unsupported conversion {key}")
    if target == "F32" and strategy == "Real":
        return x.astype(F32)
    if target == "CF32" and strategy == "Real":
        return x.astype(F32).astype(np.complex64)
    if strategy == "Modulus":
        return np.hypot(x.real.astype(np.float64), x.imag.astype(np.float64)).astype(F32)
    if strategy == "Argument":
        return np.arctan2(x.imag.astype(np.float64), x.real.astype(np.float64)).astype(F32)
    # Scaled
    top = F32(255.0) if target == "U8" else F32(65535.0)
    xf = x.astype(F32)
    mn, mx = F32(xf.min()), F32(xf.max())
    scale = F32(top / F32(mx - mn))
    val = (F32(xf - mn) * scale + F32(0.5)).astype(F32)
    iv = np.trunc(val.astype(np.float64))
    iv = np.clip(iv, 0, float(top))
    return iv.astype(np.uint8 if target == "U8" else np.uint16)


# -------------------------------------------------------------------------------------------------
# a3/a4: BatchQueue window semantics (holotask/src/asyncs/batch_queue.cc:92-174, 209-210)
# -------------------------------------------------------------------------------------------------

def windows(frames: np.ndarray, size: int, stride: int) -> list[np.ndarray]:
    """Windows of ``size`` frames every ``stride`` frames (first window starts at frame 0).

    The reference only allows stride % size == 0 (batch_queue.cc:209-210); overlapping windows
    (stride < size) are this build's extension, defined as the same sliding-window rule.
    """
    n = frames.shape[0]
    out = []
    start = 0
    while start + size <= n:
        out.append(frames[start:start + size])
        start += stride
    return out


# -------------------------------------------------------------------------------------------------
# a5/a6/a7: temporal FFT / RFFT along an axis + band slice (holonp/src/fft.cu:100-109 norm,
# rfft.cu:142-170; graph_builder.cc:260-287 slice)
# -------------------------------------------------------------------------------------------------

def norm_scale(norm: str, n: int) -> float:
    if norm == "backward":
        return 1.0
    if norm == "forward":
        return 1.0 / n
    if norm == "ortho":
        return 1.0 / math.sqrt(n)
    raise ValueError(norm)


def fft_axis(x: np.ndarray, axis: int, norm: str = "backward") -> np.ndarray:
    return _fft(np.asarray(x, dtype=np.complex128), axis) * norm_scale(norm, x.shape[axis])


def rfft_axis(x: np.ndarray, axis: int, norm: str = "backward") -> np.ndarray:
    n = x.shape[axis]
    full = _fft(np.asarray(x, dtype=np.float64), axis)
    sl = [slice(None)] * full.ndim
    sl[axis] = slice(0, n // 2 + 1)
    return full[tuple(sl)] * norm_scale(norm, n)


def band_dft(frames: np.ndarray, z0: int, z1: int) -> np.ndarray:
    """Bins [z0, z1) of the unnormalised DFT along axis 0 (= RFFT then Slice along T)."""
    f = np.asarray(frames, dtype=np.float64)
    return _fft(f, 0)[z0:z1]


# -------------------------------------------------------------------------------------------------
# a8: PCA (holotask/src/syncs/pca.cc:68-119) and the SVD clutter filter built from it
# -------------------------------------------------------------------------------------------------

def covariance(x: np.ndarray) -> np.ndarray:
    """C = X^T X over pixels, no centring and no 1/N (pca.cc:92-98).  x: [T, H, W] or [T, P]."""
    X = np.asarray(x, dtype=np.float64).reshape(x.shape[0], -1)
    return X @ X.T


def eigh_ascending(c: np.ndarray):
    """Symmetric eigendecomposition, eigenvalues ascending (syev/heev order, pca_test.cu:134-145)."""
    w, v = np.linalg.eigh(np.asarray(c, dtype=np.float64))
    return w, v


def pca(x: np.ndarray, begin: int, end: int) -> np.ndarray:
    """Projection of every pixel's T-vector onto eigenvectors [begin, end) (pca.cc:106-116).

    x: [..., T, H, W] float; returns [..., end-begin, H, W].  Eigenvector signs are arbitrary in
    the reference, so comparisons must be sign-invariant (energies / projectors).
    """
    x = np.asarray(x, dtype=np.float64)
    lead = x.shape[:-3]
    T, H, W = x.shape[-3:]
    xb = x.reshape(-1, T, H * W)
    out = np.empty((xb.shape[0], end - begin, H * W))
    for b in range(xb.shape[0]):
        _, v = eigh_ascending(covariance(xb[b]))
        out[b] = (xb[b].T @ v[:, begin:end]).T
    return out.reshape(*lead, end - begin, H, W)


def clutter_basis(frames: np.ndarray, rank: int) -> np.ndarray:
    """The ``rank`` eigenvectors of X^T X with the largest eigenvalues, [T, rank]."""
    if rank <= 0:
        return np.zeros((frames.shape[0], 0))
    _, v = eigh_ascending(covariance(frames))
    return v[:, v.shape[1] - rank:]


def svd_filter(frames: np.ndarray, rank: int) -> np.ndarray:
    """Remove the top-``rank`` eigenvectors along time: Y = X (I - V V^T) per pixel.

    The full-size workload (1024^2 12-bit frames, T = 64) removes the top-4 eigenvectors of the
    64x64 complex covariance of the propagated frames.  Propagation A (unit-modulus lens + unnormalised DFT)
    satisfies A^H A = N I, so (A X)^H (A X) = N X^T X for real frames: the eigenvectors are those
    of the real covariance and the filter commutes with propagation (tested in
    tests/test_oracle_model.py).
    """
    X = np.asarray(frames, dtype=np.float64)
    T = X.shape[0]
    V = clutter_basis(X, rank)
    Xf = X.reshape(T, -1)
    return (Xf - V @ (V.T @ Xf)).reshape(X.shape)


def band_bin_list(T: int, z0: int, z1: int, method: str = "rfft") -> np.ndarray:
    """The DFT bins of the band planes: [z0, z1), and for the two-sided FFT method also the
    negative band [T - z1, T - z0) after it (graph_builder.cc:270-287: slice, slice, concatenate)."""
    pos = np.arange(z0, z1)
    return np.concatenate([pos, np.arange(T - z1, T - z0)]) if method == "fft" else pos


def band_matrix(T: int, z0: int, z1: int, V: Optional[np.ndarray] = None, method: str = "rfft") -> np.ndarray:
    """W = (I - V V^T) D[:, bins], the T x Nz complex matrix one window's filter+DFT reduces to."""
    t = np.arange(T)[:, None]
    k = band_bin_list(T, z0, z1, method)[None, :]
    D = np.exp(-2j * np.pi * (t * k % T) / T)
    if V is not None and V.shape[1]:
        D = D - V @ (V.T @ D)
    return D


# -------------------------------------------------------------------------------------------------
# a9: Fresnel diffraction (holotask/src/syncs/fresnel_diffraction.cu:326-341 lens, 359-380 output
# phase, 410-441 execute)
# -------------------------------------------------------------------------------------------------

def fresnel_lens_phase_f32(height: int, width: int, lam: float, z: float, dx: float) -> np.ndarray:
    """Lens phase exactly as quadratic_lens_kernel computes it in float32 (no FMA contraction).

    size = max(H, W); x = ((col + (size-W)/2) - size/2) * dx; likewise y with the same dx;
    phase = (pi / (lambda*z)) * (x*x + y*y).
    """
    size = max(width, height)
    off_x = (size - width) // 2
    off_y = (size - height) // 2
    half = F32(size / 2.0)
    px = F32(dx)
    col = np.arange(width)
    row = np.arange(height)
    x = ((col + off_x).astype(F32) - half) * px
    y = ((row + off_y).astype(F32) - half) * px
    k = PI_F32 / (F32(lam) * F32(z))
    r2 = (x * x)[None, :] + (y * y)[:, None]
    return (k * r2).astype(F32)


def fresnel_lens(height: int, width: int, lam: float, z: float, dx: float,
                 phase_mode: str = "f32") -> np.ndarray:
    """Complex lens L = exp(i*phase) as complex128.  ``phase_mode="f32"`` follows the reference's
    float32 phase argument; ``"f64"`` evaluates the same formula in float64 (error reference)."""
    if phase_mode == "f32":
        ph = fresnel_lens_phase_f32(height, width, lam, z, dx).astype(np.float64)
    else:
        size = max(width, height)
        x = ((np.arange(width) + (size - width) // 2) - size / 2.0) * dx
        y = ((np.arange(height) + (size - height) // 2) - size / 2.0) * dx
        ph = math.pi / (lam * z) * (x[None, :] ** 2 + y[:, None] ** 2)
    return np.exp(1j * ph)


def fresnel(u: np.ndarray, lam: float, dx: float, dy: float, z: float,
            output_magnitude: bool = False, skip_phase_shift: bool = True,
            phase_mode: str = "f32") -> np.ndarray:
    """FFT2_forward(u * L) over the last two axes, unnormalised, no fftshift.

    output_magnitude -> |.| (store callback, fresnel_diffraction.cu:305-311); otherwise complex,
    multiplied once more by the same lens array when skip_phase_shift is False
    (apply_output_phase_shift_kernel, fresnel_diffraction.cu:359-380).
    """
    if dx != dy:
        raise ValueError("dx must equal dy")
    H, W = u.shape[-2:]
    L = fresnel_lens(H, W, lam, z, dx, phase_mode)
    out = _fft2(np.asarray(u, dtype=np.complex128) * L)
    if output_magnitude:
        return np.abs(out)
    if not skip_phase_shift:
        out = out * L
    return out


# -------------------------------------------------------------------------------------------------
# a10: Angular spectrum (holotask/src/syncs/angular_spectrum.cu:189-229 padding, 261-278 TF,
# 280-330 filter, 332-363 corner swap, 408-431 execute)
# -------------------------------------------------------------------------------------------------

def as_tf_phase_f32(height: int, width: int, lam: float, z: float, dx: float) -> np.ndarray:
    """spectral_lens_kernel's float32 phase: u = (col - W/2) * (1/(W*dx)) with integer W/2,
    tmp = max(0, 1 - (lam*lam)*(u*u + v*v)), phase = ((2*pi*z)/lam) * sqrt(tmp)."""
    lamf, zf, px = F32(lam), F32(z), F32(dx)
    du = F32(1.0) / F32(F32(width) * px)
    dv = F32(1.0) / F32(F32(height) * px)
    u = (np.arange(width) - width // 2).astype(F32) * du
    v = (np.arange(height) - height // 2).astype(F32) * dv
    s = (u * u)[None, :] + (v * v)[:, None]
    tmp = F32(1.0) - F32(lamf * lamf) * s
    tmp = np.maximum(tmp, F32(0.0))
    k = F32(F32(F32(2.0) * PI_F32) * zf) / lamf
    return (k * np.sqrt(tmp)).astype(F32)


def as_filter_weight(height: int, width: int, r_inner: int, r_outer: int,
                     s_inner: int, s_outer: int) -> np.ndarray:
    """Raised-sine annulus of multiply_filter_2d_kernel (value squared), float32 arithmetic."""
    x = np.arange(width, dtype=F32) - F32(width / 2.0)
    y = np.arange(height, dtype=F32) - F32(height / 2.0)
    dist = np.hypot(x[None, :].astype(np.float64), y[:, None].astype(np.float64)).astype(F32)
    ri, ro, si, so = F32(r_inner), F32(r_outer), F32(s_inner), F32(s_outer)
    inner_start, inner_end = ri - si, ri + si
    outer_start, outer_end = ro - so, ro + so
    val = np.zeros_like(dist)
    with np.errstate(divide="ignore", invalid="ignore"):
        fade_in = F32(0.5) * (F32(1.0) + np.sin((PI_F32 / (F32(2.0) * si) * (dist - inner_start))
                                               .astype(np.float64)).astype(F32))
        fade_out = F32(0.5) * (F32(1.0) + np.sin((PI_F32 / (F32(2.0) * so) * (outer_end - dist))
                                                .astype(np.float64)).astype(F32))
    in_hole = dist < inner_start
    in_tr_in = (dist >= inner_start) & (dist < inner_end)
    plateau = (dist >= inner_end) & (dist < outer_start)
    in_tr_out = (dist >= outer_start) & (dist < outer_end)
    val = np.where(in_tr_in, fade_in, val)
    val = np.where(plateau, F32(1.0), val)
    val = np.where(in_tr_out, fade_out, val)
    val = np.where(in_hole, F32(0.0), val)
    return (val * val).astype(F32)


def swap_corners(a: np.ndarray) -> np.ndarray:
    """swap_corners_kernel: exchange the (H/2 x W/2) quadrants (integer halves); for odd sizes
    the last row/column stays in place (not numpy's ifftshift)."""
    H, W = a.shape[-2:]
    h2, w2 = H // 2, W // 2
    out = a.copy()
    out[..., :h2, :w2] = a[..., h2:2 * h2, w2:2 * w2]
    out[..., h2:2 * h2, w2:2 * w2] = a[..., :h2, :w2]
    out[..., :h2, w2:2 * w2] = a[..., h2:2 * h2, :w2]
    out[..., h2:2 * h2, :w2] = a[..., :h2, w2:2 * w2]
    return out


def as_transfer_function(height: int, width: int, lam: float, z: float, dx: float,
                         filt: Optional[dict] = None, phase_mode: str = "f32") -> np.ndarray:
    if phase_mode == "f32":
        ph = as_tf_phase_f32(height, width, lam, z, dx).astype(np.float64)
        tf = np.exp(1j * ph)
        tf = (tf.real.astype(F32) + 1j * tf.imag.astype(F32)).astype(np.complex128)
    else:
        u = (np.arange(width) - width // 2) / (width * dx)
        v = (np.arange(height) - height // 2) / (height * dx)
        tmp = np.maximum(0.0, 1 - lam ** 2 * (u[None, :] ** 2 + v[:, None] ** 2))
        tf = np.exp(1j * 2 * math.pi * z / lam * np.sqrt(tmp))
    if filt is not None:
        w = as_filter_weight(height, width, filt["r_inner"], filt["r_outer"],
                             filt["s_inner"], filt["s_outer"]).astype(np.float64)
        tf = tf * w
    return swap_corners(tf)


def angular_spectrum(u: np.ndarray, lam: float, dx: float, dy: float, z: float,
                     filt: Optional[dict] = None, padding: Optional[dict] = None,
                     phase_mode: str = "f32") -> np.ndarray:
    """IFFT2(FFT2(pad_center(u)) * TF), both unnormalised (so x H*W overall)."""
    if dx != dy:
        raise ValueError("dx must equal dy")
    u = np.asarray(u)
    H, W = u.shape[-2:]
    OH, OW = (padding["height"], padding["width"]) if padding else (H, W)
    if padding:
        if OW < W or OH < H or (OW - W) % 2 or (OH - H) % 2:
            raise ValueError("invalid padding")
        p = np.zeros(u.shape[:-2] + (OH, OW), dtype=np.complex128)
        oy, ox = (OH - H) // 2, (OW - W) // 2
        p[..., oy:oy + H, ox:ox + W] = u
        u = p
    tf = as_transfer_function(OH, OW, lam, z, dx, filt, phase_mode)
    return _fft2(_fft2(u.astype(np.complex128)) * tf, inverse=True)


# -------------------------------------------------------------------------------------------------
# a11-a13: Mean, MeanAbs, moment weights (holonp/src/mean.cu:268-305; holotask/src/syncs/
# mean_abs.cu:240-275; holonp/src/arange.cu:62-75; graph_builder.cc:578-631)
# -------------------------------------------------------------------------------------------------

def mean(x: np.ndarray, axes: Sequence[int], keepdims: bool = True) -> np.ndarray:
    return np.mean(np.asarray(x, dtype=np.complex128 if np.iscomplexobj(x) else np.float64),
                   axis=tuple(axes), keepdims=keepdims)


def mean_abs(x: np.ndarray, axes: Sequence[int], keepdims: bool = True) -> np.ndarray:
    return np.mean(np.abs(np.asarray(x)), axis=tuple(axes), keepdims=keepdims)


def arange_len(start: float, stop: float, step: float) -> int:
    """arange.cu arange_len: ceil((stop-start)/step), 0 for empty ranges."""
    if (step > 0 and stop <= start) or (step < 0 and stop >= start):
        return 0
    n = math.ceil((stop - start) / step)
    if not math.isfinite(n) or n <= 0:
        raise ValueError("invalid arange length")
    return int(n)


def arange_f32(start: float, stop: float, step: float) -> np.ndarray:
    """arange_kernel_scalar: v = start + step*i in double, then cast to float32."""
    n = arange_len(start, stop, step)
    return (start + step * np.arange(n, dtype=np.float64)).astype(F32)


def freq_weights(T: int, z0: int, z1: int, fs: float = 37e3, method: str = "rfft") -> np.ndarray:
    """build_freq_weights (graph_builder.cc:578-602): df = fs/T, f0 = z0*df, f1 = z1*df.

    The reference hard-codes fs = 37e3; it is a parameter here.  For the two-sided FFT method the
    negative band is arange(f0-fs, f1-fs, df).
    """
    df = fs / float(T)
    f0, f1 = z0 * df, z1 * df
    pos = arange_f32(f0, f1, df)
    if method == "fft":
        return np.concatenate([pos, arange_f32(f0 - fs, f1 - fs, df)])
    return pos


def moments_from_magnitude(mag: np.ndarray, weights: np.ndarray, fftshift: bool = False):
    """M0 = mean_k |S_k|, M1 = mean_k f_k |S_k|, M2 = mean_k f_k^2 |S_k| over axis 0.

    graph_builder.cc:612-631: the M2 weights are freqs*freqs formed in float32 before the
    multiply.  Returns float64 [3, H, W]; optional fftshift over the image axes
    (graph_builder.cc:633-635, numpy semantics).
    """
    w1 = np.asarray(weights, dtype=F32)
    w2 = (w1 * w1).astype(F32)
    m = np.asarray(mag, dtype=np.float64)
    nz = m.shape[0]
    m0 = m.sum(axis=0) / nz
    m1 = np.tensordot(w1.astype(np.float64), m, axes=(0, 0)) / nz
    m2 = np.tensordot(w2.astype(np.float64), m, axes=(0, 0)) / nz
    out = np.stack([m0, m1, m2])
    if fftshift:
        out = np.fft.fftshift(out, axes=(-2, -1))
    return out


# -------------------------------------------------------------------------------------------------
# a14: the per-window path end to end (graph_builder.cc:245-305 TFA, 522-566 propagation,
# 604-678 view), with the SVD clutter filter of the full-size workload inserted before the band DFT
# -------------------------------------------------------------------------------------------------

@dataclass
class PathConfig:
    height: int
    width: int
    frames: int                    # T, window length
    hop: int                       # S, window stride
    z0: int                        # first band bin
    z1: int                        # one past the last band bin
    fs: float = 37e3               # sampling rate used by the moment weights
    propagation: str = "fresnel"   # "fresnel" | "angular_spectrum" | "none"
    lam: float = 852e-9
    pitch: float = 12e-6
    z: float = 0.25
    clutter_rank: int = 0          # eigenvectors removed by the SVD filter (0 = no filter)
    fftshift: bool = False
    as_filter: Optional[dict] = None
    as_padding: Optional[dict] = None
    phase_mode: str = "f32"
    time_method: str = "rfft"      # "rfft" (one-sided band) | "fft" (two-sided, 2 Nz planes)
    filter2d: Optional[dict] = None  # r_inner/r_outer/s_inner/s_outer: Filter2D on the band planes
                                     # before Fresnel (graph_builder.cc:124-126)
    autofocus: Optional[dict] = None  # nb, orders, n_iter, roi_radius, keep_outside: Shack-Hartmann
                                      # autofocus before Fresnel (graph_builder.cc:139-153)

    @property
    def nz(self) -> int:
        return (self.z1 - self.z0) * (2 if self.time_method == "fft" else 1)


def band_planes(window: np.ndarray, cfg: PathConfig) -> np.ndarray:
    """[Nz, H, W] complex: SVD filter (optional) then the band DFT along time."""
    X = np.asarray(window, dtype=np.float64).reshape(cfg.frames, -1)
    V = clutter_basis(X, cfg.clutter_rank) if cfg.clutter_rank else None
    Wm = band_matrix(cfg.frames, cfg.z0, cfg.z1, V, cfg.time_method)
    S = Wm.T @ X  # [Nz, P]
    return S.reshape(cfg.nz, cfg.height, cfg.width)


def propagate(planes: np.ndarray, cfg: PathConfig) -> np.ndarray:
    if cfg.propagation == "fresnel":
        return fresnel(planes, cfg.lam, cfg.pitch, cfg.pitch, cfg.z, output_magnitude=True,
                       phase_mode=cfg.phase_mode)
    if cfg.propagation == "angular_spectrum":
        return np.abs(angular_spectrum(planes, cfg.lam, cfg.pitch, cfg.pitch, cfg.z,
                                       cfg.as_filter, cfg.as_padding, cfg.phase_mode))
    if cfg.propagation == "none":
        return np.abs(planes)
    raise ValueError(cfg.propagation)


def reconstruct_window(window: np.ndarray, cfg: PathConfig) -> np.ndarray:
    """One T-frame window -> float64 [3, H', W'] (M0, M1, M2)."""
    planes = band_planes(window, cfg)
    if cfg.filter2d and cfg.propagation != "angular_spectrum":
        f = cfg.filter2d
        planes = filter2d(planes, f["r_inner"], f["r_outer"], f["s_inner"], f["s_outer"])
    if cfg.autofocus and cfg.autofocus.get("orders"):
        planes = autofocus_planes(planes, cfg)[0]
    mag = propagate(planes, cfg)
    w = freq_weights(cfg.frames, cfg.z0, cfg.z1, cfg.fs, cfg.time_method)
    return moments_from_magnitude(mag, w, cfg.fftshift)


def autofocus_planes(planes: np.ndarray, cfg: PathConfig):
    """The autofocus passes on one window's band planes (oracle/shack.py); returns the corrected
    planes and the coefficients summed over the passes."""
    from . import shack as SH
    a = cfg.autofocus
    acfg = SH.AutofocusConfig(a["nb"], cfg.lam, cfg.pitch, cfg.z, list(a["orders"]), a.get("roi_radius", 0.5),
                              not a.get("keep_outside", False), a.get("flatfield_period", 0.0),
                              bool(a.get("full_pairwise", False)))
    total = np.zeros(len(acfg.indexes))
    cur = np.asarray(planes, np.complex128)
    for _ in range(a.get("n_iter", 1)):
        r = SH.autofocus(cur, acfg)
        cur, total = r[4], total + r[2]
    return cur, total


def reconstruct_sequence(windows: Sequence[np.ndarray], cfg: PathConfig) -> list:
    """Consecutive windows of one stream with the autofocus over pp_accumulation = n > 1 spectra
    (graph_builder.cc:128-153, 348): window w's sub-aperture M0 images enter a causal sliding
    average over the last n windows; the fit of that average corrects the DELAYED window w - d,
    d = (n - 1) // 2, which the dual-reader queue supplies (dual_reader_batch_queue.cc:214-227;
    zero planes while the stream is younger than d windows).  Output w is the moments of the
    corrected delayed window (zeros for w < d).  One autofocus pass (graph_builder.cc:143-146)."""
    from . import shack as SH
    a = cfg.autofocus
    n = int(a.get("pp_accumulation", 1))
    if a.get("n_iter", 1) != 1 and n > 1:
        raise ValueError("sliding Shack-Hartmann correction only supports one autofocus iteration")
    d = (n - 1) // 2
    acfg = SH.AutofocusConfig(a["nb"], cfg.lam, cfg.pitch, cfg.z, list(a["orders"]), a.get("roi_radius", 0.5),
                              not a.get("keep_outside", False), a.get("flatfield_period", 0.0),
                              bool(a.get("full_pairwise", False)))
    avg = SH.CausalSlidingAverage(n) if n > 1 else None
    weights = freq_weights(cfg.frames, cfg.z0, cfg.z1, cfg.fs, cfg.time_method)
    hist, outs = [], []
    for w, win in enumerate(windows):
        planes = band_planes(win, cfg)
        hist.append(planes)
        delayed = hist[w - d] if w >= d else np.zeros_like(planes)
        corrected = SH.autofocus(planes, acfg, delayed=delayed, average=avg)[4]
        outs.append(moments_from_magnitude(propagate(corrected, cfg), weights, cfg.fftshift))
    return outs


def band_bins(f_lo: float, f_hi: float, fs: float, T: int) -> tuple[int, int]:
    """z0 = ceil(f_lo/df), z1 = floor(f_hi/df) + 1 with df = fs/T, clipped to the RFFT range."""
    df = fs / T
    z0 = int(math.ceil(f_lo / df - 1e-9))
    z1 = int(math.floor(f_hi / df + 1e-9)) + 1
    return max(z0, 0), min(z1, T // 2 + 1)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / ||b|| over all elements (complex-aware, float64/complex128)."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    a = np.asarray(a, dtype=np.complex128 if cplx else np.float64)
    b = np.asarray(b, dtype=np.complex128 if cplx else np.float64)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n else float(d)


# ----------------------------------------------------------------------------------------------
# Post-moment display chain (graph_builder.cc:633-676)
# ----------------------------------------------------------------------------------------------
def fftshift_ref(x: np.ndarray, axes: Optional[Sequence[int]] = None) -> np.ndarray:
    """holonp/src/fftshift.cu:98-134: out[j] = x[(j + n // 2) % n] along each shifted axis (numpy's
    fftshift for even n, its ifftshift for odd n)."""
    out = x
    for a in (range(x.ndim) if axes is None else axes):
        out = np.roll(out, -(x.shape[a] // 2), axis=a)
    return out


def gaussian_taps(sigma: float) -> np.ndarray:
    """make_gaussian_kernel (flatfield.cu:57-77): radius ceil(3 sigma) in float32, taps
    exp(-i^2 / (2 sigma^2)) normalized to sum 1 (float64 here)."""
    r = int(math.ceil(float(np.float32(3.0) * np.float32(sigma))))
    if r <= 0:
        raise ValueError("sigma is too small to form a Gaussian kernel")
    i = np.arange(-r, r + 1, dtype=np.float64)
    w = np.exp(-(i * i) / (2.0 * float(sigma) ** 2))
    return w / w.sum()


def flatfield_uses_fourier(height: int, width: int, sigma_y: float, sigma_x: float) -> bool:
    """should_use_fft_flatfield (flatfield.cu:169-174): kernels of 65 taps or more."""
    n = max(len(gaussian_taps(sigma_y)), len(gaussian_taps(sigma_x)))
    return height > 1 and width > 1 and n >= 65


def flatfield_spatial(x: np.ndarray, sigma_y: float, sigma_x: float) -> np.ndarray:
    """flatfield.cu:179-221: out = x - Gy * (Gx * x) with clamp-at-edge borders, per [H][W] plane."""
    x = np.asarray(x, dtype=np.float64)
    ky, kx = gaussian_taps(sigma_y), gaussian_taps(sigma_x)
    ry, rx = len(ky) // 2, len(kx) // 2
    H, W = x.shape[-2:]
    xi = np.clip(np.arange(W)[:, None] + np.arange(-rx, rx + 1)[None, :], 0, W - 1)   # [W][taps]
    tmp = np.einsum("...yk,k->...y", x[..., :, xi].reshape(*x.shape[:-1], W, len(kx)), kx)
    yi = np.clip(np.arange(H)[:, None] + np.arange(-ry, ry + 1)[None, :], 0, H - 1)   # [H][taps]
    bg = np.einsum("...hkw,k->...hw", tmp[..., yi, :], ky)
    return x - bg


def _six_decimals(v: float) -> float:
    """std::to_string(float): the value the reference's JIT source holds (flatfield.cu:124-131)."""
    return float("%f" % float(np.float32(v)))


def flatfield_fourier(x: np.ndarray, sigma_y: float, sigma_x: float) -> np.ndarray:
    """flatfield.cu:121-158, 229-233: R2C FFT, x (1 - exp(-2 pi^2 (sx^2 fx^2 + sy^2 fy^2))) * SCALE,
    C2R FFT (unnormalized), with sigma and SCALE = 1 / (W H) at six decimals as the JIT source has
    them."""
    x = np.asarray(x, dtype=np.float64)
    H, W = x.shape[-2:]
    sy, sx = _six_decimals(sigma_y), _six_decimals(sigma_x)
    scale = _six_decimals(1.0 / (W * H))
    fx = np.arange(W // 2 + 1) / W
    y = np.arange(H)
    fy = np.where(y <= H // 2, y, y - H) / H
    low = np.exp(-2.0 * math.pi ** 2 * (sx * sx * fx[None, :] ** 2 + sy * sy * fy[:, None] ** 2))
    gain = (1.0 - low) * scale
    spec = np.fft.rfft2(x, axes=(-2, -1)) * gain
    return np.fft.irfft2(spec, s=(H, W), axes=(-2, -1)) * (W * H)


def ellipse_mask(depth: int, height: int, width: int, cx: float, cy: float, rx: float, ry: float,
                 angle: float) -> np.ndarray:
    """in_ellipse (pct_clip.cu:91-110) in float32 for a zero angle (cos = 1, sin = 0 exactly)."""
    if angle != 0.0:
        raise ValueError("the float32 restatement covers angle 0 only")
    f = np.float32
    xn = (np.arange(width, dtype=f) + f(0.5)) / f(width)
    yn = (np.arange(height, dtype=f) + f(0.5)) / f(height)
    dx, dy = xn[None, :] - f(cx), yn[:, None] - f(cy)
    m = (dx * dx) / (f(rx) * f(rx)) + (dy * dy) / (f(ry) * f(ry)) <= f(1.0)
    return np.broadcast_to(m, (depth, height, width))


def pct_clip(x: np.ndarray, min_pct: float, max_pct: float, mask: np.ndarray):
    """pct_clip.cu:117-145, 283-296: sort the masked values, take ranks int(p/100 (n-1)) in float32,
    clip every pixel to them.  Returns (clipped float32, lo, hi)."""
    v = np.sort(np.asarray(x, dtype=np.float32)[mask])
    n = v.size
    lo_i = int(np.float32(min_pct) / np.float32(100.0) * np.float32(n - 1))
    hi_i = int(np.float32(max_pct) / np.float32(100.0) * np.float32(n - 1))
    lo, hi = v[lo_i], v[hi_i]
    return np.minimum(np.maximum(np.asarray(x, dtype=np.float32), lo), hi), lo, hi


def slide_avg(images: Sequence[np.ndarray], window: int, discard_first: int = 0) -> list:
    """slide_avg.cu:211-250 in float32: avg += x / n; avg -= x_(k-n) / n (zeros before the first
    n images); one output per image once n images have entered."""
    f = np.float32
    n = f(window)
    avg, ring, outs, k = None, [], [], 0
    for i, img in enumerate(images):
        if i < discard_first:
            continue
        img = np.asarray(img, dtype=f)
        if avg is None:
            avg = np.zeros_like(img)
            ring = [np.zeros_like(img) for _ in range(window)]
        old = ring[k % window]
        avg = (avg + img / n).astype(f)
        avg = (avg - old / n).astype(f)
        ring[k % window] = img
        k += 1
        if k >= window:
            outs.append(avg.copy())
    return outs


def filter2d_mask(height: int, width: int, r_inner: int, r_outer: int, s_inner: int, s_outer: int,
                  real: bool) -> np.ndarray:
    """The Filter2D annulus a (1 - b) in natural frequency order (filter2d.cu:109-199), float32.
    Complex input: the centred mask, corners swapped (fftshift for even sides).  Real input: the
    R2C half spectrum [H][W/2+1], with the `smooth > 0` guards."""
    f = np.float32

    def annulus(dist, guards):
        ri, ro, si, so = f(r_inner), f(r_outer), f(s_inner), f(s_outer)
        with np.errstate(divide="ignore", invalid="ignore"):
            a = np.where(dist < ro, f(1), np.where((so > 0 if guards else True) & (dist < ro + so),
                                                   np.cos((dist - ro) / so * f(np.pi) / f(2)), f(0)))
            b = np.where(dist < ri, f(1), np.where((si > 0 if guards else True) & (dist < ri + si),
                                                   np.cos((dist - ri) / si * f(np.pi) / f(2)), f(0)))
        return (a * (f(1) - b)).astype(f)

    if real:
        x = np.arange(width // 2 + 1, dtype=f)
        y = np.arange(height)
        fy = np.where(y <= height // 2, y, y - height).astype(f)
        return annulus(np.hypot(x[None, :], fy[:, None]), True)
    x = np.arange(width, dtype=f) - f(width) / f(2)
    y = np.arange(height, dtype=f) - f(height) / f(2)
    centred = annulus(np.hypot(x[None, :], y[:, None]), False)
    return np.fft.ifftshift(centred)


def filter2d(x: np.ndarray, r_inner: int, r_outer: int, s_inner: int, s_outer: int) -> np.ndarray:
    """Filter2D (filter2d.cu:229-244): complex planes -> FFT2 x (g + i g) -> IFFT2, real planes ->
    RFFT2 x g -> IRFFT2; both unnormalized (cuFFT), per [H][W] plane."""
    H, W = x.shape[-2:]
    if np.iscomplexobj(x):
        g = filter2d_mask(H, W, r_inner, r_outer, s_inner, s_outer, False).astype(np.float64)
        spec = np.fft.fft2(np.asarray(x, dtype=np.complex128), axes=(-2, -1)) * (g + 1j * g)
        return np.fft.ifft2(spec, axes=(-2, -1)) * (H * W)
    g = filter2d_mask(H, W, r_inner, r_outer, s_inner, s_outer, True).astype(np.float64)
    spec = np.fft.rfft2(np.asarray(x, dtype=np.float64), axes=(-2, -1)) * g
    return np.fft.irfft2(spec, s=(H, W), axes=(-2, -1)) * (H * W)
