"""Post-moment display chain on torch CUDA tensors (include/holoflow_b200.h, hf_fftshift /
hf_flatfield_* / hf_pctclip_* / hf_slideavg_*): the steps between a moment image and the display
(graph_builder.cc:633-676), ending with ``pipeline.convert(..., HF_CONV_SCALED)`` to U8.

    ff = Flatfield((1, 1024, 1024), sigma_y=18.7, sigma_x=18.7)
    sa = SlidingAverage(1024 * 1024, window_size=4)
    pc = PctClip((1, 1024, 1024), 0.5, 99.5, roi=(0.5, 0.5, 0.5, 0.5, 0.0))
    img = ff(m0); avg = sa.push(img); img = pc(avg) if avg is not None else None
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import torch

from . import HfEllipse, check, lib
from .pipeline import _ptr, _stream


def fftshift(x: torch.Tensor, axes: Optional[Sequence[int]] = None, out: Optional[torch.Tensor] = None,
             stream=None) -> torch.Tensor:
    """holonp FFTShift: out[j] = x[(j + n // 2) % n] along `axes` (all axes when None)."""
    assert x.is_cuda and x.is_contiguous()
    if out is None:
        out = torch.empty_like(x)
    nd = x.dim()
    mask = (1 << nd) - 1 if axes is None else sum(1 << (a % nd) for a in axes)
    shape = (C.c_int64 * nd)(*x.shape)
    check(lib().hf_fftshift(_ptr(x), _ptr(out), x.element_size(), nd, shape, mask, _stream(stream)))
    return out


class Flatfield:
    """out = x - Gaussian(x) on every [H][W] plane of x (sigmas in pixels)."""

    def __init__(self, shape: Sequence[int], sigma_y: float, sigma_x: float, stream=None):
        planes = 1
        for n in shape[:-2]:
            planes *= n
        self.shape = tuple(shape)
        self._f = C.c_void_p()
        check(lib().hf_flatfield_create(planes, shape[-2], shape[-1], sigma_y, sigma_x, _stream(stream),
                                        C.byref(self._f)))

    @property
    def fourier(self) -> bool:
        v = C.c_int()
        check(lib().hf_flatfield_is_fourier(self._f, C.byref(v)))
        return bool(v.value)

    def __call__(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        assert x.is_cuda and x.dtype == torch.float32 and tuple(x.shape) == self.shape and x.is_contiguous()
        if out is None:
            out = torch.empty_like(x)
        check(lib().hf_flatfield_exec(self._f, _ptr(x), _ptr(out), _stream(stream)))
        return out

    def close(self) -> None:
        if self._f:
            lib().hf_flatfield_destroy(self._f)
            self._f = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Filter2D:
    """IFFT2(FFT2(x) x annulus) per [H][W] plane, unnormalized, of complex64 (in place allowed)
    or float32 planes (filter2d.cu)."""

    def __init__(self, shape: Sequence[int], real: bool, r_inner: int, r_outer: int, s_inner: int, s_outer: int,
                 stream=None):
        planes = 1
        for n in shape[:-2]:
            planes *= n
        self.shape, self.real = tuple(shape), real
        self._f = C.c_void_p()
        check(lib().hf_filter2d_create(planes, shape[-2], shape[-1], int(real), r_inner, r_outer, s_inner, s_outer,
                                       _stream(stream), C.byref(self._f)))

    def __call__(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        assert x.is_cuda and tuple(x.shape) == self.shape and x.is_contiguous()
        assert x.dtype == (torch.float32 if self.real else torch.complex64)
        if out is None:
            out = torch.empty_like(x)
        check(lib().hf_filter2d_exec(self._f, _ptr(x), _ptr(out), _stream(stream)))
        return out

    def close(self) -> None:
        if self._f:
            lib().hf_filter2d_destroy(self._f)
            self._f = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PctClip:
    """Clips [D][H][W] to the values at the min_pct / max_pct ranks of the pixels inside `roi`
    (cx, cy, rx, ry normalized to the image, angle in degrees)."""

    def __init__(self, shape: Sequence[int], min_pct: float, max_pct: float,
                 roi: Sequence[float] = (0.5, 0.5, 0.5, 0.5, 0.0), stream=None):
        self.shape = tuple(shape)
        self._p = C.c_void_p()
        e = HfEllipse(*roi)
        check(lib().hf_pctclip_create(shape[0], shape[1], shape[2], min_pct, max_pct, C.byref(e), _stream(stream),
                                      C.byref(self._p)))

    @property
    def roi_count(self) -> int:
        v = C.c_int()
        check(lib().hf_pctclip_roi_count(self._p, C.byref(v)))
        return v.value

    def __call__(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, bounds: Optional[torch.Tensor] = None,
                 stream=None) -> torch.Tensor:
        assert x.is_cuda and x.dtype == torch.float32 and tuple(x.shape) == self.shape and x.is_contiguous()
        if out is None:
            out = torch.empty_like(x)
        check(lib().hf_pctclip_exec(self._p, _ptr(x), _ptr(out), _ptr(bounds), _stream(stream)))
        return out

    def close(self) -> None:
        if self._p:
            lib().hf_pctclip_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SlidingAverage:
    """Mean of the last window_size images (after dropping the first discard_first)."""

    def __init__(self, npix: int, window_size: int, discard_first: int = 0, stream=None):
        self.npix = npix
        self._a = C.c_void_p()
        check(lib().hf_slideavg_create(npix, window_size, discard_first, _stream(stream), C.byref(self._a)))

    def push(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> Optional[torch.Tensor]:
        """The average once window_size images have entered, else None."""
        assert x.is_cuda and x.dtype == torch.float32 and x.numel() == self.npix and x.is_contiguous()
        if out is None:
            out = torch.empty_like(x)
        ready = C.c_int()
        check(lib().hf_slideavg_push(self._a, _ptr(x), _ptr(out), C.byref(ready), _stream(stream)))
        return out if ready.value else None

    def close(self) -> None:
        if self._a:
            lib().hf_slideavg_destroy(self._a)
            self._a = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
