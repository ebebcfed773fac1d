"""Shack-Hartmann autofocus on torch CUDA tensors (include/holoflow_b200.h, hf_stfd_* /
hf_shslopes_* / hf_zernike_* / hf_correct_phase / hf_wrap2pi / hf_autofocus_*), the reference's
ShortTimeFresnelDiffraction, ShackHartmannSlopes, ZernikeFromSlopes, ZernikePhase, CorrectPhase,
Wrap2Pi and ZernikeDefocusZProp operators and their chain (graph_builder.cc:307-501).

    af = Autofocus(nz=16, height=512, width=512, nb_subaps=5, lam=852e-9, dx=20e-6, z=0.25,
                   indexes=[4, 5, 6])
    corrected = af(planes)          # planes: [nz][512][512] complex64 band planes of one spectrum
    af.coefficients()               # radians, in `indexes` order
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

import torch

from . import (HF_STFD_COMPLEX, HF_STFD_GLOBAL, HF_STFD_LOCAL, HF_STFD_MAGNITUDE, HF_STFD_MEAN_MAGNITUDE, HfEllipse,
               check, lib)
from .pipeline import _ptr, _stream

_OUTPUTS = {"complex": HF_STFD_COMPLEX, "magnitude": HF_STFD_MAGNITUDE, "mean_magnitude": HF_STFD_MEAN_MAGNITUDE}


class _Handle:
    _destroy = ""

    def __init__(self):
        self._h = C.c_void_p()

    def close(self) -> None:
        if self._h:
            getattr(lib(), self._destroy)(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ShortTimeFresnel(_Handle):
    """ShortTimeFresnelDiffraction over fields [..., H, W] (complex64 or float32).  output:
    "complex" [..., ny, nx, win_h, win_w] complex64, "magnitude" the same in float32, or
    "mean_magnitude" [ny, nx, win_h, win_w], the mean of |.| over the leading axes (the band), each
    window fftshifted when fftshift_windows."""
    _destroy = "hf_stfd_destroy"

    def __init__(self, shape: Sequence[int], win: Tuple[int, int], stride: Tuple[int, int], lam: float, dx: float,
                 dy: float, z: float, phase_ref: str = "local", output: str = "complex",
                 skip_phase_shift: bool = True, fftshift_windows: bool = False, real_input: bool = False, stream=None):
        super().__init__()
        planes = 1
        for n in shape[:-2]:
            planes *= n
        self.shape, self.output, self.real_input = tuple(shape), output, real_input
        ref = {"local": HF_STFD_LOCAL, "global": HF_STFD_GLOBAL}[phase_ref.lower()]
        check(lib().hf_stfd_create(planes, shape[-2], shape[-1], int(real_input), win[0], win[1], stride[0], stride[1],
                                   lam, dx, dy, z, ref, _OUTPUTS[output], int(skip_phase_shift),
                                   int(fftshift_windows), _stream(stream), C.byref(self._h)))
        ny, nx = C.c_int(), C.c_int()
        check(lib().hf_stfd_grid(self._h, C.byref(ny), C.byref(nx)))
        self.grid, self.win = (ny.value, nx.value), tuple(win)

    def out_shape(self) -> tuple:
        if self.output == "mean_magnitude":
            return self.grid + self.win
        return self.shape[:-2] + self.grid + self.win

    def set_z(self, z: float, stream=None) -> None:
        check(lib().hf_stfd_set_z(self._h, z, _stream(stream)))

    def __call__(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        want = torch.float32 if self.real_input else torch.complex64
        assert x.is_cuda and x.dtype == want and tuple(x.shape) == self.shape and x.is_contiguous()
        if out is None:
            dt = torch.complex64 if self.output == "complex" else torch.float32
            out = torch.empty(self.out_shape(), dtype=dt, device=x.device)
        check(lib().hf_stfd_exec(self._h, _ptr(x), _ptr(out), _stream(stream)))
        return out


class ShackHartmannSlopes(_Handle):
    """Slopes of sub-aperture images [sy, sx, h, w] float32 -> [sy, sx, 2]: against the centre
    sample (mode "single_reference") or from every pair of active samples with the complete-graph
    Laplacian solve (mode "full_pairwise", pair_batch_size maps at a time)."""
    _destroy = "hf_shslopes_destroy"

    def __init__(self, sy: int, sx: int, height: int, width: int, lam: float, dx: float, dy: float, z: float,
                 roi: Sequence[float] = (0.5, 0.5, 0.5, 0.5, 0.0), skip_outside_pupil: bool = True,
                 sub: Tuple[int, int] = (0, 0), stride: Tuple[int, int] = (0, 0), stream=None,
                 mode: str = "single_reference", pair_batch_size: int = 256):
        super().__init__()
        self.shape = (sy, sx, height, width)
        e = HfEllipse(*[float(v) for v in roi])
        m = {"single_reference": 0, "full_pairwise": 1}[mode]
        check(lib().hf_shslopes_create_mode(sy, sx, height, width, sub[0], sub[1], stride[0], stride[1], lam, dx, dy,
                                            z, C.byref(e), int(skip_outside_pupil), m, int(pair_batch_size),
                                            _stream(stream), C.byref(self._h)))

    def active(self) -> list:
        buf = (C.c_uint8 * (self.shape[0] * self.shape[1]))()
        check(lib().hf_shslopes_active(self._h, buf))
        return [bool(v) for v in buf]

    def __call__(self, images: torch.Tensor, maps: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        assert images.is_cuda and images.dtype == torch.float32 and tuple(images.shape) == self.shape
        slopes = torch.empty(self.shape[:2] + (2,), dtype=torch.float32, device=images.device)
        check(lib().hf_shslopes_exec(self._h, _ptr(images.contiguous()), _ptr(slopes), _ptr(maps), _stream(stream)))
        return slopes


def _ints(v: Sequence[int]):
    return (C.c_int * max(1, len(v)))(*v), len(v)


class ZernikeFit(_Handle):
    """ZernikeFromSlopes: slopes [sy, sx, 2] -> coefficients (radians) in `indexes` order."""
    _destroy = "hf_zernike_fit_destroy"

    def __init__(self, sy: int, sx: int, sub: Tuple[int, int], stride: Tuple[int, int], lam: float, dx: float,
                 dy: float, indexes: Sequence[int], skip_outside_pupil: bool = True):
        super().__init__()
        self.indexes = list(indexes)
        arr, n = _ints(self.indexes)
        check(lib().hf_zernike_fit_create(sy, sx, sub[0], sub[1], stride[0], stride[1], lam, dx, dy,
                                          int(skip_outside_pupil), arr, n, C.byref(self._h)))

    @property
    def pupil_radius(self) -> float:
        r = C.c_float()
        check(lib().hf_zernike_fit_pupil_radius(self._h, C.byref(r)))
        return r.value

    def __call__(self, slopes: torch.Tensor, stream=None) -> torch.Tensor:
        assert slopes.is_cuda and slopes.dtype == torch.float32 and slopes.is_contiguous()
        out = torch.empty(len(self.indexes), dtype=torch.float32, device=slopes.device)
        check(lib().hf_zernike_fit_exec(self._h, _ptr(slopes), _ptr(out), None, _stream(stream)))
        return out

    def host(self, slopes) -> list:
        """The same fit on host memory (the reference runs it on the host)."""
        s = (C.c_float * len(slopes))(*[float(v) for v in slopes])
        out = (C.c_float * len(self.indexes))()
        check(lib().hf_zernike_fit_host(self._h, s, out))
        return list(out)


def zernike_phase(coeffs: torch.Tensor, indexes: Sequence[int], ny: int, nx: int, stream=None) -> torch.Tensor:
    arr, n = _ints(list(indexes))
    out = torch.empty((ny, nx), dtype=torch.float32, device=coeffs.device)
    check(lib().hf_zernike_phase(_ptr(coeffs), arr, n, ny, nx, _ptr(out), None, _stream(stream)))
    return out


def correct_phase(x: torch.Tensor, phase: torch.Tensor, out: Optional[torch.Tensor] = None,
                  stream=None) -> torch.Tensor:
    """x [..., H, W] (complex64 or float32) times exp(-i phase[H, W])."""
    assert x.is_cuda and x.is_contiguous() and phase.shape == x.shape[-2:]
    planes = x.numel() // (x.shape[-2] * x.shape[-1])
    if out is None:
        out = torch.empty(x.shape, dtype=torch.complex64, device=x.device)
    check(lib().hf_correct_phase(_ptr(x), int(x.dtype == torch.complex64), _ptr(phase.contiguous()), planes,
                                 x.shape[-2], x.shape[-1], _ptr(out), _stream(stream)))
    return out


def wrap2pi(x: torch.Tensor, stream=None) -> torch.Tensor:
    assert x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
    out = torch.empty_like(x)
    check(lib().hf_wrap2pi(_ptr(x), _ptr(out), x.numel(), _stream(stream)))
    return out


def defocus_z(a4: float, lam: float, z_curr: float, pupil_radius: float) -> tuple:
    """(delta 1/z, new z, delta z in mm) from the defocus coefficient (radians)."""
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    check(lib().hf_defocus_z(a4, lam, z_curr, pupil_radius, C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


class Autofocus(_Handle):
    """The autofocus chain on the band planes of one spectrum [nz, H, W] complex64."""
    _destroy = "hf_autofocus_destroy"

    def __init__(self, nz: int, height: int, width: int, nb_subaps: int, lam: float, dx: float, z: float,
                 indexes: Sequence[int] = (), n_iter: int = 1, roi_radius: float = 0.5,
                 skip_outside_pupil: bool = True, flatfield_period: float = 0.0, stream=None):
        super().__init__()
        self.shape, self.nb, self.indexes = (nz, height, width), nb_subaps, list(indexes)
        self.sub = (height // nb_subaps, width // nb_subaps)
        arr, n = _ints(self.indexes)
        check(lib().hf_autofocus_create(nz, height, width, nb_subaps, n_iter, lam, dx, z, roi_radius,
                                        int(skip_outside_pupil), arr, n, flatfield_period, _stream(stream),
                                        C.byref(self._h)))

    @property
    def pupil_radius(self) -> float:
        r = C.c_float()
        check(lib().hf_autofocus_pupil_radius(self._h, C.byref(r)))
        return r.value

    def __call__(self, planes: torch.Tensor, delayed: Optional[torch.Tensor] = None,
                 out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        for t in (planes, delayed):
            assert t is None or (t.is_cuda and t.dtype == torch.complex64 and tuple(t.shape) == self.shape
                                 and t.is_contiguous())
        if out is None:
            out = torch.empty_like(planes)
        check(lib().hf_autofocus_exec(self._h, _ptr(planes), _ptr(delayed), _ptr(out), _stream(stream)))
        return out

    def _read(self, which: int, shape: tuple, stream=None) -> torch.Tensor:
        out = torch.empty(shape, dtype=torch.float32, device="cuda")
        ptrs = [None] * 4
        ptrs[which] = _ptr(out)
        check(lib().hf_autofocus_outputs(self._h, *ptrs, _stream(stream)))
        return out

    def m0(self) -> torch.Tensor:
        """Mean sub-aperture magnitudes [nb, nb, sh, sw] of the last pass."""
        return self._read(0, (self.nb, self.nb) + self.sub)

    def slopes(self) -> torch.Tensor:
        return self._read(1, (self.nb, self.nb, 2))

    def coefficients(self) -> torch.Tensor:
        """Zernike coefficients (radians) summed over the passes, in `indexes` order."""
        return self._read(2, (len(self.indexes),))

    def phase(self) -> torch.Tensor:
        """The phase map [H, W] summed over the passes."""
        return self._read(3, self.shape[1:])
