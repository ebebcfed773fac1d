"""Python wrappers over the C ABI for device tensors (torch is used for device memory and streams
only).  Each wrapper mirrors one C entry point; errors raise :class:`holoflow_b200.HfError`."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from . import (HF_CF32, HF_F32, HF_M0, HF_M1, HF_M2, HF_MONO12P, HF_PROP_FRESNEL, HF_U16, HF_U8,
               HfDesc, check, lib)

_DT = {torch.uint8: HF_U8, torch.int16: HF_U16, torch.float32: HF_F32, torch.complex64: HF_CF32}


def _stream(stream: Optional[torch.cuda.Stream] = None) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t: Optional[torch.Tensor]) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


def unpack12(packed: torch.Tensor, npix: int, out_dtype: int = HF_F32, out: Optional[torch.Tensor] = None):
    if out is None:
        shape, dt = (npix,), {HF_U16: torch.int16, HF_F32: torch.float32, HF_CF32: torch.complex64}[out_dtype]
        out = torch.empty(shape, dtype=dt, device=packed.device)
    check(lib().hf_unpack12(_ptr(packed), _ptr(out), out_dtype, npix, _stream()))
    return out


def pack12(values_u16: torch.Tensor) -> torch.Tensor:
    n = values_u16.numel()
    out = torch.empty(n * 3 // 2, dtype=torch.uint8, device=values_u16.device)
    check(lib().hf_pack12(_ptr(values_u16), _ptr(out), n, _stream()))
    return out


def temporal_dft(frames: torch.Tensor, dtype: int, batch: int, T: int, P: int, z0: int, z1: int,
                 norm: int = 0) -> torch.Tensor:
    out = torch.empty((batch, z1 - z0, P), dtype=torch.complex64, device=frames.device)
    check(lib().hf_temporal_dft(_ptr(frames), dtype, batch, T, P, z0, z1, norm, _ptr(out), _stream()))
    return out


def covariance(frames: torch.Tensor, dtype: int, batch: int, T: int, P: int) -> torch.Tensor:
    ws_bytes = lib().hf_covariance_workspace_bytes(T, P) * batch
    ws = torch.empty(max(ws_bytes, 16), dtype=torch.uint8, device=frames.device)
    gram = torch.empty((batch, T, T), dtype=torch.float64, device=frames.device)
    check(lib().hf_covariance(_ptr(frames), dtype, batch, T, P, _ptr(gram), _ptr(ws), _stream()))
    return gram


def covariance_noalloc(frames: torch.Tensor, dtype: int, batch: int, T: int, P: int,
                       gram: torch.Tensor) -> torch.Tensor:
    """Gram matrices into the caller's `gram` [batch][T][T] float64 using the library's fixed
    device workspace: the call allocates nothing (hf_covariance_noalloc)."""
    check(lib().hf_covariance_noalloc(_ptr(frames), dtype, batch, T, P, _ptr(gram), _stream()))
    return gram


def eigh_jacobi(a: torch.Tensor):
    batch, n, _ = a.shape
    evecs = torch.empty_like(a)
    evals = torch.empty((batch, n), dtype=torch.float64, device=a.device)
    info = torch.empty((batch,), dtype=torch.int32, device=a.device)
    check(lib().hf_eigh_jacobi_f64(_ptr(a.contiguous()), _ptr(evecs), _ptr(evals), _ptr(info), n, batch,
                                   _stream()))
    return evals, evecs, info


def eigh_top(a: torch.Tensor, r: int):
    """The r largest eigenpairs: (evals [batch][r] ascending, evecs [batch][n][r], info)."""
    batch, n, _ = a.shape
    a = a.contiguous()
    evecs = torch.zeros_like(a)
    evals = torch.zeros((batch, n), dtype=torch.float64, device=a.device)
    info = torch.empty((batch,), dtype=torch.int32, device=a.device)
    check(lib().hf_eigh_top_f64(_ptr(a), _ptr(evecs), _ptr(evals), _ptr(info), n, r, batch, _stream()))
    return evals[:, n - r:], evecs[:, :, n - r:], info


@dataclass
class PipelineConfig:
    height: int
    width: int
    frames: int
    hop: int
    z_begin: int
    z_end: int
    input_dtype: int = HF_MONO12P
    propagation: int = HF_PROP_FRESNEL
    clutter_rank: int = 0
    moment_mask: int = HF_M0 | HF_M1 | HF_M2
    fftshift: int = 0
    form: int = 0
    max_batch: int = 1
    lam: float = 852e-9
    pitch: float = 12e-6
    z: float = 0.25
    fs: float = 37e3
    pad_w: int = 0
    pad_h: int = 0
    as_filter: int = 0
    r_inner: int = 0
    r_outer: int = 0
    s_inner: int = 0
    s_outer: int = 0
    time_method: int = 0  # HF_TIME_RFFT; HF_TIME_FFT = two-sided band, 2 (z_end - z_begin) planes
    autofocus_nb_subaps: int = 0  # Shack-Hartmann autofocus before the lens (odd; 0 = off)
    autofocus_n_iter: int = 1
    autofocus_orders: Sequence[int] = ()  # Noll indexes 2..10 (empty = off)
    autofocus_roi_radius: float = 0.5
    autofocus_keep_outside: int = 0
    autofocus_flatfield_period: float = 0.0  # pp_flatfield cutoff period [m] on the sub-aperture images
    autofocus_pp_accumulation: int = 1  # sliding correction over n windows, applied to window w - (n - 1) / 2
    autofocus_full_pairwise: int = 0    # graph-Laplacian (full pairwise) slopes

    def desc(self) -> HfDesc:
        orders = list(self.autofocus_orders)
        return HfDesc(self.height, self.width, self.frames, self.hop, self.z_begin, self.z_end,
                      self.input_dtype, self.propagation, self.clutter_rank, self.moment_mask,
                      self.fftshift, self.form, self.max_batch, self.lam, self.pitch, self.z, self.fs,
                      self.pad_w, self.pad_h, self.as_filter, self.r_inner, self.r_outer,
                      self.s_inner, self.s_outer, self.time_method, self.autofocus_nb_subaps,
                      self.autofocus_n_iter, len(orders), (C.c_int32 * 9)(*orders), self.autofocus_roi_radius,
                      self.autofocus_keep_outside, self.autofocus_flatfield_period,
                      self.autofocus_pp_accumulation, self.autofocus_full_pairwise)

    @property
    def frame_bytes(self) -> int:
        P = self.height * self.width
        return {HF_MONO12P: 3 * P // 2, HF_U16: 2 * P, HF_U8: P, HF_F32: 4 * P}[self.input_dtype]


class Pipeline:
    """Owns an hf_plan; ``run(ring, first_frame, nwin)`` reconstructs nwin windows of a device ring."""

    def __init__(self, cfg: PipelineConfig, stream: Optional[torch.cuda.Stream] = None):
        self.cfg = cfg
        self._plan = C.c_void_p()
        d = cfg.desc()
        check(lib().hf_plan_create(C.byref(d), C.byref(self._plan), _stream(stream)))
        oh, ow, nm = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().hf_plan_output_shape(self._plan, C.byref(oh), C.byref(ow), C.byref(nm)))
        self.out_shape = (nm.value, oh.value, ow.value)

    def device_bytes(self) -> int:
        b = C.c_size_t()
        check(lib().hf_plan_device_bytes(self._plan, C.byref(b)))
        return b.value

    def band_pass(self) -> int:
        """Which band-DFT pass the plan runs: HF_BAND_FP32, HF_BAND_TC_ROWS, HF_BAND_TC_RAW_ROWS or
        HF_BAND_TC_SEGMENTS."""
        k = C.c_int()
        check(lib().hf_plan_band_pass(self._plan, C.byref(k)))
        return k.value

    def set_z(self, z: float, stream=None) -> None:
        check(lib().hf_plan_set_z(self._plan, z, _stream(stream)))

    def run(self, ring: torch.Tensor, ring_frames: int, first_frame: int, nwin: int,
            out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        if out is None:
            out = torch.empty((nwin, *self.out_shape), dtype=torch.float32, device=ring.device)
        check(lib().hf_pipeline_exec(self._plan, _ptr(ring), ring_frames, first_frame, nwin, _ptr(out),
                                     _stream(stream)))
        return out

    def inspect(self, w: int = 0):
        T, nz = self.cfg.frames, (self.cfg.z_end - self.cfg.z_begin) * (2 if self.cfg.time_method else 1)
        gram = torch.empty((T, T), dtype=torch.float64, device="cuda") if self.cfg.clutter_rank else None
        wm = torch.empty((T, nz), dtype=torch.complex64, device="cuda")
        check(lib().hf_pipeline_inspect(self._plan, w, _ptr(gram), _ptr(wm), _stream()))
        return gram, wm

    def status(self, reset: bool = True) -> int:
        st = C.c_int()
        check(lib().hf_plan_status(self._plan, C.byref(st), int(reset)))
        return st.value

    def timing(self, enable: bool) -> None:
        check(lib().hf_plan_timing(self._plan, int(enable)))

    def stage_times(self):
        """{stage: (total ms, execs)} of the execs recorded since timing(True)."""
        ms = (C.c_float * 16)()  # HF_MAX_STAGES
        names = (C.c_char_p * 16)()
        ns, ne = C.c_int(), C.c_int()
        check(lib().hf_plan_stage_times(self._plan, ms, names, C.byref(ns), C.byref(ne)))
        return {names[k].decode(): (ms[k], ne.value) for k in range(ns.value)}

    def autofocus_reset(self, stream=None) -> None:
        """Starts a new window sequence (pp_accumulation): clears the sliding average and the kept
        delayed windows."""
        check(lib().hf_plan_autofocus_reset(self._plan, _stream(stream)))

    def autofocus_coefficients(self, w: int = 0) -> torch.Tensor:
        """Window w's Zernike coefficients (radians, autofocus_orders order) of the last run."""
        out = torch.empty(len(self.cfg.autofocus_orders), dtype=torch.float32, device="cuda")
        check(lib().hf_plan_autofocus_coefficients(self._plan, w, _ptr(out), _stream()))
        return out

    def close(self) -> None:
        if self._plan:
            lib().hf_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FresnelPlan:
    def __init__(self, batch, H, W, in_dtype, lam, dx, z, output_magnitude=False, skip_phase_shift=True):
        self._p = C.c_void_p()
        self.shape = (batch, H, W)
        self.magnitude = output_magnitude
        check(lib().hf_fresnel_plan_create(batch, H, W, in_dtype, lam, dx, z, int(output_magnitude),
                                           int(skip_phase_shift), C.byref(self._p), _stream()))

    def set_z(self, z):
        check(lib().hf_fresnel_plan_set_z(self._p, z, _stream()))

    def __call__(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        B, H, W = self.shape
        if out is None:
            out = torch.empty((B, H, W), dtype=torch.float32 if self.magnitude else torch.complex64,
                              device=x.device)
        sx = x.stride()
        so = out.stride()
        check(lib().hf_fresnel_exec(self._p, _ptr(x), sx[0], sx[1], sx[2], _ptr(out), so[0], so[1], so[2],
                                    _stream()))
        return out

    def __del__(self):
        try:
            lib().hf_fresnel_plan_destroy(self._p)
        except Exception:
            pass


class AngularSpectrumPlan:
    def __init__(self, batch, H, W, in_dtype, lam, dx, z, padding=None, filt=None):
        self._p = C.c_void_p()
        pw, ph = (padding["width"], padding["height"]) if padding else (0, 0)
        f = filt or {}
        self.out_shape = (batch, ph or H, pw or W)
        check(lib().hf_as_plan_create(batch, H, W, in_dtype, lam, dx, z, pw, ph, int(filt is not None),
                                      f.get("r_inner", 0), f.get("r_outer", 0), f.get("s_inner", 0),
                                      f.get("s_outer", 0), C.byref(self._p), _stream()))

    def __call__(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if out is None:
            out = torch.empty(self.out_shape, dtype=torch.complex64, device=x.device)
        check(lib().hf_as_exec(self._p, _ptr(x), _ptr(out), _stream()))
        return out

    def __del__(self):
        try:
            lib().hf_as_plan_destroy(self._p)
        except Exception:
            pass


class CameraStream:
    """A device ring + window cursor bound to a Pipeline (hf_stream_*)."""

    def __init__(self, pipeline: Pipeline, ring_frames: int):
        self.pipeline = pipeline
        self._s = C.c_void_p()
        check(lib().hf_stream_create(pipeline._plan, ring_frames, C.byref(self._s)))

    def push(self, frames: torch.Tensor, nframes: int, stream=None) -> None:
        check(lib().hf_stream_push(self._s, _ptr(frames), nframes, _stream(stream)))

    def ready(self) -> int:
        return lib().hf_stream_ready(self._s)

    def process(self, max_windows: int, out: torch.Tensor, stream=None, async_copy: bool = False) -> int:
        """Reconstructs up to `max_windows` ready windows into `out` (device, or pinned host).
        With a host `out` and async_copy, the D2H copy overlaps later work: call output_wait()
        before reading `out`."""
        n = C.c_int()
        mode = 0 if out.is_cuda else (2 if async_copy else 1)
        check(lib().hf_stream_process(self._s, max_windows, _ptr(out), mode, C.byref(n), _stream(stream)))
        return n.value

    def output_wait(self, stream=None, host_block: bool = False) -> None:
        """Waits for the latest asynchronous output copy (on the host, or by making `stream` wait)."""
        check(lib().hf_stream_output_wait(self._s, _stream(stream), int(host_block)))

    def close(self):
        if self._s:
            lib().hf_stream_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
