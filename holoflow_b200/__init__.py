"""holoflow_b200: B200 (sm_100a) laser Doppler reconstruction — Python binding of the C ABI.

The product is the shared library ``_lib/libholoflow_b200.so`` (CUDA kernels + C ABI declared in
``include/holoflow_b200.h`` + the C++ node layer).  This module only loads it with ctypes and
declares the prototypes; every call goes straight through the C ABI.  There is no fallback: if the
library is missing or cannot be loaded, importing this package raises.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "_lib" / "libholoflow_b200.so"

# status codes / enums (include/holoflow_b200.h)
HF_OK, HF_ERR_INVALID, HF_ERR_CUDA, HF_ERR_UNSUPPORTED, HF_ERR_NOMEM, HF_ERR_TIMEOUT = 0, -1, -2, -3, -4, -5
HF_ERR_STATE, HF_ERR_CANCELLED = -6, -7
HF_TIME_RFFT, HF_TIME_FFT = 0, 1  # one-sided band / two-sided method (graph_builder.cc:270-287)
HF_U8, HF_U16, HF_F32, HF_CF32, HF_MONO12P = 0, 1, 2, 3, 16
HF_CONV_REAL, HF_CONV_SCALED, HF_CONV_MODULUS, HF_CONV_ARGUMENT = 0, 1, 2, 3
HF_NORM_BACKWARD, HF_NORM_FORWARD, HF_NORM_ORTHO = 0, 1, 2
HF_PROP_NONE, HF_PROP_FRESNEL, HF_PROP_ANGULAR_SPECTRUM = 0, 1, 2
HF_M0, HF_M1, HF_M2 = 1, 2, 4
HF_FORM_PLAIN, HF_FORM_CHOSEN = 0, 1
# band-DFT pass of a plan (hf_plan_band_pass)
HF_BAND_FP32, HF_BAND_TC_ROWS, HF_BAND_TC_RAW_ROWS, HF_BAND_TC_SEGMENTS = 0, 1, 2, 3
HF_STFD_LOCAL, HF_STFD_GLOBAL = 0, 1
HF_STFD_COMPLEX, HF_STFD_MAGNITUDE, HF_STFD_MEAN_MAGNITUDE = 0, 1, 2
HF_SHSLOPES_SINGLE_REFERENCE, HF_SHSLOPES_FULL_PAIRWISE = 0, 1


class HfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class HfDesc(C.Structure):
    _fields_ = [
        ("height", C.c_int32), ("width", C.c_int32), ("frames", C.c_int32), ("hop", C.c_int32),
        ("z_begin", C.c_int32), ("z_end", C.c_int32), ("input_dtype", C.c_int32),
        ("propagation", C.c_int32), ("clutter_rank", C.c_int32), ("moment_mask", C.c_int32),
        ("fftshift", C.c_int32), ("form", C.c_int32), ("max_batch", C.c_int32),
        ("lambda_", C.c_float), ("pitch", C.c_float), ("z", C.c_float), ("fs", C.c_float),
        ("pad_w", C.c_int32), ("pad_h", C.c_int32), ("as_filter", C.c_int32),
        ("r_inner", C.c_uint32), ("r_outer", C.c_uint32), ("s_inner", C.c_uint32),
        ("s_outer", C.c_uint32), ("time_method", C.c_int32),
        ("autofocus_nb_subaps", C.c_int32), ("autofocus_n_iter", C.c_int32), ("autofocus_n_orders", C.c_int32),
        ("autofocus_orders", C.c_int32 * 9), ("autofocus_roi_radius", C.c_float),
        ("autofocus_keep_outside", C.c_int32), ("autofocus_flatfield_period", C.c_float),
        ("autofocus_pp_accumulation", C.c_int32), ("autofocus_full_pairwise", C.c_int32),
    ]


_vp, _i32, _i64, _f32, _sz = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_size_t


class HoloHeader(C.Structure):
    """hf_holo_header: the 64-byte packed .holo header (holofile.hh:87-104 field order)."""
    _pack_ = 1
    _fields_ = [("magic_number", C.c_uint32), ("version", C.c_uint16), ("bits_per_pixel", C.c_uint16),
                ("frame_width", C.c_uint32), ("frame_height", C.c_uint32), ("frame_count", C.c_uint32),
                ("data_size_in_bytes", C.c_uint64), ("endianness", C.c_uint8), ("padding", C.c_char * 35)]


class HfEllipse(C.Structure):
    """hf_ellipse: the percentile clip's region (normalized centre and radii, angle in degrees)."""
    _fields_ = [("cx", C.c_float), ("cy", C.c_float), ("rx", C.c_float), ("ry", C.c_float), ("angle", C.c_float)]


class HfTDesc(C.Structure):
    """hf_tdesc: holoflow::core::TDesc across the C ABI (strides in bytes, zero = contiguous)."""
    _fields_ = [("rank", C.c_int32), ("dtype", C.c_int32), ("mem_loc", C.c_int32), ("reserved", C.c_int32),
                ("shape", C.c_int64 * 8), ("strides", C.c_int64 * 8), ("offset", C.c_int64)]

class HfMultiSchedule(C.Structure):
    """hf_multi_schedule: branches, assignment, fusion of the segment band passes and its tile
    parameters."""
    _fields_ = [("branches", C.c_int32), ("largest_first", C.c_int32), ("fused", C.c_int32),
                ("seg_tiles", C.c_int32), ("band_ctas", C.c_int32)]

# name -> (restype, argtypes)
_PROTOS = {
    "hf_last_error": (C.c_char_p, []),
    "hf_version": (C.c_int, []),
    "hf_launch_count": (_i64, []),
    "hf_reset_launch_count": (None, []),
    "hf_unpack12": (C.c_int, [_vp, _vp, C.c_int, _i64, _vp]),
    "hf_pack12": (C.c_int, [_vp, _vp, _i64, _vp]),
    "hf_convert": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_int, _i64, _vp, _vp]),
    "hf_temporal_dft": (C.c_int, [_vp, C.c_int, _i64, C.c_int, _i64, C.c_int, C.c_int, C.c_int, _vp, _vp]),
    "hf_covariance_workspace_bytes": (_sz, [C.c_int, _i64]),
    "hf_covariance": (C.c_int, [_vp, C.c_int, _i64, C.c_int, _i64, _vp, _vp, _vp]),
    "hf_covariance_noalloc": (C.c_int, [_vp, C.c_int, _i64, C.c_int, _i64, _vp, _vp]),
    "hf_eigh_jacobi_f64": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _i64, _vp]),
    "hf_eigh_top_f64": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _i64, _vp]),
    "hf_pca_project": (C.c_int, [_vp, _i64, C.c_int, _i64, _vp, C.c_int, C.c_int, _vp, _vp]),
    "hf_band_matrix": (C.c_int, [_vp, _i64, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp]),
    "hf_fresnel_plan_create": (C.c_int, [_i64, C.c_int, C.c_int, C.c_int, _f32, _f32, _f32, C.c_int,
                                         C.c_int, C.POINTER(_vp), _vp]),
    "hf_fresnel_plan_set_z": (C.c_int, [_vp, _f32, _vp]),
    "hf_fresnel_exec": (C.c_int, [_vp, _vp, _i64, _i64, _i64, _vp, _i64, _i64, _i64, _vp]),
    "hf_fresnel_plan_destroy": (C.c_int, [_vp]),
    "hf_as_plan_create": (C.c_int, [_i64, C.c_int, C.c_int, C.c_int, _f32, _f32, _f32, C.c_int, C.c_int,
                                    C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.POINTER(_vp), _vp]),
    "hf_as_exec": (C.c_int, [_vp, _vp, _vp, _vp]),
    "hf_as_plan_destroy": (C.c_int, [_vp]),
    "hf_mean_axis": (C.c_int, [_vp, C.c_int, _i64, _i64, _i64, _vp, _vp]),
    "hf_mean_abs_axis": (C.c_int, [_vp, C.c_int, _i64, _i64, _i64, _vp, _vp]),
    "hf_band_moments": (C.c_int, [_vp, C.c_int, C.c_int, _i64, C.POINTER(C.c_float), C.c_int, _vp, _vp]),
    "hf_plan_create": (C.c_int, [C.POINTER(HfDesc), C.POINTER(_vp), _vp]),
    "hf_plan_destroy": (C.c_int, [_vp]),
    "hf_plan_set_z": (C.c_int, [_vp, _f32, _vp]),
    "hf_plan_output_shape": (C.c_int, [_vp, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)]),
    "hf_plan_device_bytes": (C.c_int, [_vp, C.POINTER(_sz)]),
    "hf_plan_band_pass": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "hf_pipeline_exec": (C.c_int, [_vp, _vp, _i64, _i64, C.c_int, _vp, _vp]),
    "hf_pipeline_inspect": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "hf_plan_timing": (C.c_int, [_vp, C.c_int]),
    "hf_plan_status": (C.c_int, [_vp, C.POINTER(C.c_int), C.c_int]),
    "hf_stream_create": (C.c_int, [_vp, _i64, C.POINTER(_vp)]),
    "hf_stream_destroy": (C.c_int, [_vp]),
    "hf_stream_push": (C.c_int, [_vp, _vp, _i64, _vp]),
    "hf_stream_ready": (_i64, [_vp]),
    "hf_stream_process": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.POINTER(C.c_int), _vp]),
    "hf_stream_output_wait": (C.c_int, [_vp, _vp, C.c_int]),
    "hf_server_create": (C.c_int, [_sz, C.c_int, C.POINTER(_vp)]),
    "hf_server_destroy": (C.c_int, [_vp]),
    "hf_server_open": (C.c_int, [_vp, C.POINTER(HfDesc), _i64, C.POINTER(C.c_int)]),
    "hf_server_close": (C.c_int, [_vp, C.c_int]),
    "hf_server_push": (C.c_int, [_vp, C.c_int, _vp, _i64]),
    "hf_server_ready": (_i64, [_vp, C.c_int]),
    "hf_server_step": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(C.c_int)]),
    "hf_server_sync": (C.c_int, [_vp]),
    "hf_server_poll": (C.c_int, [_vp, _vp]),
    "hf_server_inflight": (C.c_int, [_vp, C.c_int]),
    "hf_server_reserve": (C.c_int, [_vp, _sz]),
    "hf_server_latencies": (C.c_int, [_vp, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "hf_server_open_count": (C.c_int, [_vp]),
    "hf_multi_create": (C.c_int, [C.c_int, C.POINTER(HfDesc), C.POINTER(_vp)]),
    "hf_multi_destroy": (C.c_int, [_vp]),
    "hf_multi_exec": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_i64), C.POINTER(_i64), C.POINTER(C.c_int),
                                C.POINTER(_vp), _vp]),
    "hf_multi_tune": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_i64), C.POINTER(_i64), C.POINTER(C.c_int),
                                C.POINTER(_vp), C.c_int, _vp, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "hf_multi_plan": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "hf_multi_get_schedule": (C.c_int, [_vp, C.POINTER(HfMultiSchedule)]),
    "hf_multi_set_schedule": (C.c_int, [_vp, C.POINTER(HfMultiSchedule)]),
    "hf_node_kinds": (C.c_int, [C.c_char_p, _sz]),
    "hf_node_infer": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(HfTDesc), C.POINTER(C.c_int),
                                C.POINTER(HfTDesc), C.c_int]),
    "hf_node_create": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(HfTDesc), _vp, C.POINTER(_vp)]),
    "hf_node_update": (C.c_int, [_vp, C.c_char_p, C.c_int, C.POINTER(HfTDesc), _vp]),
    "hf_node_execute": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.c_int)]),
    "hf_node_output_desc": (C.c_int, [_vp, C.c_int, C.POINTER(HfTDesc)]),
    "hf_node_destroy": (C.c_int, [_vp]),
    "hf_node_output_alias": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    "hf_node_is_async": (C.c_int, [_vp]),
    "hf_node_acquire_input": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "hf_node_try_push": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "hf_node_try_pop": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
    "hf_node_release_output": (C.c_int, [_vp, C.c_int]),
    "hf_fftshift": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.POINTER(_i64), C.c_uint32, _vp]),
    "hf_flatfield_create": (C.c_int, [_i64, C.c_int, C.c_int, C.c_float, C.c_float, _vp, C.POINTER(_vp)]),
    "hf_flatfield_is_fourier": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "hf_flatfield_exec": (C.c_int, [_vp, _vp, _vp, _vp]),
    "hf_flatfield_destroy": (C.c_int, [_vp]),
    "hf_filter2d_create": (C.c_int, [_i64, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.c_uint32, _vp, C.POINTER(_vp)]),
    "hf_filter2d_exec": (C.c_int, [_vp, _vp, _vp, _vp]),
    "hf_filter2d_destroy": (C.c_int, [_vp]),
    "hf_pctclip_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.POINTER(HfEllipse), _vp,
                                    C.POINTER(_vp)]),
    "hf_pctclip_roi_count": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "hf_pctclip_exec": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "hf_pctclip_destroy": (C.c_int, [_vp]),
    "hf_slideavg_create": (C.c_int, [_i64, C.c_int, C.c_int, _vp, C.POINTER(_vp)]),
    "hf_slideavg_push": (C.c_int, [_vp, _vp, _vp, C.POINTER(C.c_int), _vp]),
    "hf_slideavg_destroy": (C.c_int, [_vp]),
    "hf_node_output_ptr": (C.c_int, [_vp, C.c_int, C.POINTER(_vp), C.POINTER(C.c_int)]),
    "hf_holo_open": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "hf_holo_header_get": (C.c_int, [_vp, C.POINTER(HoloHeader)]),
    "hf_holo_footer": (C.c_int, [_vp, C.c_char_p, _sz, C.POINTER(_sz)]),
    "hf_holo_seek": (C.c_int, [_vp, _i64]),
    "hf_holo_tell": (C.c_int, [_vp, C.POINTER(_i64)]),
    "hf_holo_read": (C.c_int, [_vp, _vp, _i64]),
    "hf_holo_close": (C.c_int, [_vp]),
    "hf_holo_create": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint16, C.c_char_p,
                                 C.POINTER(_vp)]),
    "hf_holo_write": (C.c_int, [_vp, _vp, _i64]),
    "hf_holo_finish": (C.c_int, [_vp]),
    "hf_plan_autofocus_coefficients": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "hf_plan_autofocus_reset": (C.c_int, [_vp, _vp]),
    "hf_autofocus_set_accumulation": (C.c_int, [_vp, C.c_int, _vp]),
    "hf_autofocus_reset": (C.c_int, [_vp, _vp]),
    "hf_autofocus_set_slope_mode": (C.c_int, [_vp, C.c_int, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float,
                                              C.c_float, _vp]),
    "hf_plan_stage_times": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_char_p), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
    "hf_stfd_create": (C.c_int, [_i64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                 C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int, _vp,
                                 C.POINTER(_vp)]),
    "hf_stfd_grid": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hf_stfd_set_z": (C.c_int, [_vp, C.c_float, _vp]),
    "hf_stfd_exec": (C.c_int, [_vp, _vp, _vp, _vp]),
    "hf_stfd_destroy": (C.c_int, [_vp]),
    "hf_shslopes_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(HfEllipse), C.c_int, _vp,
                                     C.POINTER(_vp)]),
    "hf_shslopes_create_mode": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(HfEllipse), C.c_int,
                                          C.c_int, C.c_int, _vp, C.POINTER(_vp)]),
    "hf_shslopes_active": (C.c_int, [_vp, _vp]),
    "hf_shslopes_exec": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "hf_shslopes_destroy": (C.c_int, [_vp]),
    "hf_zernike_fit_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        C.c_float, C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(_vp)]),
    "hf_zernike_fit_pupil_radius": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "hf_zernike_fit_exec": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "hf_zernike_fit_host": (C.c_int, [_vp, _vp, _vp]),
    "hf_zernike_fit_destroy": (C.c_int, [_vp]),
    "hf_zernike_phase": (C.c_int, [_vp, C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, _vp, _vp, _vp]),
    "hf_correct_phase": (C.c_int, [_vp, C.c_int, _vp, _i64, C.c_int, C.c_int, _vp, _vp]),
    "hf_wrap2pi": (C.c_int, [_vp, _vp, _i64, _vp]),
    "hf_defocus_z": (C.c_int, [C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "hf_autofocus_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                      C.c_float, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_float, _vp,
                                      C.POINTER(_vp)]),
    "hf_autofocus_pupil_radius": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "hf_autofocus_exec": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "hf_autofocus_outputs": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "hf_autofocus_destroy": (C.c_int, [_vp]),
}

_lib = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load the shared library (raises if it is absent: there is no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"holoflow_b200: {p} not built (run __graft_entry__.build())")
    lib = C.CDLL(str(p))
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue  # symbol checks are done by the tests
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def lib() -> C.CDLL:
    return load()


def check(rc: int) -> None:
    if rc != HF_OK:
        raise HfError(rc, lib().hf_last_error().decode(errors="replace"))


def declared_symbols(header: os.PathLike | str | None = None) -> list[str]:
    """Every hf_* function declared in include/*.h (parsed from the header text)."""
    import re
    root = _HERE.parent / "include"
    names: list[str] = []
    files = [pathlib.Path(header)] if header else sorted(root.glob("*.h"))
    for h in files:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"\b(hf_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))
