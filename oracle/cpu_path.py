"""ctypes binding of oracle/cpu_path.cc, the FP32 C++/OpenMP restatement of the per-window path
(TEST AND BASELINE INFRASTRUCTURE ONLY: the CPU baseline and the reference arm of bench.py; the
library never uses it).  ``build()`` compiles it with g++ into oracle/_build/libhfcpu.so."""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
SRC = HERE / "cpu_path.cc"
LIB = HERE / "_build" / "libhfcpu.so"
# x86-64-v3 (AVX2 + FMA) rather than -march=native: the library is built here and run on the GPU
# box's host, whose CPU may differ.  No fast-math: float32 arithmetic stays IEEE and uncontracted.
FLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c++17"]


class _Cfg(C.Structure):
    _fields_ = [("H", C.c_int32), ("W", C.c_int32), ("T", C.c_int32), ("z0", C.c_int32), ("z1", C.c_int32),
                ("clutter_rank", C.c_int32), ("propagation", C.c_int32), ("fmt", C.c_int32),
                ("lam", C.c_float), ("pitch", C.c_float), ("z", C.c_float), ("fs", C.c_float)]


def build(force: bool = False) -> pathlib.Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        LIB.parent.mkdir(exist_ok=True)
        subprocess.run(["g++", *FLAGS, str(SRC), "-o", str(LIB)], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        _lib.hfc_window.argtypes = [C.POINTER(_Cfg), C.c_void_p, C.c_void_p, C.c_int]
        _lib.hfc_window.restype = C.c_int
    return _lib


PROP = {"none": 0, "fresnel": 1, "angular_spectrum": 2}


def window(frames: np.ndarray, cfg, packed: bool = True, threads: int = 0) -> np.ndarray:
    """One window -> float32 [3, H, W] (M0, M1, M2).  ``frames``: T Mono12p frames as bytes
    (packed=True, [T, 3P/2] uint8) or uint16 values [T, H, W]; ``cfg``: an oracle.PathConfig
    (one-sided band, no padding / filter / fftshift / autofocus)."""
    if cfg.time_method != "rfft" or cfg.as_padding or cfg.as_filter or cfg.fftshift or cfg.filter2d or cfg.autofocus:
        raise ValueError("the CPU restatement covers the plain one-sided path only")
    c = _Cfg(cfg.height, cfg.width, cfg.frames, cfg.z0, cfg.z1, cfg.clutter_rank, PROP[cfg.propagation],
             16 if packed else 1, cfg.lam, cfg.pitch, cfg.z, cfg.fs)
    src = np.ascontiguousarray(frames)
    out = np.empty((3, cfg.height, cfg.width), dtype=np.float32)
    rc = lib().hfc_window(C.byref(c), src.ctypes.data, out.ctypes.data, int(threads))
    if rc != 0:
        raise ValueError("hfc_window: unsupported configuration")
    return out


def threads() -> int:
    """OpenMP threads a call with threads=0 uses (all host threads unless OMP_NUM_THREADS says)."""
    return int(lib().hfc_threads())
