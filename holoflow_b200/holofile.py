"""Python face of the .holo reader / writer (include/holoflow_b200.h, hf_holo_*).

The container is Holoflow's acquisition file (holofile/include/holofile/holofile.hh:87-152): a
64-byte header, the frames, and an optional JSON footer with the pipeline settings.  Besides the
reference's 8- and 16-bit pixels, ``bits_per_pixel = 12`` holds Mono12p frames (HF_MONO12P
layout), which feed the Doppler path's packed-input kernels directly.

    with holofile.Reader("run.holo") as r:
        frames = r.read(64)              # uint8 [64, frame_bytes]
    holofile.write("out.holo", frames_u16, bits_per_pixel=16, footer={"fs": 67000})
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Any, Optional

import numpy as np

from . import HoloHeader, check, lib

MAGIC_NUMBER_LE = 0x4F4C4F48  # "HOLO"
CURRENT_VERSION = 66


def frame_bytes(h: HoloHeader) -> int:
    return h.frame_width * h.frame_height * h.bits_per_pixel // 8


class Reader:
    """hf_holo_open / seek / read: a cursor over the frames of a .holo file."""

    def __init__(self, path: str):
        self._r = C.c_void_p()
        check(lib().hf_holo_open(str(path).encode(), C.byref(self._r)))
        self.header = HoloHeader()
        check(lib().hf_holo_header_get(self._r, C.byref(self.header)))

    @property
    def frame_bytes(self) -> int:
        return frame_bytes(self.header)

    def footer(self) -> Optional[dict[str, Any]]:
        """The footer's pipeline settings, or None when the file has no valid footer."""
        n = C.c_size_t()
        check(lib().hf_holo_footer(self._r, None, 0, C.byref(n)))
        if n.value == 0:
            return None
        buf = C.create_string_buffer(n.value + 1)
        check(lib().hf_holo_footer(self._r, buf, n.value + 1, C.byref(n)))
        return json.loads(buf.value.decode())

    def seek(self, frame_index: int) -> None:
        check(lib().hf_holo_seek(self._r, frame_index))

    def tell(self) -> int:
        i = C.c_int64()
        check(lib().hf_holo_tell(self._r, C.byref(i)))
        return i.value

    def read(self, count: int, out=None):
        """`count` frames at the cursor as uint8 [count, frame_bytes], or into `out`: a host
        numpy array or (pinned) CPU torch tensor of at least count * frame_bytes bytes."""
        if out is None:
            out = np.empty((count, self.frame_bytes), dtype=np.uint8)
        if isinstance(out, np.ndarray):
            assert out.flags.c_contiguous and out.nbytes >= count * self.frame_bytes
            ptr = out.ctypes.data
        else:
            assert not out.is_cuda and out.is_contiguous()
            assert out.numel() * out.element_size() >= count * self.frame_bytes
            ptr = out.data_ptr()
        check(lib().hf_holo_read(self._r, C.c_void_p(ptr), count))
        return out

    def close(self) -> None:
        if self._r:
            lib().hf_holo_close(self._r)
            self._r = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Writer:
    """hf_holo_create / write / finish: the header first, frames in order, the footer last."""

    def __init__(self, path: str, frame_count: int, width: int, height: int, bits_per_pixel: int,
                 footer: Optional[dict[str, Any]] = None):
        self._w = C.c_void_p()
        self.frame_bytes = width * height * bits_per_pixel // 8
        text = json.dumps(footer, separators=(",", ":")).encode() if footer is not None else None
        check(lib().hf_holo_create(str(path).encode(), frame_count, width, height, bits_per_pixel, text,
                                   C.byref(self._w)))

    def write(self, frames) -> None:
        """Frames as a C-contiguous numpy array (any dtype) whose bytes are whole frames."""
        a = np.ascontiguousarray(frames)
        assert a.nbytes % self.frame_bytes == 0
        check(lib().hf_holo_write(self._w, C.c_void_p(a.ctypes.data), a.nbytes // self.frame_bytes))

    def finish(self) -> None:
        if self._w:
            w, self._w = self._w, C.c_void_p()
            check(lib().hf_holo_finish(w))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.finish()


def write(path: str, frames: np.ndarray, bits_per_pixel: int, width: Optional[int] = None,
          height: Optional[int] = None, footer: Optional[dict[str, Any]] = None) -> None:
    """Writes a whole acquisition: frames [n, H, W] (uint8 / uint16), or packed 12-bit frames
    [n, 3 H W / 2] uint8 with width and height given."""
    n = frames.shape[0]
    if bits_per_pixel != 12:
        height, width = frames.shape[1], frames.shape[2]
    assert width is not None and height is not None
    with Writer(path, n, width, height, bits_per_pixel, footer) as w:
        w.write(frames)
