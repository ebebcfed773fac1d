"""Streaming server over the C ABI (hf_server_*): concurrent camera streams with continuous
batching, admission by free device memory, and per-window frame-to-image latencies."""
from __future__ import annotations

import ctypes as C
from typing import Mapping, Optional

import torch

from . import HfError, HF_ERR_NOMEM, check, lib
from .pipeline import PipelineConfig, _ptr


class Server:
    def __init__(self, max_streams: int = 32, hbm_reserve_bytes: int = 0):
        self._s = C.c_void_p()
        self.max_streams = max_streams
        check(lib().hf_server_create(hbm_reserve_bytes, max_streams, C.byref(self._s)))
        self.cfgs: dict[int, PipelineConfig] = {}

    def open(self, cfg: PipelineConfig, ring_frames: int) -> Optional[int]:
        """Admits a stream; None when the device (or the slot table) has no room for it now."""
        sid = C.c_int(-1)
        d = cfg.desc()
        rc = lib().hf_server_open(self._s, C.byref(d), ring_frames, C.byref(sid))
        if rc == HF_ERR_NOMEM:
            return None
        check(rc)
        self.cfgs[sid.value] = cfg
        return sid.value

    def close(self, sid: int) -> None:
        check(lib().hf_server_close(self._s, sid))
        self.cfgs.pop(sid, None)

    def push(self, sid: int, frames: torch.Tensor, nframes: int) -> None:
        check(lib().hf_server_push(self._s, sid, _ptr(frames), nframes))

    def ready(self, sid: int) -> int:
        return lib().hf_server_ready(self._s, sid)

    def step(self, outs: Mapping[int, torch.Tensor]) -> dict[int, int]:
        """One scheduling round; outs[sid] = pinned host [max_batch, n_moments, OH, OW]."""
        arr = (C.c_void_p * self.max_streams)()
        for sid, t in outs.items():
            arr[sid] = t.data_ptr()
        done = (C.c_int * self.max_streams)()
        check(lib().hf_server_step(self._s, arr, done))
        return {i: done[i] for i in range(self.max_streams) if done[i] > 0}

    def sync(self) -> None:
        """Waits for the server's own streams, then collects (latencies, delivered windows)."""
        check(lib().hf_server_sync(self._s))

    def poll(self) -> dict[int, int]:
        """Collects the batches whose images have reached the host, without waiting for the others;
        returns {stream: cumulative windows delivered} for the open streams."""
        done = (C.c_int64 * self.max_streams)()
        check(lib().hf_server_poll(self._s, done))
        return {sid: done[sid] for sid in self.cfgs}

    def inflight(self, sid: int) -> int:
        """Batches of stream `sid` still on the device."""
        return lib().hf_server_inflight(self._s, sid)

    def reserve(self, nbytes: int) -> None:
        """Grows the server's memory pool once, so later streams open without device allocations."""
        check(lib().hf_server_reserve(self._s, nbytes))

    def latencies(self) -> list[float]:
        buf = (C.c_float * 65536)()
        n = C.c_int()
        check(lib().hf_server_latencies(self._s, buf, 65536, C.byref(n)))
        return list(buf[: n.value])

    def open_count(self) -> int:
        return lib().hf_server_open_count(self._s)

    def close_all(self) -> None:
        if self._s:
            lib().hf_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close_all()
        except Exception:
            pass
