"""Many acquisitions of uneven size in one CUDA graph launch (hf_multi_*), with the schedule
autotuner: branches and assignment, and the fused segment band pass (one persistent launch per
window length and format) with its tiles per segment and grid cap."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import torch

from . import HfDesc, HfMultiSchedule, check, lib
from .pipeline import PipelineConfig, _stream


class Multi:
    def __init__(self, cfgs: Sequence[PipelineConfig]):
        self.cfgs = list(cfgs)
        n = len(self.cfgs)
        descs = (HfDesc * n)(*[c.desc() for c in self.cfgs])
        self._m = C.c_void_p()
        check(lib().hf_multi_create(n, descs, C.byref(self._m)))

    def _args(self, rings, ring_frames, first, nwin, outs):
        n = len(self.cfgs)
        r = (C.c_void_p * n)(*[t.data_ptr() for t in rings])
        rf = (C.c_int64 * n)(*ring_frames)
        f = (C.c_int64 * n)(*first)
        nw = (C.c_int * n)(*nwin) if nwin is not None else None
        o = (C.c_void_p * n)(*[t.data_ptr() for t in outs])
        return r, rf, f, nw, o

    def exec(self, rings: Sequence[torch.Tensor], ring_frames: Sequence[int], first: Sequence[int],
             outs: Sequence[torch.Tensor], nwin: Optional[Sequence[int]] = None, stream=None) -> None:
        r, rf, f, nw, o = self._args(rings, ring_frames, first, nwin, outs)
        check(lib().hf_multi_exec(self._m, r, rf, f, nw, o, _stream(stream)))

    def tune(self, rings, ring_frames, first, outs, nwin=None, reps: int = 3, stream=None) -> tuple[int, float]:
        r, rf, f, nw, o = self._args(rings, ring_frames, first, nwin, outs)
        bs, bm = C.c_int(), C.c_float()
        check(lib().hf_multi_tune(self._m, r, rf, f, nw, o, reps, _stream(stream), C.byref(bs), C.byref(bm)))
        return bs.value, bm.value

    def schedule(self) -> dict:
        sch = HfMultiSchedule()
        check(lib().hf_multi_get_schedule(self._m, C.byref(sch)))
        return {f: getattr(sch, f) for f, _ in HfMultiSchedule._fields_}

    def set_schedule(self, branches: int = 1, largest_first: int = 1, fused: int = 0, seg_tiles: int = 0,
                     band_ctas: int = 0) -> None:
        sch = HfMultiSchedule(branches, largest_first, fused, seg_tiles, band_ctas)
        check(lib().hf_multi_set_schedule(self._m, C.byref(sch)))

    def close(self) -> None:
        if self._m:
            lib().hf_multi_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
