"""Compute nodes by kind string through the C ABI's hf_node_* functions.

Mirrors how Holoflow drives a sync task: `infer` (descriptors only), `create` (allocations on a
stream), `update` (reuse where the factory can), `execute` on device tensors.  `run_sync_factory`
is the full path used by the reference's tests (sync_task_runner.cc:84-96).
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Any, Optional, Sequence

import torch

from . import HfError, HfTDesc, check, lib
from .pipeline import _ptr, _stream as _cuda_stream


def _stream(stream=None) -> C.c_void_p:
    """The stream handle for create/update: torch's current stream, or the null handle where no
    CUDA device exists (host-only nodes such as a Live or CPUCached "Holofile" source need no
    stream; a compute node given it fails inside the library with HF_ERR_CUDA)."""
    if stream is None and not torch.cuda.is_available():
        return C.c_void_p(0)
    return _cuda_stream(stream)

_DT = {torch.uint8: 0, torch.int16: 1, torch.float32: 2, torch.complex64: 3}
_TORCH = {0: torch.uint8, 1: torch.int16, 2: torch.float32, 3: torch.complex64}  # U16 carried as int16
_SIZE = {0: 1, 1: 2, 2: 4, 3: 8}


def desc_of(t: torch.Tensor, dtype: Optional[int] = None) -> HfTDesc:
    """Descriptor of a tensor (U16 data travels in int16 tensors: pass dtype=1)."""
    d = HfTDesc()
    d.rank = t.dim()
    d.dtype = _DT[t.dtype] if dtype is None else dtype
    d.mem_loc = 1 if t.is_cuda else 0
    es = _SIZE[d.dtype]
    for i, (n, st) in enumerate(zip(t.shape, t.stride())):
        d.shape[i] = n
        d.strides[i] = st * es
    return d


def shape_of(d: HfTDesc) -> tuple[int, ...]:
    return tuple(d.shape[i] for i in range(d.rank))


def _arr(descs: Sequence[HfTDesc]):
    a = (HfTDesc * max(1, len(descs)))()
    for i, d in enumerate(descs):
        a[i] = d
    return a


def kinds() -> list[str]:
    b = C.create_string_buffer(4096)
    check(lib().hf_node_kinds(b, 4096))
    return b.value.decode().split(",")


def infer(kind: str, settings: dict[str, Any], descs: Sequence[HfTDesc]) -> list[HfTDesc]:
    out = (HfTDesc * 8)()
    n = C.c_int()
    check(lib().hf_node_infer(kind.encode(), json.dumps(settings).encode(), len(descs), _arr(descs), C.byref(n),
                              out, 8))
    return [out[i] for i in range(n.value)]


class Node:
    def __init__(self, kind: str, settings: dict[str, Any], descs: Sequence[HfTDesc], stream=None):
        self._n = C.c_void_p()
        check(lib().hf_node_create(kind.encode(), json.dumps(settings).encode(), len(descs), _arr(descs),
                                   _stream(stream), C.byref(self._n)))
        self.kind = kind

    def update(self, settings: dict[str, Any], descs: Sequence[HfTDesc], stream=None) -> None:
        check(lib().hf_node_update(self._n, json.dumps(settings).encode(), len(descs), _arr(descs), _stream(stream)))

    def output_desc(self, i: int = 0) -> HfTDesc:
        d = HfTDesc()
        check(lib().hf_node_output_desc(self._n, i, C.byref(d)))
        return d

    def execute(self, inputs: Sequence[Any], outputs: Sequence[Optional[torch.Tensor]]) -> int:
        """Inputs are tensors or raw origin pointers (ints, e.g. another node's output_ptr()).
        An output the node owns (a cached "Holofile" source) is given as None; its pointer is then
        available from output_ptr()."""
        def addr(t):
            return int(t) if isinstance(t, int) else _ptr(t).value
        ins = (C.c_void_p * max(1, len(inputs)))(*[addr(t) for t in inputs])
        outs = (C.c_void_p * max(1, len(outputs)))(*[None if t is None else _ptr(t).value for t in outputs])
        r = C.c_int()
        check(lib().hf_node_execute(self._n, ins, outs, C.byref(r)))
        return r.value

    def output_ptr(self, i: int = 0) -> tuple[int, bool]:
        """(origin pointer of output i as of the last execute, whether the node owns it)."""
        p, owned = C.c_void_p(), C.c_int()
        check(lib().hf_node_output_ptr(self._n, i, C.byref(p), C.byref(owned)))
        return (p.value or 0), bool(owned.value)

    def close(self) -> None:
        if self._n:
            lib().hf_node_destroy(self._n)
            self._n = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def empty_like_desc(d: HfTDesc, device) -> torch.Tensor:
    return torch.empty(shape_of(d), dtype=_TORCH[d.dtype], device=device)


def run_sync_factory(kind: str, settings: dict[str, Any], inputs: Sequence[torch.Tensor],
                     dtypes: Optional[Sequence[Optional[int]]] = None) -> list[torch.Tensor]:
    """infer -> create -> execute -> synchronize; returns the outputs."""
    descs = [desc_of(t, None if dtypes is None else dtypes[i]) for i, t in enumerate(inputs)]
    node = Node(kind, settings, descs)
    try:
        n_out = len(infer(kind, settings, descs))
        outs = []
        for i in range(n_out):
            d = node.output_desc(i)
            outs.append(empty_like_desc(d, inputs[0].device if d.mem_loc == 1 else "cpu"))
        r = node.execute(inputs, outs)
        if r != 0:
            raise HfError(r, f"{kind}: execute returned OpResult {r}")
        torch.cuda.synchronize()
        return outs
    finally:
        node.close()
