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
        An output the node owns (a cached "Holofile" source) or that views an input (a "Slice") is
        given as None; its pointer is then available from output_ptr() (see views())."""
        def addr(t):
            return int(t) if isinstance(t, int) else _ptr(t).value
        ins = (C.c_void_p * max(1, len(inputs)))(*[addr(t) for t in inputs])
        outs = (C.c_void_p * max(1, len(outputs)))(*[None if t is None else _ptr(t).value for t in outputs])
        r = C.c_int()
        check(lib().hf_node_execute(self._n, ins, outs, C.byref(r)))
        return r.value

    def alias(self, i: int) -> int:
        """The input that output i views (InferResult::in_place), or -1."""
        a = C.c_int()
        check(lib().hf_node_output_alias(self._n, i, C.byref(a)))
        return a.value

    def view(self, i: int, inputs: Sequence[torch.Tensor]) -> torch.Tensor:
        """Output i, an in-place view of one of `inputs`, as a torch view of that tensor."""
        a = self.alias(i)
        src = inputs[a]
        d = self.output_desc(i)
        es = _SIZE[d.dtype]
        p, _ = self.output_ptr(i)
        base = src.data_ptr() - src.storage_offset() * src.element_size()
        return torch.as_strided(src, shape_of(d), tuple(d.strides[k] // es for k in range(d.rank)),
                                (p - base) // es)

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


class _DevPtr:
    """A raw device pointer with a shape, exposed to torch through __cuda_array_interface__."""
    _TYPESTR = {0: "|u1", 1: "<i2", 2: "<f4", 3: "<c8"}

    def __init__(self, ptr: int, d: HfTDesc):
        es = _SIZE[d.dtype]
        self.__cuda_array_interface__ = {
            "shape": shape_of(d), "typestr": self._TYPESTR[d.dtype], "data": (ptr, False), "version": 3,
            "strides": tuple(d.strides[k] for k in range(d.rank)) if any(d.strides[k] for k in range(d.rank)) else None}
        self.es = es


def _wrap(ptr: int, d: HfTDesc) -> torch.Tensor:
    if d.mem_loc == 1:
        return torch.as_tensor(_DevPtr(ptr, d), device="cuda")
    n = 1
    for k in range(d.rank):
        n *= d.shape[k]
    buf = (C.c_char * (n * _SIZE[d.dtype])).from_address(ptr)
    return torch.frombuffer(buf, dtype=_TORCH[d.dtype]).reshape(shape_of(d))


class AsyncNode(Node):
    """An asynchronous kind (a queue): the producer writes the view acquire_input() returns and
    calls try_push(); the consumer's try_pop() makes the owned outputs readable (output()) until
    release_output()."""

    def acquire_input(self, i: int = 0, desc: Optional[HfTDesc] = None) -> Optional[torch.Tensor]:
        p = C.c_void_p()
        check(lib().hf_node_acquire_input(self._n, i, C.byref(p)))
        if not p.value:
            return None
        return _wrap(p.value, desc if desc is not None else self.input_descs[i])

    def try_push(self) -> int:
        r = C.c_int()
        check(lib().hf_node_try_push(self._n, C.byref(r)))
        return r.value

    def try_pop(self, outputs: Sequence[Optional[torch.Tensor]] = ()) -> int:
        outs = (C.c_void_p * 8)(*[None if t is None else _ptr(t).value for t in outputs])
        r = C.c_int()
        check(lib().hf_node_try_pop(self._n, outs, C.byref(r)))
        return r.value

    def output(self, i: int = 0) -> torch.Tensor:
        p, _ = self.output_ptr(i)
        return _wrap(p, self.output_desc(i))

    def release_output(self, i: int = 0) -> None:
        check(lib().hf_node_release_output(self._n, i))


def async_node(kind: str, settings: dict[str, Any], descs: Sequence[HfTDesc], stream=None) -> AsyncNode:
    n = AsyncNode(kind, settings, descs, stream)
    n.input_descs = list(descs)
    return n


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
            dev = (inputs[0].device if inputs else "cuda") if d.mem_loc == 1 else "cpu"
            outs.append(None if node.alias(i) >= 0 else empty_like_desc(d, dev))
        r = node.execute(inputs, outs)
        if r != 0:
            raise HfError(r, f"{kind}: execute returned OpResult {r}")
        torch.cuda.synchronize()
        return [node.view(i, inputs) if o is None else o for i, o in enumerate(outs)]
    finally:
        node.close()
