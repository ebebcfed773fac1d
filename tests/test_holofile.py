"""The .holo container and the "Holofile" source node, without a GPU.

The header layout, validation order, footer rules and exception messages are restated from
holofile/include/holofile/holofile.hh:87-104 and holofile/src/holofile.cc:42-268; the node's
settings keys, inference checks and messages, load kinds, wrap-around and update() reuse rules
from holotask/src/sources/holofile.cc:190-434.  Files built byte by byte here with `struct`
pin the layout independently of the library's own writer."""
import ctypes as C
import json
import struct
import time

import numpy as np
import pytest
import torch

import holoflow_b200 as hf
from holoflow_b200 import holofile as H
from holoflow_b200 import nodes as N
from oracle.oracle import pack12

MAGIC = 0x4F4C4F48


def header_bytes(count, w, h, bpp, data_size=None, magic=MAGIC, version=66):
    """The reference's 64-byte header: u32 magic, u16 version, u16 bits_per_pixel, u32 width,
    u32 height, u32 frame_count, u64 data_size_in_bytes, u8 endianness, 35 padding bytes."""
    if data_size is None:
        data_size = count * w * h * bpp // 8
    return struct.pack("<IHHIIIQB35x", magic, version, bpp, w, h, count, data_size, 0)


def make_file(path, frames_bytes, count, w, h, bpp, footer=b""):
    path.write_bytes(header_bytes(count, w, h, bpp) + frames_bytes + footer)
    return str(path)


def expect_error(fn, code, text):
    with pytest.raises(hf.HfError) as e:
        fn()
    assert e.value.code == code and text in str(e.value), str(e.value)


def test_header_struct_is_64_packed_bytes():
    assert C.sizeof(hf.HoloHeader) == 64
    assert hf.HoloHeader.data_size_in_bytes.offset == 20
    assert hf.HoloHeader.endianness.offset == 28


@pytest.mark.parametrize("bpp,w,h", [(8, 6, 4), (16, 5, 3), (12, 8, 2)])
def test_writer_output_matches_reference_layout(tmp_path, bpp, w, h):
    rng = np.random.default_rng(bpp)
    n = 7
    fb = w * h * bpp // 8
    frames = rng.integers(0, 256, size=(n, fb), dtype=np.uint8)
    footer = {"fs": 67000, "time_window": {"size": 64, "stride": 16}}
    p = tmp_path / "a.holo"
    with H.Writer(str(p), n, w, h, bpp, footer) as wr:
        wr.write(frames[:3])
        wr.write(frames[3:])
    raw = p.read_bytes()
    assert raw[:64] == header_bytes(n, w, h, bpp)
    assert raw[64:64 + n * fb] == frames.tobytes()
    assert json.loads(raw[64 + n * fb:]) == footer
    with H.Reader(str(p)) as r:
        assert (r.header.magic_number, r.header.version, r.header.bits_per_pixel) == (MAGIC, 66, bpp)
        assert (r.header.frame_width, r.header.frame_height, r.header.frame_count) == (w, h, n)
        assert r.header.data_size_in_bytes == n * fb and r.frame_bytes == fb
        assert r.footer() == footer
        assert np.array_equal(r.read(n), frames)
        assert r.tell() == n
        r.seek(2)
        assert r.tell() == 2
        assert np.array_equal(r.read(3), frames[2:5])


def test_twelve_bit_file_round_trips_packed_frames(tmp_path):
    """A 12-bit .holo holds Mono12p frames: the bytes the path's packed-input kernels read."""
    rng = np.random.default_rng(5)
    w, h, n = 16, 4, 3
    px = rng.integers(0, 4096, size=(n, h * w)).astype(np.uint16)
    packed = np.stack([pack12(f) for f in px])
    assert packed.shape == (n, 3 * w * h // 2)
    p = str(tmp_path / "m.holo")
    H.write(p, packed, 12, width=w, height=h)
    with H.Reader(p) as r:
        assert r.header.bits_per_pixel == 12 and r.frame_bytes == 96
        assert np.array_equal(r.read(n), packed)
        assert r.footer() == {}


def test_reader_without_footer_and_with_invalid_footers(tmp_path):
    fr = bytes(range(24))
    for name, footer in [("none", b""), ("notjson", b"xyz"), ("badjson", b"{oops"),
                         ("huge", b"{" + b" " * (1024 * 1024) + b"}")]:
        p = make_file(tmp_path / f"{name}.holo", fr, 2, 4, 3, 8, footer)
        with H.Reader(p) as r:
            assert r.footer() is None, name
            assert r.tell() == 0
            assert r.read(2).tobytes() == fr  # positioned at the first frame after the footer probe
    p = make_file(tmp_path / "ok.holo", fr, 2, 4, 3, 8, b'{"a": [1, 2]}')
    with H.Reader(p) as r:
        assert r.footer() == {"a": [1, 2]}
        assert r.read(1).tobytes() == fr[:12]


def test_reader_errors_match_reference_exceptions(tmp_path):
    short = tmp_path / "short.holo"
    short.write_bytes(header_bytes(1, 2, 2, 8)[:40])
    expect_error(lambda: H.Reader(str(short)), hf.HF_ERR_INVALID, "Holofile: Incomplete header")
    bad = tmp_path / "magic.holo"
    bad.write_bytes(header_bytes(1, 2, 2, 8, magic=0x12345678) + bytes(4))
    expect_error(lambda: H.Reader(str(bad)), hf.HF_ERR_INVALID, "Holofile: Invalid magic number")
    odd = tmp_path / "odd.holo"
    odd.write_bytes(header_bytes(1, 3, 1, 12, data_size=4) + bytes(5))  # 36 bits per frame
    expect_error(lambda: H.Reader(str(odd)), hf.HF_ERR_INVALID, "Holofile: Invalid frame size")
    expect_error(lambda: H.Reader(str(tmp_path / "absent.holo")), hf.HF_ERR_STATE, "Failed to open")
    p = make_file(tmp_path / "eof.holo", bytes(8), 2, 2, 2, 8)
    with H.Reader(p) as r:
        r.read(1)
        expect_error(lambda: r.read(2), hf.HF_ERR_STATE, "Holofile: End of file reached")
        assert r.tell() == 2  # the frame that was there was read
    # the version field is not checked (the reference leaves version support open)
    p = tmp_path / "v.holo"
    p.write_bytes(header_bytes(1, 2, 2, 8, version=7) + bytes(4))
    with H.Reader(str(p)) as r:
        assert r.header.version == 7


def test_writer_rejects_bad_geometry(tmp_path):
    w = C.c_void_p()
    rc = hf.lib().hf_holo_create(str(tmp_path / "x.holo").encode(), 1, 3, 1, 12, None, C.byref(w))
    assert rc == hf.HF_ERR_INVALID
    rc = hf.lib().hf_holo_create(str(tmp_path / "x.holo").encode(), 1, 4, 4, 10, None, C.byref(w))
    assert rc == hf.HF_ERR_INVALID


# ---- the "Holofile" source node ----------------------------------------------------------------
def settings(path, kind="Live", start=0, end=10, batch=2, **kw):
    s = {"path": path, "load_kind": kind, "start_frame": start, "end_frame": end, "batch_size": batch}
    s.update(kw)
    return s


@pytest.fixture
def u16_file(tmp_path):
    rng = np.random.default_rng(3)
    frames = rng.integers(0, 65536, size=(10, 3, 4), dtype=np.uint16)
    p = str(tmp_path / "u16.holo")
    H.write(p, frames, 16, footer={"camera": "synthetic"})
    return p, frames


def test_node_infer_descriptors_and_messages(u16_file, tmp_path):
    p, _ = u16_file
    assert "Holofile" in N.kinds()
    (o,) = N.infer("Holofile", settings(p, batch=4), [])
    assert N.shape_of(o) == (4, 3, 4) and o.dtype == 1 and o.mem_loc == 0
    (o,) = N.infer("Holofile", settings(p, kind="GPUCached"), [])
    assert o.mem_loc == 1
    packed = str(tmp_path / "p.holo")
    H.write(packed, np.zeros((4, 3 * 8 * 2 // 2), np.uint8), 12, width=8, height=2)
    (o,) = N.infer("Holofile", settings(packed, end=4), [])
    assert N.shape_of(o) == (2, 2, 12) and o.dtype == 0
    cases = [
        (settings(p, start=5, end=5), "Invalid frame range"),
        (settings(p, batch=0), "Batch size must be positive"),
        (settings(p, max_fps=0), "max_fps must be positive when provided"),
        (settings(p, end=11), "end_frame exceeds total frames in file"),
        (settings(p, start=8, batch=3), "Batch size exceeds available frames"),
    ]
    for s, msg in cases:
        expect_error(lambda: N.infer("Holofile", s, []), hf.HF_ERR_INVALID, "HolofileFactory inference error: " + msg)
    d = hf.HfTDesc()
    d.rank, d.dtype, d.mem_loc, d.shape[0] = 1, 0, 1, 4
    expect_error(lambda: N.infer("Holofile", settings(p), [d]), hf.HF_ERR_INVALID,
                 "HolofileFactory inference error: Holofile task must have no inputs")
    expect_error(lambda: N.infer("Holofile", settings(p, kind="Disk"), []), hf.HF_ERR_INVALID,
                 "Invalid LoadKind string: Disk")


def test_node_live_reads_batches_and_wraps(u16_file):
    p, frames = u16_file
    node = N.Node("Holofile", settings(p, start=1, end=8, batch=3), [])
    out = torch.empty((3, 3, 4), dtype=torch.int16)
    got = []
    for _ in range(5):
        assert node.execute([], [out]) == 0
        got.append(out.numpy().view(np.uint16).copy())
    # frames 1-3, 4-6, then 7-9 would pass end_frame = 8: back to start_frame
    idx = [[1, 2, 3], [4, 5, 6], [1, 2, 3], [4, 5, 6], [1, 2, 3]]
    for g, i in zip(got, idx):
        assert np.array_equal(g, frames[i])


def host_view(ptr, shape, dtype):
    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    return np.frombuffer((C.c_ubyte * n).from_address(ptr), dtype=dtype).reshape(shape)


def test_node_cpu_cached_publishes_views_into_the_cache(u16_file):
    p, frames = u16_file
    node = N.Node("Holofile", settings(p, kind="CPUCached", start=2, end=9, batch=2), [])
    seen = []
    for _ in range(4):
        assert node.execute([], [None]) == 0
        ptr, owned = node.output_ptr(0)
        assert owned and ptr
        seen.append(host_view(ptr, (2, 3, 4), np.uint16).copy())
    for g, i in zip(seen, [[2, 3], [4, 5], [6, 7], [2, 3]]):
        assert np.array_equal(g, frames[i])
    with pytest.raises(hf.HfError):  # a Live node needs the caller's output buffer
        N.Node("Holofile", settings(p), []).execute([], [None])


def test_node_update_keeps_or_resets_the_cursor(u16_file):
    p, frames = u16_file
    out = torch.empty((2, 3, 4), dtype=torch.int16)
    node = N.Node("Holofile", settings(p, batch=2), [])
    node.execute([], [out])
    node.execute([], [out])  # cursor at frame 4
    node.update(settings(p, batch=2), [])
    node.execute([], [out])
    assert np.array_equal(out.numpy().view(np.uint16), frames[[4, 5]])
    node.update(settings(p, batch=2, keep_cursor=False), [])
    node.execute([], [out])
    assert np.array_equal(out.numpy().view(np.uint16), frames[[0, 1]])
    # bounds that exclude the cursor start over at the new start_frame
    node.update(settings(p, start=6, end=10, batch=2), [])
    node.execute([], [out])
    assert np.array_equal(out.numpy().view(np.uint16), frames[[6, 7]])


def test_node_max_fps_paces_batches(u16_file):
    p, _ = u16_file
    node = N.Node("Holofile", settings(p, batch=2, max_fps=400), [])  # one batch per 5 ms
    out = torch.empty((2, 3, 4), dtype=torch.int16)
    t0 = time.perf_counter()
    for _ in range(9):
        node.execute([], [out])
    assert time.perf_counter() - t0 >= 8 * 0.005 * 0.9
