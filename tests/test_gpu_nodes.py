"""The path's compute nodes driven like the reference drives its sync tasks (infer -> create ->
execute, sync_task_runner.cc:84-96), through hf_node_*, checked against the oracle and the golden
vectors of the reference's NumPy oracle."""
import json
import math
import pathlib

import numpy as np
import pytest

from oracle import oracle as O
from oracle import synth as S

pytestmark = pytest.mark.gpu

LAM, DX = 852e-9, 12e-6
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "holonp_ops.npz"


def _n():
    from holoflow_b200 import nodes as N
    return N


def rel(a, b):
    return O.rel_l2(np.asarray(a), np.asarray(b))


def _gold(name):
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["__index__"]).decode())[name]
    ins = [z[f"{name}__in{i}"] for i in range(meta["ninputs"])]
    return meta["settings"], ins, z[f"{name}__out0"]


def test_fresnel_node_and_z_update(cuda, rng):
    import torch
    N = _n()
    x = (rng.standard_normal((3, 64, 128)) + 1j * rng.standard_normal((3, 64, 128))).astype(np.complex64)
    dev = torch.from_numpy(x).to(cuda)
    s = {"lambda": LAM, "dx": DX, "dy": DX, "z": 0.05, "skip_phase_shift": False}
    (got,) = N.run_sync_factory("FresnelDiffraction", s, [dev])
    exp = O.fresnel(x, LAM, DX, DX, 0.05, output_magnitude=False, skip_phase_shift=False)
    assert rel(got.cpu().numpy(), exp) < 2e-6 * math.log2(64 * 128)
    (mag,) = N.run_sync_factory("FresnelDiffraction", {**s, "output_magnitude": True}, [dev])
    assert rel(mag.cpu().numpy(), np.abs(exp)) < 2e-6 * math.log2(64 * 128)
    # update with only z changed reuses the task and equals a fresh task at the new z
    node = N.Node("FresnelDiffraction", s, [N.desc_of(dev)])
    node.update({**s, "z": 0.07}, [N.desc_of(dev)])
    out = torch.empty_like(dev)
    assert node.execute([dev], [out]) == 0
    (fresh,) = N.run_sync_factory("FresnelDiffraction", {**s, "z": 0.07}, [dev])
    assert torch.equal(out, fresh)
    node.close()


@pytest.mark.parametrize("shape,axes", [((64, 128, 3), [0, 1]), ((2, 64, 3, 128), [1, 3]), ((3, 64, 128), [-2, -1])])
def test_fresnel_node_over_any_two_axes(cuda, rng, shape, axes):
    """Axes other than the last two (fresnel_diffraction.cu:118-200, 519-570): the planes spanned by
    (axes[0], axes[1]) at every index of the other dimensions, one batch group per launch plus a
    launch per remaining index; equal to the last-two-axes transform of the permuted tensor."""
    import torch
    N = _n()
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    dev = torch.from_numpy(x).to(cuda)
    s = {"lambda": LAM, "dx": DX, "dy": DX, "z": 0.05, "axes": axes}
    (got,) = N.run_sync_factory("FresnelDiffraction", s, [dev])
    (mag,) = N.run_sync_factory("FresnelDiffraction", {**s, "output_magnitude": True}, [dev])
    a0, a1 = (a % len(shape) for a in axes)
    perm = [d for d in range(len(shape)) if d not in (a0, a1)] + [a0, a1]
    xp = np.ascontiguousarray(x.transpose(perm))
    exp = O.fresnel(xp, LAM, DX, DX, 0.05, output_magnitude=False, skip_phase_shift=False)
    inv = np.argsort(perm)
    tol = 2e-6 * math.log2(shape[a0] * shape[a1])
    assert rel(got.cpu().numpy(), exp.transpose(inv)) < tol
    assert rel(mag.cpu().numpy(), np.abs(exp).transpose(inv)) < tol


def test_angular_spectrum_node_kats(cuda, rng):
    """angular_spectrum_test.cu:146-283: z = 0 scales a real input by H*W and centres it in the
    padding; with a filter the result matches the oracle."""
    import torch
    N = _n()
    x = rng.standard_normal((2, 32, 48)).astype(np.float32)
    s = {"lambda": LAM, "dx": DX, "dy": DX, "z": 0.0, "padding": {"width": 64, "height": 40}}
    (got,) = N.run_sync_factory("AngularSpectrum", s, [torch.from_numpy(x).to(cuda)])
    got = got.cpu().numpy()
    exp = np.zeros((2, 40, 64), np.complex64)
    exp[:, 4:36, 8:56] = x * (40 * 64)
    assert np.abs(got - exp).max() <= 1e-3 * np.abs(exp).max()
    xc = (rng.standard_normal((2, 64, 64)) + 1j * rng.standard_normal((2, 64, 64))).astype(np.complex64)
    filt = {"r_inner": 4, "r_outer": 20, "s_inner": 2, "s_outer": 3}
    s2 = {"lambda": LAM, "dx": DX, "dy": DX, "z": 0.2, "filter": filt}
    (got,) = N.run_sync_factory("AngularSpectrum", s2, [torch.from_numpy(xc).to(cuda)])
    exp = O.angular_spectrum(xc, LAM, DX, DX, 0.2, filt=filt)
    assert rel(got.cpu().numpy(), exp) < 1e-5


def test_pca_node_matches_oracle(cuda, rng):
    import torch
    N = _n()
    x = rng.standard_normal((2, 12, 16, 16)).astype(np.float32)
    x[:, 3] += 5 * x[:, 0]  # a dominant direction
    (got,) = N.run_sync_factory("Pca", {"begin": 8, "end": 12}, [torch.from_numpy(x).to(cuda)])
    exp = O.pca(x, 8, 12)
    got = got.cpu().numpy()
    assert got.shape == (2, 4, 16, 16)
    # eigenvector signs are arbitrary: compare each component up to sign
    for b in range(2):
        for c in range(4):
            g, e = got[b, c].ravel(), exp[b, c].ravel()
            sgn = 1.0 if np.dot(g, e) >= 0 else -1.0
            assert rel(sgn * g, e) < 1e-4, (b, c)


@pytest.mark.parametrize("kind,name,dtype", [("FFT", "fft_f32_axis1_ortho", None), ("FFT", "fft_u16_axis1", 1),
                                             ("FFT", "fft_cf32_axis1", None), ("RFFT", "rfft_f32_axis1_t64", None)])
def test_fft_nodes_match_golden(cuda, kind, name, dtype):
    import torch
    N = _n()
    st, (x,), y = _gold(name)
    dev = torch.from_numpy(x.view(np.int16) if x.dtype == np.uint16 else x).to(cuda)
    (got,) = N.run_sync_factory(kind, st, [dev], dtypes=[dtype])
    assert got.shape == y.shape
    assert rel(got.cpu().numpy(), y) < 2e-6


@pytest.mark.parametrize("kind,name", [("Mean", "mean_f32_axis_m3"), ("Mean", "mean_cf32_axis_m3"),
                                       ("Mean", "mean_f32_axis0")])
def test_mean_nodes_match_golden(cuda, kind, name):
    import torch
    N = _n()
    st, (x,), y = _gold(name)
    (got,) = N.run_sync_factory(kind, st, [torch.from_numpy(x).to(cuda)])
    assert tuple(got.shape) == y.shape
    assert rel(got.cpu().numpy(), y) < 1e-6


def test_mean_abs_node(cuda):
    import torch
    N = _n()
    _, (s,), mag = _gold("abs_cf32")
    (got,) = N.run_sync_factory("MeanAbs", {"axis": -3, "keepdims": True}, [torch.from_numpy(s).to(cuda)])
    assert rel(got.cpu().numpy(), np.mean(mag, axis=-3, keepdims=True)) < 1e-6


def test_conversion_nodes(cuda, rng):
    import torch
    N = _n()
    u = rng.integers(0, 4096, (4, 33)).astype(np.uint16)
    (c,) = N.run_sync_factory("Conversion", {"target": "CF32", "strategy": "Real"},
                              [torch.from_numpy(u.view(np.int16)).to(cuda)], dtypes=[1])
    assert np.array_equal(c.cpu().numpy(), O.convert(u, "U16", "CF32", "Real"))
    z = (rng.standard_normal((5, 7)) + 1j * rng.standard_normal((5, 7))).astype(np.complex64)
    (m,) = N.run_sync_factory("Conversion", {"target": "F32", "strategy": "Modulus"}, [torch.from_numpy(z).to(cuda)])
    assert rel(m.cpu().numpy(), O.convert(z, "CF32", "F32", "Modulus")) < 1e-6
    f = rng.standard_normal((6, 10)).astype(np.float32)
    (q,) = N.run_sync_factory("Conversion", {"target": "U8", "strategy": "Scaled"}, [torch.from_numpy(f).to(cuda)])
    assert np.array_equal(q.cpu().numpy(), O.convert(f, "F32", "U8", "Scaled"))


def _windows(frames, T):
    n = frames.shape[0] // T
    return frames[: n * T].reshape(n, T, *frames.shape[1:])


def test_doppler_moments_node_u16_angular_spectrum(cuda):
    import torch
    N = _n()
    frames = S.Interferograms(S.config0(64)).frames(0, 64)[:, :128, :128].copy()
    win = _windows(frames, 32)
    s = {"time_z_begin": 6, "time_z_end": 16, "propagation": "angular_spectrum", "lambda": LAM, "dx": DX, "z": 0.3,
         "input_format": "u16", "padding": {"width": 256, "height": 256}}
    (got,) = N.run_sync_factory("DopplerMoments", s, [torch.from_numpy(win.view(np.int16)).to(cuda)], dtypes=[1])
    cfg = O.PathConfig(128, 128, 32, 32, 6, 16, propagation="angular_spectrum", z=0.3,
                       as_padding={"width": 256, "height": 256})
    for w in range(win.shape[0]):
        exp = O.reconstruct_window(win[w], cfg)
        for m in range(3):
            assert rel(got[w, m].cpu().numpy(), exp[m]) < 1e-4, (w, m)


def test_doppler_moments_node_mono12p_chosen_and_z_update(cuda):
    import torch
    N = _n()
    H = W = 128
    frames = S.Interferograms(S.config1(128, height=H, width=W)).frames(0, 128)
    packed = O.pack12(frames.reshape(-1)).reshape(2, 64, H * W * 3 // 2)
    dev = torch.from_numpy(packed).to(cuda)
    s = {"time_z_begin": 4, "time_z_end": 32, "propagation": "fresnel", "lambda": LAM, "dx": DX, "z": 0.25,
         "fs": 67e3, "clutter_rank": 4, "input_format": "mono12p", "height": H, "width": W, "form": "chosen"}
    (got,) = N.run_sync_factory("DopplerMoments", s, [dev])
    for z in (0.25, 0.3):
        cfg = O.PathConfig(H, W, 64, 64, 4, 32, fs=67e3, z=z, clutter_rank=4)
        if z != 0.25:  # update with only z changed keeps the task and rebuilds the lens
            node = N.Node("DopplerMoments", s, [N.desc_of(dev)])
            node.update({**s, "z": z}, [N.desc_of(dev)])
            got = torch.empty((2, 3, H, W), dtype=torch.float32, device=cuda)
            assert node.execute([dev], [got]) == 0
            torch.cuda.synchronize()
            node.close()
        for w in range(2):
            exp = O.reconstruct_window(frames[64 * w: 64 * w + 64], cfg)
            for m in range(3):
                assert rel(got[w, m].cpu().numpy(), exp[m]) < 1e-3, (z, w, m)


def test_holofile_gpu_cached_source_feeds_doppler_moments(cuda, tmp_path):
    """A 12-bit .holo loaded once into device memory ("Holofile", GPUCached) hands out each batch
    of packed frames as a view into its cache; fed to "DopplerMoments" as one 64-frame window, the
    moment images equal those of the same frames uploaded directly (same kernels, same bytes)."""
    import torch
    from holoflow_b200 import holofile as HF
    N = _n()
    H = W = 128
    frames = S.Interferograms(S.config1(128, height=H, width=W)).frames(0, 128)
    packed = O.pack12(frames.reshape(-1)).reshape(128, H * W * 3 // 2)
    path = str(tmp_path / "acq.holo")
    HF.write(path, packed, 12, width=W, height=H, footer={"fs": 67000})
    src = N.Node("Holofile", {"path": path, "load_kind": "GPUCached", "start_frame": 0, "end_frame": 128,
                              "batch_size": 64}, [])
    od = src.output_desc(0)
    assert N.shape_of(od) == (64, H, W * 3 // 2) and od.mem_loc == 1
    s = {"time_z_begin": 4, "time_z_end": 32, "propagation": "fresnel", "lambda": LAM, "dx": DX, "z": 0.25,
         "fs": 67e3, "clutter_rank": 4, "input_format": "mono12p", "height": H, "width": W, "form": "chosen"}
    win = N.desc_of(torch.empty((1, 64, H * W * 3 // 2), dtype=torch.uint8, device=cuda))
    dop = N.Node("DopplerMoments", s, [win])
    got = torch.empty((1, 3, H, W), dtype=torch.float32, device=cuda)
    for b in range(3):  # the third batch wraps back to frame 0
        assert src.execute([], [None]) == 0
        ptr, owned = src.output_ptr(0)
        assert owned and ptr
        assert dop.execute([ptr], [got]) == 0
        torch.cuda.synchronize()
        first = 64 * (b % 2)
        direct = torch.from_numpy(packed[first:first + 64].reshape(1, 64, -1).copy()).to(cuda)
        (ref,) = N.run_sync_factory("DopplerMoments", s, [direct])
        assert torch.equal(got, ref), b
    dop.close()
    src.close()


# ---- the thin holonp kinds and the queues --------------------------------------------------------
def test_thin_kinds_against_the_reference_oracle_goldens(cuda):
    """Slice (a view), Copy, Arange, Multiply and Abs through hf_node_* against the outputs of the
    reference's own NumPy test oracle (tests/golden/holonp_ops.npz)."""
    import torch
    N = _n()
    st, (x,), y = _gold("slice_band_4_32")
    dev = torch.from_numpy(x).to(cuda)
    # numpy pads missing trailing items with ':'; the node takes one item per dimension
    # (slice.cu:199-200)
    st = {"slices": st["slices"] + [{}] * (x.ndim - len(st["slices"]))}
    (v,) = N.run_sync_factory("Slice", st, [dev])
    assert v.data_ptr() == dev[:, 4:32].data_ptr() and tuple(v.shape) == y.shape   # a view, no copy
    (c,) = N.run_sync_factory("Copy", {}, [v])
    assert c.is_contiguous() and np.array_equal(c.cpu().numpy(), y)
    st, _, y = _gold("arange_band_t64")
    (a,) = N.run_sync_factory("Arange", st, [])
    assert np.array_equal(a.cpu().numpy(), y)
    st, (p, q), y = _gold("multiply_weights")
    (m,) = N.run_sync_factory("Multiply", st, [torch.from_numpy(p).to(cuda), torch.from_numpy(q).to(cuda)])
    assert rel(m.cpu().numpy(), y) < 1e-7
    st, (z,), y = _gold("abs_cf32")
    (b,) = N.run_sync_factory("Abs", st, [torch.from_numpy(z).to(cuda)])
    assert rel(b.cpu().numpy(), y) < 1e-6


def test_reshape_concatenate_and_causal_average(cuda, rng):
    import torch
    N = _n()
    x = torch.from_numpy(rng.standard_normal((2, 6, 10)).astype(np.float32)).to(cuda)
    (r,) = N.run_sync_factory("Reshape", {"shape": [1, 2, 6, -1]}, [x])
    assert r.data_ptr() == x.data_ptr() and torch.equal(r, x.reshape(1, 2, 6, 10))
    t = x.transpose(1, 2)                                       # [2, 10, 6], not viewable flat
    (r2,) = N.run_sync_factory("Reshape", {"shape": [120]}, [t])
    assert r2.data_ptr() != t.data_ptr() and torch.equal(r2, t.reshape(120))
    a = torch.from_numpy((rng.standard_normal((2, 3, 5)) + 1j * rng.standard_normal((2, 3, 5))).astype(np.complex64))
    b = torch.from_numpy((rng.standard_normal((2, 4, 5)) + 1j * rng.standard_normal((2, 4, 5))).astype(np.complex64))
    (c,) = N.run_sync_factory("Concatenate", {"axis": -2}, [a.to(cuda), b.to(cuda)])
    assert torch.equal(c.cpu(), torch.cat([a, b], dim=1))
    from oracle import shack as SH
    node = N.Node("CausalSlidingAverage", {"window_size": 3}, [N.desc_of(x)])
    avg = SH.CausalSlidingAverage(3)
    for k in range(5):
        inp = torch.from_numpy(rng.standard_normal((2, 6, 10)).astype(np.float32)).to(cuda)
        out = torch.empty_like(inp)
        node.execute([inp], [out])
        torch.cuda.synchronize()
        assert np.allclose(out.cpu().numpy(), avg(inp.cpu().numpy()), rtol=1e-6, atol=1e-6), k
    node.close()


def test_batch_queue_and_dual_reader(cuda, rng):
    """BatchQueue windows of output_size elements every output_stride pushes (zero-copy views into
    its ring), and the DualReaderBatchQueue's current / delayed elements and valid flag
    (dual_reader_batch_queue.cc:104-156)."""
    import torch
    N = _n()
    el = N.desc_of(torch.empty((1, 4, 3), device=cuda))
    bq = N.async_node("BatchQueue", {"target_capacity": 4, "output_size": 2, "output_stride": 2}, [el])
    vals = [torch.full((1, 4, 3), float(k), device=cuda) for k in range(6)]
    got = []
    for k in range(6):
        slot = bq.acquire_input()
        assert slot is not None
        slot.copy_(vals[k])
        assert bq.try_push() == 0
        if bq.try_pop() == 0:
            got.append(bq.output().clone())
            bq.release_output()
    torch.cuda.synchronize()
    assert [g[:, 0, 0].tolist() for g in got] == [[0.0, 1.0], [2.0, 3.0], [4.0, 5.0]]
    bq.close()
    d = N.desc_of(torch.empty((2, 3, 4), device=cuda))
    dr = N.async_node("DualReaderBatchQueue", {"target_capacity": 4, "window_size": 5}, [d])   # delay 2
    flag = torch.zeros(1, dtype=torch.uint8)
    seen = []
    for k in range(3):                                        # pushes of 2 elements: values 2k, 2k + 1
        slot = dr.acquire_input()
        slot.copy_(torch.stack([torch.full((3, 4), 2.0 * k, device=cuda), torch.full((3, 4), 2.0 * k + 1, device=cuda)]))
        assert dr.try_push() == 0
        while dr.try_pop([None, None, flag]) == 0:
            torch.cuda.synchronize()
            seen.append((dr.output(0)[0, 0, 0].item(), dr.output(1)[0, 0, 0].item(), int(flag.item())))
            dr.release_output(0)
            dr.release_output(1)
    # element w, delayed element w - 2 (zero before), valid once 4 elements were popped before
    assert seen == [(0, 0, 0), (1, 0, 0), (2, 0, 0), (3, 1, 0), (4, 2, 1), (5, 3, 1)]
    dr.close()


def test_reference_graph_node_by_node_equals_the_fused_node(cuda):
    """The node sequence GraphBuilder emits for the RFFT time method with Fresnel and M0/M1/M2
    (graph_builder.cc:245-305, 522-566, 578-631): Conversion -> Reshape [1, T, H, W] -> BatchQueue
    -> RFFT(axis 1) -> Slice [z0, z1) -> Copy -> DualReaderBatchQueue -> FresnelDiffraction (|.|) ->
    Mean(-3) for M0, Arange -> Reshape -> Multiply -> Mean for M1 and M2; against the fused
    DopplerMoments node on the same frames (the weights with fs = 37 kHz, as the reference's)."""
    import torch
    N = _n()
    T, H, W, z0, z1, NPRE = 32, 64, 64, 6, 16, 2
    frames = S.Interferograms(S.config0(T * NPRE)).frames(0, T * NPRE)[:, :H, :W]
    # 8-bit frames: the reference's Conversion takes U8 -> F32 Real only (conversion.cu:140-147)
    u8 = torch.from_numpy((frames >> 4).astype(np.uint8)).to(cuda)
    fres = {"lambda": LAM, "dx": DX, "dy": DX, "z": 0.3, "output_magnitude": True, "skip_phase_shift": True}
    desc = N.desc_of
    bq = N.async_node("BatchQueue", {"target_capacity": 2 * NPRE, "output_size": NPRE, "output_stride": NPRE},
                      [desc(torch.empty((1, T, H, W), device=cuda))])
    for w in range(NPRE):                                     # one window of T frames per push
        (f32,) = N.run_sync_factory("Conversion", {"target": "F32", "strategy": "Real"}, [u8[w * T:(w + 1) * T]])
        (win,) = N.run_sync_factory("Reshape", {"shape": [1, T, H, W]}, [f32])
        slot = bq.acquire_input()
        slot.copy_(win)
        assert bq.try_push() == 0
    assert bq.try_pop() == 0
    batch = bq.output()                                       # [NPRE, T, H, W]
    (spec,) = N.run_sync_factory("RFFT", {"axis": 1}, [batch])
    (band,) = N.run_sync_factory("Slice", {"slices": [{}, {"start": z0, "stop": z1}, {}, {}]}, [spec])
    (band,) = N.run_sync_factory("Copy", {}, [band])
    bq.release_output()
    dr = N.async_node("DualReaderBatchQueue", {"target_capacity": 4, "window_size": 1}, [desc(band)])
    slot = dr.acquire_input()
    slot.copy_(band)
    assert dr.try_push() == 0
    df = 37e3 / T
    (freqs,) = N.run_sync_factory("Arange", {"start": z0 * df, "stop": z1 * df, "step": df, "dtype": "F32"}, [])
    (fw,) = N.run_sync_factory("Reshape", {"shape": [1, z1 - z0, 1, 1]}, [freqs])
    (fw2,) = N.run_sync_factory("Multiply", {}, [fw, fw])
    flag = torch.zeros(1, dtype=torch.uint8)
    graph = []
    while dr.try_pop([None, None, flag]) == 0:
        cur = dr.output(0)                                    # [1, Nz, H, W]
        (mag,) = N.run_sync_factory("FresnelDiffraction", fres, [cur])
        (m0,) = N.run_sync_factory("Mean", {"axis": [-3], "keepdims": True}, [mag])
        (w1,) = N.run_sync_factory("Multiply", {}, [fw, mag])
        (m1,) = N.run_sync_factory("Mean", {"axis": [-3], "keepdims": True}, [w1])
        (w2,) = N.run_sync_factory("Multiply", {}, [fw2, mag])
        (m2,) = N.run_sync_factory("Mean", {"axis": [-3], "keepdims": True}, [w2])
        graph.append(torch.cat([m0, m1, m2], dim=1)[0].cpu().numpy())
        dr.release_output(0)
        dr.release_output(1)
    assert len(graph) == NPRE
    s = {"time_z_begin": z0, "time_z_end": z1, "propagation": "fresnel", "lambda": LAM, "dx": DX, "z": 0.3,
         "input_format": "u8", "fs": 37e3, "form": "plain"}
    for w in range(NPRE):
        (fused,) = N.run_sync_factory("DopplerMoments", s, [u8[w * T:(w + 1) * T].reshape(1, T, H, W)])
        f = fused.cpu().numpy()[0]
        for m in range(3):
            assert rel(f[m], graph[w][m]) < 1e-5, (w, m, rel(f[m], graph[w][m]))
    bq.close()
    dr.close()
