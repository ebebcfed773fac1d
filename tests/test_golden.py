"""Pins the oracle and the CUDA entry points to golden vectors made by the reference's own NumPy
test oracle (test/holonp/python/oracle.py; fixtures and generator in tests/golden/).

CPU tests check this repository's oracle against every fixture.  GPU tests run the matching C-ABI
entry points (temporal DFT, Mean, MeanAbs, band moments) on the same inputs.
"""
import json
import pathlib

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "holonp_ops.npz"


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLDEN)
    index = json.loads(bytes(z["__index__"]).decode())
    cases = {}
    for name, meta in index.items():
        ins = [z[f"{name}__in{i}"] for i in range(meta["ninputs"])]
        outs = [z[f"{name}__out{i}"] for i in range(meta["noutputs"])]
        cases[name] = (meta["op"], meta["settings"], ins, outs)
    return cases


def _rel(a, b):
    return O.rel_l2(np.asarray(a), np.asarray(b))


# ------------------------------------------------------------------------------------------------
# oracle vs the reference's NumPy oracle
# ------------------------------------------------------------------------------------------------
def test_every_fixture_has_an_oracle_check(gold):
    assert len(gold) == 16


@pytest.mark.parametrize("name", ["fft_f32_axis1_backward", "fft_f32_axis1_forward", "fft_f32_axis1_ortho",
                                  "fft_cf32_axis1", "fft_u16_axis1"])
def test_oracle_fft_axis(gold, name):
    _, st, (x,), (y,) = gold[name]
    got = O.fft_axis(x, st["axis"], st["norm"])
    assert y.dtype == np.complex64 and got.shape == y.shape
    assert _rel(got, y) < 1e-7


def test_oracle_rfft_and_band_slice(gold):
    _, st, (x,), (y,) = gold["rfft_f32_axis1_t64"]
    assert _rel(O.rfft_axis(x, st["axis"], st["norm"]), y) < 1e-7
    # band_dft = RFFT then Slice [4:32) along T (graph_builder.cc:264-286)
    got = np.stack([O.band_dft(x[b], 4, 32) for b in range(x.shape[0])])
    assert _rel(got, y[:, 4:32]) < 1e-7
    _, st, (s,), (t,) = gold["slice_band_4_32"]
    assert np.array_equal(s[:, 4:32], t)


@pytest.mark.parametrize("name", ["mean_f32_axis_m3", "mean_cf32_axis_m3", "mean_f32_axis0"])
def test_oracle_mean(gold, name):
    _, st, (x,), (y,) = gold[name]
    got = O.mean(x, [st["axis"]], keepdims=st["keepdims"])
    assert got.shape == y.shape
    assert _rel(got, y) < 1e-6


def test_oracle_abs_and_mean_abs(gold):
    _, _, (x,), (y,) = gold["abs_cf32"]
    assert y.dtype == np.float32
    assert _rel(np.abs(x.astype(np.complex128)), y) < 1e-7
    assert _rel(O.mean_abs(x, [-3]), np.mean(y, axis=-3, keepdims=True)) < 1e-6


@pytest.mark.parametrize("name,T,z0,z1", [("arange_band_t64", 64, 4, 32), ("arange_band_t32", 32, 6, 16)])
def test_oracle_freq_weights(gold, name, T, z0, z1):
    _, st, _, (y,) = gold[name]
    assert np.array_equal(O.arange_f32(st["start"], st["stop"], st["step"]), y)
    assert np.array_equal(O.freq_weights(T, z0, z1, fs=37e3), y)


def test_oracle_moments_follow_multiply_then_mean(gold):
    _, _, (a, w), (y,) = gold["multiply_weights"]
    assert np.array_equal(a * w, y)
    _, _, (s,), (mag,) = gold["abs_cf32"]
    _, _, _, (f,) = gold["arange_band_t64"]
    m = O.moments_from_magnitude(mag[0], f)
    assert _rel(m[0], np.mean(mag[0], axis=0)) < 1e-6
    assert _rel(m[1], np.mean(f[:, None, None] * mag[0], axis=0)) < 1e-6
    f2 = (f * f).astype(np.float32)
    assert _rel(m[2], np.mean(f2[:, None, None] * mag[0], axis=0)) < 1e-6


def test_oracle_fft2_and_fftshift(gold):
    _, st, (x,), (y,) = gold["fft2_cf32"]
    got = O.fft_axis(O.fft_axis(x, -1), -2)
    assert _rel(got, y) < 1e-7
    _, st, (x,), (y,) = gold["fftshift_f32"]
    assert np.array_equal(np.fft.fftshift(x, axes=tuple(st["axes"])), y)


# ------------------------------------------------------------------------------------------------
# CUDA entry points vs the same fixtures
# ------------------------------------------------------------------------------------------------
def _dev(cuda, a):
    import torch
    if a.dtype == np.uint16:
        return torch.from_numpy(a.view(np.int16).copy()).to(cuda)
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fft_f32_axis1_backward", "fft_f32_axis1_forward", "fft_f32_axis1_ortho",
                                  "fft_cf32_axis1", "fft_u16_axis1", "rfft_f32_axis1_t64"])
def test_gpu_temporal_dft(cuda, gold, name):
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    _, st, (x,), (y,) = gold[name]
    B, T = x.shape[:2]
    P = int(np.prod(x.shape[2:]))
    dt = {np.dtype(np.float32): hf.HF_F32, np.dtype(np.complex64): hf.HF_CF32,
          np.dtype(np.uint16): hf.HF_U16}[x.dtype]
    norm = {"backward": hf.HF_NORM_BACKWARD, "forward": hf.HF_NORM_FORWARD, "ortho": hf.HF_NORM_ORTHO}[st["norm"]]
    nb = y.shape[1]
    got = pl.temporal_dft(_dev(cuda, x), dt, B, T, P, 0, nb, norm).cpu().numpy()
    assert _rel(got, y.reshape(B, nb, P)) < 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["mean_f32_axis_m3", "mean_cf32_axis_m3", "mean_f32_axis0"])
def test_gpu_mean(cuda, gold, name):
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    _, st, (x,), (y,) = gold[name]
    ax = st["axis"] % x.ndim
    outer = int(np.prod(x.shape[:ax]))
    n = x.shape[ax]
    inner = int(np.prod(x.shape[ax + 1:]))
    cplx = x.dtype == np.complex64
    out = torch.empty(outer * inner, dtype=torch.complex64 if cplx else torch.float32, device=cuda)
    hf.check(hf.lib().hf_mean_axis(pl._ptr(_dev(cuda, x)), hf.HF_CF32 if cplx else hf.HF_F32, outer, n, inner,
                                   pl._ptr(out), pl._stream()))
    assert _rel(out.cpu().numpy(), y.reshape(-1)) < 1e-6


@pytest.mark.gpu
def test_gpu_mean_abs_and_band_moments(cuda, gold):
    import ctypes as C
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    _, _, (s,), (mag,) = gold["abs_cf32"]
    _, _, _, (f,) = gold["arange_band_t64"]
    nz, P = s.shape[1], s.shape[2] * s.shape[3]
    sd = _dev(cuda, s)
    out = torch.empty(P, dtype=torch.float32, device=cuda)
    hf.check(hf.lib().hf_mean_abs_axis(pl._ptr(sd), hf.HF_CF32, 1, nz, P, pl._ptr(out), pl._stream()))
    assert _rel(out.cpu().numpy(), np.mean(mag, axis=1).reshape(-1)) < 1e-6
    mom = torch.empty(3 * P, dtype=torch.float32, device=cuda)
    freqs = (C.c_float * nz)(*f.tolist())
    hf.check(hf.lib().hf_band_moments(pl._ptr(sd), hf.HF_CF32, nz, P, freqs, hf.HF_M0 | hf.HF_M1 | hf.HF_M2,
                                      pl._ptr(mom), pl._stream()))
    got = mom.cpu().numpy().reshape(3, P)
    m = mag[0].reshape(nz, P)
    f2 = (f * f).astype(np.float32)
    assert _rel(got[0], m.mean(0)) < 1e-6
    assert _rel(got[1], (f[:, None] * m).mean(0)) < 1e-6
    assert _rel(got[2], (f2[:, None] * m).mean(0)) < 1e-6
