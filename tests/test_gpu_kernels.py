"""GPU parity of the stage kernels against the CPU oracle, through the C ABI."""
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

LAM, DX = 852e-9, 20e-6


def _hf():
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    return hf, pl


def rel(a, b):
    return O.rel_l2(a, b)


# ---------------------------------------------------------------------------------------------
# a1: 12-bit unpack (bit exact)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("npix", [2, 6, 8, 4096 * 2, 1000002, 1 << 20])
@pytest.mark.parametrize("out", ["u16", "f32", "cf32"])
def test_unpack12_bit_exact(cuda, rng, npix, out):
    import torch
    hf, pl = _hf()
    vals = rng.integers(0, 4096, npix).astype(np.uint16)
    if npix >= 8192:
        vals[:8192] = np.tile(np.arange(4096, dtype=np.uint16), 2)  # every value, both phases
    packed = torch.from_numpy(O.pack12(vals)).to(cuda)
    dt = {"u16": hf.HF_U16, "f32": hf.HF_F32, "cf32": hf.HF_CF32}[out]
    got = pl.unpack12(packed, npix, dt)
    torch.cuda.synchronize()
    if out == "u16":
        g = got.cpu().numpy().view(np.uint16)
        assert np.array_equal(g, vals)
    elif out == "f32":
        assert np.array_equal(got.cpu().numpy(), vals.astype(np.float32))
    else:
        g = got.cpu().numpy()
        assert np.array_equal(g.real, vals.astype(np.float32)) and not g.imag.any()


def test_unpack12_misaligned_and_pack_roundtrip(cuda, rng):
    import torch
    hf, pl = _hf()
    vals = rng.integers(0, 4096, 1002).astype(np.uint16)
    buf = torch.zeros(1 + 1503, dtype=torch.uint8, device=cuda)
    buf[1:] = torch.from_numpy(O.pack12(vals)).to(cuda)
    out = torch.empty(1002, dtype=torch.float32, device=cuda)
    hf.check(hf.lib().hf_unpack12(pl._ptr(buf[1:]), pl._ptr(out), hf.HF_F32, 1002, pl._stream()))
    assert np.array_equal(out.cpu().numpy(), vals.astype(np.float32))
    t = torch.from_numpy(vals.view(np.int16)).to(cuda)
    assert np.array_equal(pl.pack12(t).cpu().numpy(), O.pack12(vals))


def test_unpack12_rejects_odd_count(cuda):
    import torch
    hf, pl = _hf()
    buf = torch.zeros(16, dtype=torch.uint8, device=cuda)
    with pytest.raises(hf.HfError) as e:
        pl.unpack12(buf, 3)
    assert e.value.code == hf.HF_ERR_INVALID


# ---------------------------------------------------------------------------------------------
# a5-a7: temporal DFT / RFFT + band slice (fft_test.cu rtol 1e-4)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("fmt,T,P,z0,z1", [
    ("mono12p", 64, 1024 * 8, 4, 32), ("u16", 32, 512 * 16, 6, 16), ("u8", 16, 4096, 0, 9),
    ("f32", 64, 2048, 0, 33), ("cf32", 8, 96, 0, 8), ("mono12p", 64, 998, 4, 32), ("f32", 7, 33, 1, 5)])
def test_temporal_dft(cuda, rng, fmt, T, P, z0, z1):
    import torch
    hf, pl = _hf()
    B = 2
    if fmt == "cf32":
        x = (rng.standard_normal((B, T, P)) + 1j * rng.standard_normal((B, T, P))).astype(np.complex64)
        dev = torch.from_numpy(x).to(cuda)
        dt = hf.HF_CF32
    else:
        top = {"mono12p": 4096, "u16": 4096, "u8": 256, "f32": 4096}[fmt]
        x = rng.integers(0, top, (B, T, P)).astype(np.float64)
        if fmt == "mono12p":
            dev = torch.from_numpy(O.pack12(x.astype(np.uint16).reshape(-1))).to(cuda)
            dt = hf.HF_MONO12P
        elif fmt == "u16":
            dev = torch.from_numpy(x.astype(np.uint16).view(np.int16)).to(cuda)
            dt = hf.HF_U16
        elif fmt == "u8":
            dev = torch.from_numpy(x.astype(np.uint8)).to(cuda)
            dt = hf.HF_U8
        else:
            dev = torch.from_numpy(x.astype(np.float32)).to(cuda)
            dt = hf.HF_F32
    got = pl.temporal_dft(dev, dt, B, T, P, z0, z1).cpu().numpy()
    exp = np.fft.fft(x, axis=1)[:, z0:z1]
    assert rel(got, exp) < 1e-5
    for norm, scale in ((hf.HF_NORM_FORWARD, 1.0 / T), (hf.HF_NORM_ORTHO, 1.0 / math.sqrt(T))):
        g2 = pl.temporal_dft(dev, dt, B, T, P, z0, z1, norm).cpu().numpy()
        assert rel(g2, exp * scale) < 1e-5


# ---------------------------------------------------------------------------------------------
# a8: covariance (Gram) and Jacobi
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("fmt,T,P", [("mono12p", 64, 1 << 16), ("u16", 32, 4096 * 3), ("mono12p", 128, 8192),
                                      ("f32", 64, 1024), ("u8", 16, 1000), ("mono12p", 64, 1000)])
def test_covariance(cuda, rng, fmt, T, P):
    import torch
    hf, pl = _hf()
    B = 2
    top = 256 if fmt == "u8" else 4096
    x = rng.integers(0, top, (B, T, P))
    if fmt == "mono12p":
        dev, dt = torch.from_numpy(O.pack12(x.astype(np.uint16).reshape(-1))).to(cuda), hf.HF_MONO12P
    elif fmt == "u16":
        dev, dt = torch.from_numpy(x.astype(np.uint16).view(np.int16)).to(cuda), hf.HF_U16
    elif fmt == "u8":
        dev, dt = torch.from_numpy(x.astype(np.uint8)).to(cuda), hf.HF_U8
    else:
        dev, dt = torch.from_numpy(x.astype(np.float32)).to(cuda), hf.HF_F32
    g = pl.covariance(dev, dt, B, T, P).cpu().numpy()
    for b in range(B):
        X = x[b].reshape(T, -1).astype(np.float64)
        exp = X @ X.T
        assert np.abs(g[b] - exp).max() / np.abs(exp).max() < 2e-7
        assert np.array_equal(g[b], g[b].T)


@pytest.mark.parametrize("fmt", ["u16", "u8", "mono12p"])
def test_misaligned_inputs_take_the_direct_kernels(cuda, rng, fmt):
    """Frames whose base is only 2-byte (u16) or 1-byte aligned are valid input: the Gram and
    temporal-DFT entry points route them to kernels without 4-byte word loads and still match."""
    import torch
    hf, pl = _hf()
    B, T, P = 2, 64, 4096
    top = 256 if fmt == "u8" else 4096
    x = rng.integers(0, top, (B, T, P))
    if fmt == "u16":
        host = x.astype(np.uint16).view(np.int16).reshape(-1)
        buf = torch.zeros(host.size + 1, dtype=torch.int16, device=cuda)
        buf[1:] = torch.from_numpy(host).to(cuda)
        dev, dt = buf[1:], hf.HF_U16              # base at a 2-byte offset
    else:
        host = O.pack12(x.astype(np.uint16).reshape(-1)) if fmt == "mono12p" else x.astype(np.uint8).reshape(-1)
        buf = torch.zeros(host.size + 3, dtype=torch.uint8, device=cuda)
        buf[3:] = torch.from_numpy(host).to(cuda)
        dev, dt = buf[3:], (hf.HF_MONO12P if fmt == "mono12p" else hf.HF_U8)  # 1-byte aligned
    assert dev.data_ptr() % 4 != 0
    g = pl.covariance(dev, dt, B, T, P).cpu().numpy()
    for b in range(B):
        X = x[b].astype(np.float64)
        exp = X @ X.T
        assert np.abs(g[b] - exp).max() / np.abs(exp).max() < 2e-7
    got = pl.temporal_dft(dev, dt, B, T, P, 4, 32).cpu().numpy()
    assert rel(got, np.fft.fft(x.astype(np.float64), axis=1)[:, 4:32]) < 1e-5


@pytest.mark.parametrize("n", [2, 3, 16, 63, 64, 128])
def test_jacobi_matches_eigh(cuda, rng, n):
    import torch
    hf, pl = _hf()
    B = 3
    a = rng.standard_normal((B, n, n))
    a = a @ a.transpose(0, 2, 1) + np.eye(n)  # SPD with a spread spectrum
    a[0] *= 1e12  # large magnitudes like Gram matrices of 12-bit frames
    ev, V, info = pl.eigh_jacobi(torch.from_numpy(a).to(cuda))
    ev, V, info = ev.cpu().numpy(), V.cpu().numpy(), info.cpu().numpy()
    assert (info == 0).all()
    for b in range(B):
        w, _ = np.linalg.eigh(a[b])
        assert np.abs(ev[b] - w).max() <= 1e-11 * np.abs(w).max()
        assert np.all(np.diff(ev[b]) >= 0)
        recon = (V[b] * ev[b]) @ V[b].T
        assert np.abs(recon - a[b]).max() <= 1e-11 * np.abs(a[b]).max()
        assert np.abs(V[b].T @ V[b] - np.eye(n)).max() < 1e-12


@pytest.mark.parametrize("n,r", [(64, 4), (128, 4), (64, 16), (17, 3), (2, 2), (1, 1)])
def test_top_eigenpairs_match_eigh(cuda, rng, n, r):
    """The clutter filter's top-r solver (tridiagonalisation, Sturm multisection, inverse
    iteration): eigenvalues, residuals, orthonormality and the top-r projector against numpy, on
    Gram matrices of 12-bit-like data (magnitudes ~1e12) and on indefinite symmetric matrices."""
    import torch
    hf, pl = _hf()
    B = 3
    x = rng.integers(0, 4096, size=(B, n, 2000)).astype(np.float64) - 2048
    a = np.einsum("bij,bkj->bik", x, x)
    m = rng.standard_normal((B, n, n))
    a[1] = m[1] + m[1].T
    ev, V, info = pl.eigh_top(torch.from_numpy(a).to(cuda), r)
    ev, V, info = ev.cpu().numpy(), V.cpu().numpy(), info.cpu().numpy()
    assert (info == 0).all()
    for b in range(B):
        w, U = np.linalg.eigh(a[b])
        scale = np.abs(w).max()
        assert np.abs(ev[b] - w[n - r:]).max() <= 1e-12 * scale
        assert np.all(np.diff(ev[b]) >= 0)
        assert np.abs(V[b].T @ V[b] - np.eye(r)).max() < 1e-12
        assert np.abs(a[b] @ V[b] - V[b] * ev[b]).max() <= 1e-12 * scale
        if n > r and (w[n - r] - w[n - r - 1]) > 1e-6 * scale:  # a separated top-r subspace
            P, Q = V[b] @ V[b].T, U[:, n - r:] @ U[:, n - r:].T
            assert np.abs(P - Q).max() < 1e-9


def test_top_eigenpairs_repeated_and_nonfinite(cuda, rng):
    """A repeated top eigenvalue gets an orthonormal basis of its eigenspace; a non-finite input
    reports info = 1 and leaves the outputs alone."""
    import torch
    hf, pl = _hf()
    q, _ = np.linalg.qr(rng.standard_normal((64, 64)))
    lam = np.concatenate([np.arange(60.0), [100.0, 100.0, 200.0, 300.0]])
    a = np.stack([q @ np.diag(lam) @ q.T, np.full((64, 64), np.nan)])
    ev, V, info = pl.eigh_top(torch.from_numpy(a).to(cuda), 4)
    ev, V, info = ev.cpu().numpy(), V.cpu().numpy(), info.cpu().numpy()
    assert list(info) == [0, 1]
    assert np.abs(ev[0] - [100, 100, 200, 300]).max() < 1e-11
    assert np.abs(V[0].T @ V[0] - np.eye(4)).max() < 1e-12
    P, Q = V[0] @ V[0].T, q[:, 60:] @ q[:, 60:].T
    assert np.abs(P - Q).max() < 1e-10
    assert not V[1].any() and not ev[1].any()


def test_jacobi_reference_pca_kat(cuda):
    """pca_test.cu:134-145 through the GPU Gram + Jacobi: energies of the projections are the
    ascending eigenvalues {1, 3}."""
    import torch
    hf, pl = _hf()
    x = np.array([math.sqrt(2), 0.0, 1 / math.sqrt(2), math.sqrt(1.5)], np.float32).reshape(1, 2, 2)
    g = pl.covariance(torch.from_numpy(x).to(cuda), hf.HF_F32, 1, 2, 2)
    ev, V, info = pl.eigh_jacobi(g)
    np.testing.assert_allclose(ev.cpu().numpy()[0], [1.0, 3.0], atol=1e-6)


# ---------------------------------------------------------------------------------------------
# a9: Fresnel diffraction node
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("B,H,W", [(2, 32, 48), (3, 64, 128), (2, 256, 512), (1, 1024, 1024), (2, 768, 1536), (1, 100, 60)])
@pytest.mark.parametrize("mode", ["complex", "magnitude", "phase"])
def test_fresnel_node(cuda, rng, B, H, W, mode):
    import torch
    hf, pl = _hf()
    x = (rng.standard_normal((B, H, W)) + 1j * rng.standard_normal((B, H, W))).astype(np.complex64)
    z = 0.05
    mag, skip = mode == "magnitude", mode != "phase"
    plan = pl.FresnelPlan(B, H, W, hf.HF_CF32, LAM, DX, z, output_magnitude=mag, skip_phase_shift=skip)
    got = plan(torch.from_numpy(x).to(cuda)).cpu().numpy()
    exp = O.fresnel(x, LAM, DX, DX, z, output_magnitude=mag, skip_phase_shift=skip)
    assert rel(got, exp) < 2e-6 * math.log2(H * W)


def test_fresnel_real_strided_input_and_set_z(cuda, rng):
    import torch
    hf, pl = _hf()
    big = rng.standard_normal((2, 64, 256)).astype(np.float32)
    dev = torch.from_numpy(big).to(cuda)[:, :, ::2]  # column stride 2 (reference: stride(H) % stride(W) == 0)
    plan = pl.FresnelPlan(2, 64, 128, hf.HF_F32, LAM, DX, 0.02, output_magnitude=True)
    got = plan(dev).cpu().numpy()
    exp = O.fresnel(big[:, :, ::2], LAM, DX, DX, 0.02, output_magnitude=True)
    assert rel(got, exp) < 3e-5
    plan.set_z(0.03)
    got = plan(dev).cpu().numpy()
    exp = O.fresnel(big[:, :, ::2], LAM, DX, DX, 0.03, output_magnitude=True)
    assert rel(got, exp) < 3e-5


# ---------------------------------------------------------------------------------------------
# a10: Angular spectrum node, the reference KATs first
# ---------------------------------------------------------------------------------------------
def _as(cuda, x, in_dtype, z=0.0, padding=None, filt=None, inplace=False):
    import torch
    hf, pl = _hf()
    B, H, W = x.shape
    plan = pl.AngularSpectrumPlan(B, H, W, in_dtype, LAM, DX, z, padding, filt)
    dev = torch.from_numpy(x).to(cuda)
    out = plan(dev, dev if inplace else None)
    return out.cpu().numpy()


def test_as_kat_zero_distance_real(cuda):
    hf, _ = _hf()
    got = _as(cuda, np.array([[[1, 2], [3, 4]]], np.float32), hf.HF_F32)
    np.testing.assert_allclose(got[0], [[4, 8], [12, 16]], atol=1e-3)


def test_as_kat_padding(cuda):
    hf, _ = _hf()
    got = _as(cuda, np.array([[[1, 2], [3, 4]]], np.float32), hf.HF_F32, padding={"width": 4, "height": 4})
    exp = np.zeros((4, 4), complex)
    exp[1:3, 1:3] = [[16, 32], [48, 64]]
    np.testing.assert_allclose(got[0], exp, atol=1e-3)


def test_as_kat_batched_complex_padding(cuda):
    hf, _ = _hf()
    v = np.arange(1, 9, dtype=np.float32)
    x = (v + 1j * v).astype(np.complex64).reshape(2, 2, 2)
    got = _as(cuda, x, hf.HF_CF32, padding={"width": 4, "height": 4})
    exp = O.angular_spectrum(x, LAM, DX, DX, 0.0, padding={"width": 4, "height": 4})
    np.testing.assert_allclose(got, exp, atol=1e-3)


def test_as_kat_all_pass_filter(cuda):
    hf, _ = _hf()
    x = np.zeros((1, 4, 4), np.complex64)
    x[0, 1, 1] = 1
    a = _as(cuda, x, hf.HF_CF32, z=0.01)
    b = _as(cuda, x, hf.HF_CF32, z=0.01, filt={"r_inner": 0, "r_outer": 100, "s_inner": 0, "s_outer": 0})
    np.testing.assert_allclose(a, b, atol=1e-3)


@pytest.mark.parametrize("B,H,W,pad,filt,inplace", [
    (2, 512, 512, None, None, False), (2, 512, 512, None, None, True),
    (1, 480, 480, {"width": 512, "height": 512}, None, False),
    (1, 256, 256, None, {"r_inner": 10, "r_outer": 100, "s_inner": 4, "s_outer": 8}, False),
    (2, 24, 40, {"width": 46, "height": 26}, None, False)])
def test_as_node_vs_oracle(cuda, rng, B, H, W, pad, filt, inplace):
    hf, _ = _hf()
    x = (rng.standard_normal((B, H, W)) + 1j * rng.standard_normal((B, H, W))).astype(np.complex64)
    got = _as(cuda, x, hf.HF_CF32, z=0.3, padding=pad, filt=filt, inplace=inplace)
    exp = O.angular_spectrum(x, LAM, DX, DX, 0.3, filt, pad)
    assert rel(got, exp) < 5e-5


# ---------------------------------------------------------------------------------------------
# a11-a13: Mean / MeanAbs / band moments
# ---------------------------------------------------------------------------------------------
def test_mean_and_mean_abs(cuda, rng):
    import torch
    hf, pl = _hf()
    x = (rng.standard_normal((2, 5, 300)) + 1j * rng.standard_normal((2, 5, 300))).astype(np.complex64)
    dev = torch.from_numpy(x).to(cuda)
    out_c = torch.empty((2, 300), dtype=torch.complex64, device=cuda)
    hf.check(hf.lib().hf_mean_axis(pl._ptr(dev), hf.HF_CF32, 2, 5, 300, pl._ptr(out_c), pl._stream()))
    out_a = torch.empty((2, 300), dtype=torch.float32, device=cuda)
    hf.check(hf.lib().hf_mean_abs_axis(pl._ptr(dev), hf.HF_CF32, 2, 5, 300, pl._ptr(out_a), pl._stream()))
    np.testing.assert_allclose(out_c.cpu().numpy(), x.mean(axis=1), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(out_a.cpu().numpy(), np.abs(x).mean(axis=1), rtol=1e-5)
    u = rng.integers(0, 4096, (3, 7, 11)).astype(np.uint16)
    du = torch.from_numpy(u.view(np.int16)).to(cuda)
    out_u = torch.empty((3, 11), dtype=torch.float32, device=cuda)
    hf.check(hf.lib().hf_mean_axis(pl._ptr(du), hf.HF_U16, 3, 7, 11, pl._ptr(out_u), pl._stream()))
    np.testing.assert_allclose(out_u.cpu().numpy(), u.mean(axis=1), rtol=1e-6)


def test_band_moments(cuda, rng):
    import ctypes as C
    import torch
    hf, pl = _hf()
    nz, P = 10, 5000
    s = (rng.standard_normal((nz, P)) + 1j * rng.standard_normal((nz, P))).astype(np.complex64)
    f = O.freq_weights(32, 6, 16, 37e3)
    out = torch.empty((3, P), dtype=torch.float32, device=cuda)
    fw = (C.c_float * nz)(*f.tolist())
    hf.check(hf.lib().hf_band_moments(pl._ptr(torch.from_numpy(s).to(cuda)), hf.HF_CF32, nz, P, fw, 7,
                                      pl._ptr(out), pl._stream()))
    exp = O.moments_from_magnitude(np.abs(s), f)
    for m in range(3):
        assert rel(out[m].cpu().numpy(), exp[m]) < 1e-6


def test_conversion_kernels(cuda, rng):
    import torch
    hf, pl = _hf()
    x = rng.standard_normal(10000).astype(np.float32)
    dev = torch.from_numpy(x).to(cuda)
    ws = torch.empty(64, dtype=torch.uint8, device=cuda)
    for top, dt, npdt in ((255, hf.HF_U8, np.uint8), (65535, hf.HF_U16, np.uint16)):
        out = torch.empty(10000, dtype=torch.uint8 if top == 255 else torch.int16, device=cuda)
        hf.check(hf.lib().hf_convert(pl._ptr(dev), hf.HF_F32, pl._ptr(out), dt, hf.HF_CONV_SCALED, 10000,
                                     pl._ptr(ws), pl._stream()))
        g = out.cpu().numpy().view(npdt)
        e = O.convert(x, "F32", "U8" if top == 255 else "U16", "Scaled")
        assert np.abs(g.astype(np.int64) - e.astype(np.int64)).max() <= 1
    c = (rng.standard_normal(999) + 1j * rng.standard_normal(999)).astype(np.complex64)
    dc = torch.from_numpy(c).to(cuda)
    for strat, fn in ((hf.HF_CONV_MODULUS, np.abs), (hf.HF_CONV_ARGUMENT, np.angle)):
        out = torch.empty(999, dtype=torch.float32, device=cuda)
        hf.check(hf.lib().hf_convert(pl._ptr(dc), hf.HF_CF32, pl._ptr(out), hf.HF_F32, strat, 999, None,
                                     pl._stream()))
        np.testing.assert_allclose(out.cpu().numpy(), fn(c), rtol=1e-5, atol=1e-6)
    with pytest.raises(hf.HfError):  # no U16 -> F32 Real route (conversion.cu:138-150)
        hf.check(hf.lib().hf_convert(pl._ptr(dc), hf.HF_U16, pl._ptr(dc), hf.HF_F32, hf.HF_CONV_REAL, 4, None,
                                     pl._stream()))
