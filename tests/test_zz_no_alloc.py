"""hf_covariance_noalloc: Gram matrices on the library's fixed device workspace.

Collected last on purpose: it must pass both in a fresh process (where its first call performs
the per-device set-up) and after every other test has used the library.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _frames(cuda, rng, fmt, B, T, P):
    import torch
    import holoflow_b200 as hf
    x = rng.integers(0, 4096, (B, T, P))
    if fmt == "mono12p":
        return torch.from_numpy(O.pack12(x.astype(np.uint16).reshape(-1))).to(cuda), hf.HF_MONO12P, x
    return torch.from_numpy(x.astype(np.uint16).view(np.int16)).to(cuda), hf.HF_U16, x


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,B,T,P,capped", [
    ("mono12p", 2, 64, 256 * 256, False),   # default CTA split fits the 16 MiB workspace
    ("u16", 4, 32, 128 * 128, False),
    ("mono12p", 1, 128, 256 * 256, True),   # default split does not fit: fewer CTAs
    ("u16", 3, 48, 4096, False),            # direct kernel, no workspace
])
def test_noalloc_matches_covariance(cuda, rng, fmt, B, T, P, capped):
    import torch
    from holoflow_b200 import pipeline as pl
    dev, dt, x = _frames(cuda, rng, fmt, B, T, P)
    expect = pl.covariance(dev, dt, B, T, P).cpu().numpy()
    gram = torch.empty((B, T, T), dtype=torch.float64, device=cuda)
    got = []
    for call in range(2):                   # two calls in a row on the same workspace
        gram.fill_(-1.0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        pl.covariance_noalloc(dev, dt, B, T, P, gram)
        torch.cuda.synchronize()
        if call == 1:                       # after the set-up call nothing more is reserved
            assert torch.cuda.mem_get_info()[0] == free0
        got.append(gram.cpu().numpy())
    assert np.array_equal(got[0], got[1])
    for b in range(B):
        X = x[b].astype(np.float64)
        exact = X @ X.T
        scale = np.abs(exact).max()
        assert np.abs(got[1][b] - exact).max() / scale < 2e-7
        assert np.abs(got[1][b] - expect[b]).max() / scale < 2e-7
        assert np.array_equal(got[1][b], got[1][b].T)
    if not capped:                          # same CTA split as hf_covariance: same rounding
        assert np.array_equal(got[1], expect)


@pytest.mark.gpu
def test_noalloc_rejects_batches_beyond_the_workspace(cuda, rng):
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    B, T, P = 300, 128, 64                  # 300 windows x one CTA's partials > 16 MiB
    dev, dt, _ = _frames(cuda, rng, "mono12p", B, T, P)
    gram = torch.zeros((B, T, T), dtype=torch.float64, device=cuda)
    with pytest.raises(hf.HfError) as e:
        pl.covariance_noalloc(dev, dt, B, T, P, gram)
    assert e.value.code == hf.HF_ERR_INVALID and "16 MiB" in str(e.value)
    assert torch.count_nonzero(gram).item() == 0
    # the library stays usable after the rejection
    dev2, dt2, x2 = _frames(cuda, rng, "mono12p", 1, 64, 8192)
    g2 = torch.empty((1, 64, 64), dtype=torch.float64, device=cuda)
    pl.covariance_noalloc(dev2, dt2, 1, 64, 8192, g2)
    X = x2[0].astype(np.float64)
    assert np.abs(g2.cpu().numpy()[0] - X @ X.T).max() / np.abs(X @ X.T).max() < 2e-7


@pytest.mark.gpu
def test_noalloc_accepts_a_two_byte_aligned_base(cuda, rng):
    """A uint16 frame view at an odd element offset is valid input; it takes the direct kernel."""
    import torch
    import holoflow_b200 as hf
    from holoflow_b200 import pipeline as pl
    B, T, P = 2, 64, 8192
    x = rng.integers(0, 4096, (B, T, P))
    host = torch.from_numpy(x.astype(np.uint16).view(np.int16).reshape(-1))
    buf = torch.zeros(host.numel() + 1, dtype=torch.int16, device=cuda)
    buf[1:] = host.to(cuda)
    view = buf[1:]
    assert view.data_ptr() % 4 == 2
    gram = torch.empty((B, T, T), dtype=torch.float64, device=cuda)
    for _ in range(2):
        gram.fill_(-1.0)
        pl.covariance_noalloc(view, hf.HF_U16, B, T, P, gram)
        g = gram.cpu().numpy()
        for b in range(B):
            X = x[b].astype(np.float64)
            assert np.abs(g[b] - X @ X.T).max() / np.abs(X @ X.T).max() < 2e-7
