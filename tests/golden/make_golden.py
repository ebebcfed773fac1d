"""Generates tests/golden/holonp_ops.npz from the reference's own NumPy test oracle.

The reference checks its holonp operators against test/holonp/python/oracle.py (driven by
manifest files from the C++ tests).  This script imports that module from a checkout of the
reference, calls its operator implementations directly on seeded inputs shaped like the
Doppler path's tensors (frames x pixels, band bins, moment weights), and stores inputs, settings
and outputs.  The tests then pin this repository's oracle and CUDA kernels to those outputs
without needing the reference at run time.

    python tests/golden/make_golden.py path/to/reference
"""
import importlib.util
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def load_reference_oracle(root: pathlib.Path):
    path = root / "test" / "holonp" / "python" / "oracle.py"
    spec = importlib.util.spec_from_file_location("holonp_reference_oracle", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cases(rng):
    f32 = lambda *s: rng.integers(0, 4096, s).astype(np.float32)                  # 12-bit samples
    c64 = lambda *s: (rng.standard_normal(s) + 1j * rng.standard_normal(s)).astype(np.complex64)
    u16 = lambda *s: rng.integers(0, 4096, s).astype(np.uint16)
    out = []
    # temporal transforms along the frame axis of a [batch, T, H, W] window stack
    for norm in ("backward", "forward", "ortho"):
        out.append((f"fft_f32_axis1_{norm}", "fft", [f32(2, 32, 6, 10)], {"axis": 1, "norm": norm}))
    out.append(("fft_cf32_axis1", "fft", [c64(2, 16, 4, 8)], {"axis": 1, "norm": "backward"}))
    out.append(("fft_u16_axis1", "fft", [u16(1, 32, 4, 8)], {"axis": 1, "norm": "backward"}))
    out.append(("rfft_f32_axis1_t64", "rfft", [f32(2, 64, 4, 8)], {"axis": 1, "norm": "backward"}))
    # band selection of the one-sided spectrum: bins 4..31 of T = 64
    out.append(("slice_band_4_32", "slice", [c64(2, 33, 4, 8)],
                {"slices": [{}, {"start": 4, "stop": 32}]}))
    # moment reductions over the band axis (axis -3, keepdims) and |.|
    out.append(("mean_f32_axis_m3", "mean", [rng.random((1, 28, 8, 8)).astype(np.float32)],
                {"axis": -3, "keepdims": True}))
    out.append(("mean_cf32_axis_m3", "mean", [c64(1, 10, 8, 8)], {"axis": -3, "keepdims": True}))
    out.append(("mean_f32_axis0", "mean", [rng.random((1, 16, 16)).astype(np.float32)],
                {"axis": 0, "keepdims": False}))
    out.append(("abs_cf32", "abs", [c64(1, 28, 8, 8)], {}))
    # frequency weights f_k = f0 + k df (df = 37 kHz / T, bins 4..31 of T = 64, and 6..15 of T = 32)
    df64, df32 = 37e3 / 64, 37e3 / 32
    out.append(("arange_band_t64", "arange", [], {"start": 4 * df64, "stop": 32 * df64, "step": df64,
                                                  "dtype": "F32"}))
    out.append(("arange_band_t32", "arange", [], {"start": 6 * df32, "stop": 16 * df32, "step": df32,
                                                  "dtype": "F32"}))
    out.append(("multiply_weights", "multiply",
                [rng.random((1, 28, 8, 8)).astype(np.float32), rng.random((1, 28, 1, 1)).astype(np.float32)],
                {}))
    # spatial transforms: 2D FFT of a plane stack and the display shift
    out.append(("fft2_cf32", "fft2", [c64(2, 16, 16)], {"axes": [-2, -1], "norm": "backward"}))
    out.append(("fftshift_f32", "fftshift", [rng.random((3, 8, 12)).astype(np.float32)], {"axes": [-2, -1]}))
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py path/to/reference")
    root = pathlib.Path(sys.argv[1])
    ref = load_reference_oracle(root)
    rng = np.random.default_rng(20260)
    store = {}
    index = {}
    for name, op, inputs, settings in cases(rng):
        outs = ref._DISPATCH[op](inputs, settings)
        index[name] = {"op": op, "settings": settings, "ninputs": len(inputs), "noutputs": len(outs)}
        for i, a in enumerate(inputs):
            store[f"{name}__in{i}"] = a
        for i, a in enumerate(outs):
            store[f"{name}__out{i}"] = np.ascontiguousarray(a)
    store["__index__"] = np.frombuffer(json.dumps(index, sort_keys=True).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / "holonp_ops.npz", **store)
    print(f"wrote {len(index)} cases to {HERE / 'holonp_ops.npz'}")


if __name__ == "__main__":
    main()
