"""Writes csrc/twiddles.inc: float32 tables exp(-2 pi i k / N) for the in-register DFT sizes.

Values are evaluated in float64 (cos/sin of 2*pi*k/N) and rounded once to float32.  The build
step runs this before nvcc; the generated file is also committed so a bare `nvcc -c` works.

c_twtN holds each twiddle w = c + i s in "tangent" form (m, t), so that a butterfly a +- b w
costs six fused multiply-adds: w = m (1 + i t) with m = c, t = s/c where |c| >= |s|, and
w = m (t + i) with m = s, t = c/s otherwise (|t| <= 1 in both).  The form is chosen by
near_real(k, N), which the CUDA side evaluates the same way at compile time.
"""
import math
import pathlib

SIZES = [4, 8, 16, 24, 32, 48, 64]


def fmt(v: float) -> str:
    import struct
    f = struct.unpack("f", struct.pack("f", v))[0]
    return repr(f) + "f"


def near_real(k: int, n: int) -> bool:
    """|cos(2 pi k/n)| >= |sin(2 pi k/n)|: the angle lies within 45 degrees of the real axis."""
    r = k % (n // 2)
    return 8 * r <= n or 8 * r >= 3 * n


def main(out: pathlib.Path) -> None:
    lines = ["// Generated by holoflow_b200/gen_twiddles.py: exp(-2 pi i k/N), float32.",
             "#pragma once", ""]
    for n in SIZES:
        vals = []
        for k in range(n):
            a = -2.0 * math.pi * k / n
            c, s = math.cos(a), math.sin(a)
            # exact values where they are known
            if k * 4 % n == 0:
                q = (k * 4 // n) % 4
                c, s = [(1.0, 0.0), (0.0, -1.0), (-1.0, 0.0), (0.0, 1.0)][q]
            vals.append("{%s, %s}" % (fmt(c), fmt(s)))
        lines.append("static __constant__ float2 c_tw%d[%d] = {%s};" % (n, n, ", ".join(vals)))
        tvals = []
        for k in range(n):
            a = -2.0 * math.pi * k / n
            c, s = math.cos(a), math.sin(a)
            if k * 4 % n == 0:  # trivial twiddles are never read from this table
                tvals.append("{0.0f, 0.0f}")
            elif near_real(k, n):
                tvals.append("{%s, %s}" % (fmt(c), fmt(s / c)))
            else:
                tvals.append("{%s, %s}" % (fmt(s), fmt(c / s)))
        lines.append("static __constant__ float2 c_twt%d[%d] = {%s};" % (n, n, ", ".join(tvals)))
    text = "\n".join(lines) + "\n"
    if not out.exists() or out.read_text() != text:  # keep the mtime (and the build) when unchanged
        out.write_text(text)


if __name__ == "__main__":
    main(pathlib.Path(__file__).resolve().parent / "csrc" / "twiddles.inc")
