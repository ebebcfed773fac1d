"""Writes csrc/twiddles.inc: float32 tables exp(-2 pi i k / N) for the in-register DFT sizes.

Values are evaluated in float64 (cos/sin of 2*pi*k/N) and rounded once to float32.  The build
step runs this before nvcc; the generated file is also committed so a bare `nvcc -c` works.
"""
import math
import pathlib

SIZES = [4, 8, 16, 24, 32, 48, 64]


def fmt(v: float) -> str:
    import struct
    f = struct.unpack("f", struct.pack("f", v))[0]
    return repr(f) + "f"


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
    out.write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main(pathlib.Path(__file__).resolve().parent / "csrc" / "twiddles.inc")
