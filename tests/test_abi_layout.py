"""The ctypes mirrors of the C ABI's structs have the C compiler's layout: every field at the same
offset and every struct the same size as include/holoflow_b200.h gives them.  gcc compiles a
small program against the header on the host; no GPU is needed."""
import ctypes
import pathlib
import shutil
import subprocess

import pytest

import holoflow_b200 as hf

ROOT = pathlib.Path(__file__).resolve().parents[1]

# C struct -> (ctypes class, {ctypes field: C member} where the names differ)
STRUCTS = {
    "hf_desc": (hf.HfDesc, {"lambda_": "lambda"}),
    "hf_ellipse": (hf.HfEllipse, {}),
    "hf_holo_header": (hf.HoloHeader, {}),
    "hf_tdesc": (hf.HfTDesc, {}),
    "hf_multi_schedule": (hf.HfMultiSchedule, {}),
}


def c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "holoflow_b200.h"', "int main(void) {"]
    for cname, (cls, rename) in STRUCTS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            member = rename.get(fname, fname)
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {member}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        s, f, v = line.split()
        table[(s, f)] = int(v)
    return table


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a host C compiler")
def test_ctypes_structs_match_the_header(tmp_path):
    table = c_layout(tmp_path)
    for cname, (cls, _) in STRUCTS.items():
        assert ctypes.sizeof(cls) == table[(cname, "sizeof")], cname
        for fname, _ in cls._fields_:
            assert getattr(cls, fname).offset == table[(cname, fname)], (cname, fname)
