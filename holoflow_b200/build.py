"""Builds the in-tree shared library holoflow_b200/_lib/libholoflow_b200.so for sm_100a.

Every CUDA / C++ source under csrc/ is compiled by nvcc (device code for
`-gencode arch=compute_100a,code=sm_100a` only) and linked into one shared object that exports
the C ABI declared in include/holoflow_b200.h.  Objects are rebuilt only when a source or header
is newer than the object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = ROOT / "_build"
LIB = HERE / "_lib" / "libholoflow_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _json_include() -> list[str]:
    """nlohmann/json (header-only; the reference's settings type) from the Python environment."""
    import site
    roots = list(site.getsitepackages()) + [site.getusersitepackages()]
    for r in roots:
        cand = pathlib.Path(r) / "include" / "cudnn_frontend" / "thirdparty"
        if (cand / "nlohmann" / "json.hpp").exists():
            return ["-I", str(cand)]
    return []


def _flags() -> list[str]:
    return ARCH + ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC,-O3",
                   "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC)] + _json_include()


def _sources() -> list[pathlib.Path]:
    return sorted(list(CSRC.glob("*.cu")) + list((CSRC / "host").glob("*.cc")))


def _headers() -> list[pathlib.Path]:
    return (list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.inc")) + list((ROOT / "include").rglob("*.h*"))
            + list((CSRC / "host").glob("*.hh")))


def _compile(src: pathlib.Path, obj: pathlib.Path, verbose: bool) -> None:
    cmd = [_nvcc(), *_flags(), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cc":
        cmd = [_nvcc(), *_flags(), "-x", "cu", "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> pathlib.Path:
    subprocess.run([sys.executable, str(HERE / "gen_twiddles.py")], check=True)
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    todo, objs = [], []
    for src in _sources():
        obj = BUILD / (src.stem + ("_cc" if src.suffix == ".cc" else "") + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            todo.append((src, obj))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda so: _compile(so[0], so[1], verbose), todo))
    if todo or not LIB.exists():
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
