"""Build libfsd.so in-tree for sm_100a.

Every CUDA and C++ source under fsd_b200/csrc is compiled with nvcc
(-gencode arch=compute_100a,code=sm_100a -lineinfo) into _build/, then linked
into fsd_b200/libfsd.so with the static CUDA runtime.  Rebuilds only what
changed (source or header newer than its object).

Usage:  python -m fsd_b200.build   (or python fsd_b200/build.py)
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libfsd.so"
RESTABLE = PKG / "data" / "resistance_table.bin"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def common_flags() -> list[str]:
    return ARCH + [
        "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
        f"-I{ROOT / 'include'}", f"-I{CSRC}",
        f'-DFSD_RESTABLE_PATH="{RESTABLE}"',
    ]


def needs_build(src: Path, obj: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, RESTABLE, Path(__file__), *headers])


def compile_one(src: Path, headers: list[Path], verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not needs_build(src, obj, headers):
        return obj
    cmd = [nvcc(), *common_flags(), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd[1:1] = ["-x", "c++"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])
    headers = sorted([*CSRC.glob("*.h"), *CSRC.glob("*.cuh"), ROOT / "include" / "fsd.h"])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, headers, verbose), srcs))
    if LIB.exists() and all(LIB.stat().st_mtime >= o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs), "-lquadmath", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
