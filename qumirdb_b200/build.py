"""Builds libqdb_gpu.so (the device kernels and the C ABI) for sm_100a.

Sources under qumirdb_b200/csrc are compiled by nvcc in parallel into
qumirdb_b200/_build/ and linked into qumirdb_b200/libqdb_gpu.so, in-tree, so
the library travels with the repository.  A source is rebuilt when it or any
header is newer than its object.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libqdb_gpu.so"
ROOT = HERE.parent

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-lineinfo", f"-I{ROOT / 'include'}"]


def _sources() -> list[Path]:
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp"))


def _headers() -> list[Path]:
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".h", ".cuh")) + [ROOT / "include" / "qdb_gpu.h"]


def _compile(src: Path) -> Path:
    obj = BUILD / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [NVCC, *COMMON, *ARCH, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [NVCC, *COMMON, "-x", "cu", *ARCH, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(_compile, srcs))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *map(str, objs), "-lcudart_static",
           "-lpthread", "-ldl", "-lrt"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    try:
        build(verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
