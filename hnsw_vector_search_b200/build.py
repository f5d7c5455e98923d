"""Builds libvdx_b200.so in-tree: the host library (C++20, g++) and the sm_100a kernels (nvcc).

    python -m hnsw_vector_search_b200.build [--force] [--jobs N]

Every CUDA file is compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a) with
-lineinfo; host files with -ffp-contract=off so that no compiler contraction changes how a
distance rounds. Objects go to _build/ next to this file; the shared library next to the
package's __init__.py, where the Python loader and the tests find it. Rebuilds only what is older
than its sources (headers included).
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
BUILD = PKG / "_build"
LIB = PKG / "libvdx_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("VDX_CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = [f"-I{PKG / 'host' / 'include'}", f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc'}"]
CXXFLAGS = ["-std=c++20", "-O3", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra",
            "-DNDEBUG", "-I/usr/local/cuda/include"]
NVFLAGS = ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
           "-ffp-contract=off", "-fmad=false", "--expt-relaxed-constexpr", "-DNDEBUG"]


def sources() -> list[Path]:
    return sorted((PKG / "host" / "src").glob("*.cpp")) + sorted((PKG / "csrc").glob("*.cu"))


def headers() -> list[Path]:
    found = list((PKG / "host").rglob("*.hpp")) + list((PKG / "csrc").glob("*.cuh"))
    return found + list((ROOT / "include").glob("*.h"))


def compile_one(src: Path, force: bool) -> Path:
    obj = BUILD / (src.stem + (".cu.o" if src.suffix == ".cu" else ".o"))
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in headers()])
    if not force and obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    if src.suffix == ".cu":
        cmd = [NVCC, *ARCH, *NVFLAGS, *INCLUDES, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [CXX, *CXXFLAGS, *INCLUDES, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{' '.join(cmd)}\n{res.stdout}{res.stderr}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as pool:
        objs = list(pool.map(lambda s: compile_one(s, force), srcs))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
               "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"linking failed:\n{' '.join(cmd)}\n{res.stdout}{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    args = ap.parse_args()
    try:
        build(force=args.force, jobs=args.jobs, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)


if __name__ == "__main__":
    main()
