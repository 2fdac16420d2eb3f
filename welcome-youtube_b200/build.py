"""Build libdpd.so (all CUDA sources in csrc/) for sm_100a, in-tree.

    python welcome-youtube_b200/build.py [--force]

The library lands in oercel_b200/libdpd.so next to the Python package that
loads it.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "oercel_b200", "libdpd.so")

OBJ = os.path.join(HERE, "_build")

COMPILE_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "--extended-lambda",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]
LINK_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-shared"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                              + glob.glob(os.path.join(INCLUDE, "*.h")))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in deps())


def _obj(src: str) -> str:
    return os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    """Compile each CUDA source to an object in parallel (a source is rebuilt
    when it, or any header, is newer than its object), then link libdpd.so."""
    if not force and not stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    os.makedirs(OBJ, exist_ok=True)
    headers = [p for p in deps() if not p.endswith(".cu")]
    newest_header = max((os.path.getmtime(p) for p in headers), default=0.0)

    def compile_one(src):
        obj = _obj(src)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= newest_header):
            return
        cmd = [nvcc, *COMPILE_FLAGS, "-I", INCLUDE, "-c", "-o", obj + ".tmp", src]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(obj + ".tmp", obj)

    with ThreadPoolExecutor(max_workers=jobs or min(len(sources()), os.cpu_count() or 4)) as ex:
        list(ex.map(compile_one, sources()))
    tmp = LIB + ".tmp"
    cmd = [nvcc, *LINK_FLAGS, "-o", tmp, *[_obj(s) for s in sources()], "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
