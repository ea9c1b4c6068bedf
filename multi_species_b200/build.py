"""Build libfs_b200.so in-tree for sm_100a.

    python -m multi_species_b200.build [--force] [--verbose]

Each source under csrc/ is compiled by nvcc (host C++ through nvcc as well)
with ``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into
``multi_species_b200/libfs_b200.so`` with the CUDA runtime linked statically,
so the library does not depend on whichever libcudart another package in the
same process loaded first.  Objects go to ``multi_species_b200/_build/``;
a source is recompiled when it or any header under csrc/ or include/ is newer
than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libfs_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _defines() -> list:
    """Extra -D flags from FS_B200_DEFINES ("NAME=VALUE NAME2=VALUE2"), for
    building variants (e.g. FS_TILE_SOURCES=512); unset for the default build."""
    return ["-D" + d for d in os.environ.get("FS_B200_DEFINES", "").split()]


def _flags_changed() -> bool:
    stamp = os.path.join(BUILD, "defines.txt")
    now = " ".join(_defines())
    old = open(stamp).read() if os.path.exists(stamp) else ""
    if old != now:
        with open(stamp, "w") as f:
            f.write(now)
        return True
    return False


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, force: bool, verbose: bool, ptxas_v: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= _headers_mtime()):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + _defines() + ["-c", src, "-o", obj]
    if src.endswith(".cu") and ptxas_v:
        cmd += ["-Xptxas", "-v"]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "cu"] + ARCH + COMMON + _defines() + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed on {src}")
    if ptxas_v and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    force = _flags_changed() or force
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose, ptxas_v), srcs))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_v))


if __name__ == "__main__":
    main()
