"""Build libhom3_b200.so in-tree for sm_100a (nvcc; no JIT, no torch extension cache).

    python -m hom3_b200.build [--force] [-v]

Each source is compiled to its own object under hom3_b200/_build/ (in
parallel; a source is recompiled when it or a header it includes changed),
then the objects are linked into hom3_b200/_lib/libhom3_b200.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
SRC = [os.path.join(CSRC, f) for f in ("h3c_solver.cu", "h3c_stage_halo.cu", "h3c_stage_cns.cu", "h3c_stage_warp.cu",
                                       "h3c_rates.cu", "h3c_noalloc.cu", "grid_build.cpp", "grid_build_device.cu",
                                       "vtk_writer.cpp")]
OBJ_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "_lib", "libhom3_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "128,177"]
_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def includes(path: str, seen=None) -> set:
    """The quoted includes of `path`, recursively (the files a change to which
    requires recompiling it)."""
    seen = set() if seen is None else seen
    try:
        text = open(path).read()
    except OSError:
        return seen
    for inc in _INCLUDE.findall(text):
        p = os.path.normpath(os.path.join(os.path.dirname(path), inc))
        if p not in seen and os.path.exists(p):
            seen.add(p)
            includes(p, seen)
    return seen


def obj_of(src: str) -> str:
    return os.path.join(OBJ_DIR, os.path.basename(src) + ".o")


def stale(src: str) -> bool:
    o = obj_of(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return any(os.path.getmtime(p) > t for p in [src, __file__] + sorted(includes(src)))


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return not any(stale(s) for s in SRC) and all(os.path.getmtime(obj_of(s)) <= t for s in SRC)


def _compile(src: str, nvcc: str, verbose: bool) -> None:
    cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose and src.endswith(".cu") else []) + \
        ["-c", "-o", obj_of(src), src]
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    todo = [s for s in SRC if force or stale(s)]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_compile, s, nvcc, verbose) for s in todo]:
            f.result()
    subprocess.run([nvcc] + ARCH + ["-shared", "-o", OUT] + [obj_of(s) for s in SRC], check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
