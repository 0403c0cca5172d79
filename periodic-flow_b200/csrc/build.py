"""Build libpfb200.so (the C-ABI library) for sm_100a with nvcc.

    python periodic-flow_b200/csrc/build.py [--force] [-j N]

Objects go to _build/ at the repository root; the library is written into
the package (periodic-flow_b200/periodicflow/_lib/) so it travels with the
source tree.  Rebuilds only what changed (sources and headers by mtime).
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
BUILD = os.path.join(ROOT, "_build")
LIBDIR = os.path.join(PKG, "periodicflow", "_lib")
LIB = os.path.join(LIBDIR, "libpfb200.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-I" + os.path.join(ROOT, "include")]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def _deps(dfile):
    """Files listed in an nvcc -MD dependency file (None when missing or when a
    listed file no longer exists, which forces a rebuild)."""
    try:
        text = open(dfile).read()
    except OSError:
        return None
    body = text.split(":", 1)[1] if ":" in text else ""
    files = [t for t in body.replace("\\\n", " ").split() if t != "\\"]
    if not files or not all(os.path.exists(f) for f in files):
        return None
    return files


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(HERE, "*.cu")))
    headers = sorted(glob.glob(os.path.join(HERE, "*.cuh")) + glob.glob(os.path.join(HERE, "*.h"))
                     + glob.glob(os.path.join(ROOT, "include", "*.h")))
    hdr_time = _newest(headers) if headers else 0.0
    objs = []
    todo = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        deps = _deps(obj[:-2] + ".d")
        # headers this object was built from (all headers when unknown)
        dep_time = _newest(deps) if deps is not None else hdr_time
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(
                os.path.getmtime(src), dep_time):
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        cmd = [NVCC] + ARCH + FLAGS + ["-MD", "-MF", obj[:-2] + ".d", "-c", src, "-o", obj]
        start = time.time()
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose and r.stderr.strip():
            sys.stderr.write(r.stderr)
        # stamp the object with the compile's start: a source or header
        # edited while it compiled is newer, so the next build redoes it
        os.utime(obj, (start, start))
        return obj

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(compile_one, todo))
    if force or todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
