"""Build libwavesim_b200.so in-tree for sm_100a:  python wavesim_b200/build.py

Each CUDA source compiles to its own object (in parallel, under _build/),
then nvcc links them into the shared library.  (Run as a script: importing the
package itself needs the built library.)
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(ROOT, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]

TARGETS = {
    "libwavesim_b200.so": ["ws_mbs.cu", "ws_noalloc.cu", "ws_net.cu", "ws_setup.cu"],
}


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", f)
                                                                  for f in os.listdir(os.path.join(ROOT, "include"))]


def _newer(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=True):
    os.makedirs(OBJ, exist_ok=True)
    deps = _deps()
    for out, srcs in TARGETS.items():
        dst = os.path.join(HERE, out)
        objs = [os.path.join(OBJ, os.path.splitext(s)[0] + ".o") for s in srcs]
        jobs = [[NVCC] + ARCH + CFLAGS + ["-c", "-o", o, os.path.join(CSRC, s)]
                for s, o in zip(srcs, objs) if force or _newer(o, deps)]
        if jobs:
            with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
                list(ex.map(lambda c: _run(c, verbose), jobs))
        if force or jobs or _newer(dst, objs):
            _run([NVCC] + ARCH + ["-shared", "-o", dst] + objs, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
