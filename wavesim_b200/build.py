"""Build libwavesim_b200.so in-tree for sm_100a:  python wavesim_b200/build.py

(Run as a script: importing the package itself needs the built library.)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include")]

TARGETS = {
    "libwavesim_b200.so": ["ws_mbs.cu", "ws_noalloc.cu", "ws_net.cu", "ws_setup.cu"],
}


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "wavesim_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=True):
    for out, srcs in TARGETS.items():
        dst = os.path.join(HERE, out)
        if not force and not _stale(dst, srcs):
            continue
        cmd = [NVCC] + ARCH + FLAGS + ["-o", dst] + [os.path.join(CSRC, s) for s in srcs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
