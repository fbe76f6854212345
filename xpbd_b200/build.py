"""Build the engine library ``libxpbd_b200.so`` in-tree with nvcc for sm_100a.

    python -m xpbd_b200.build            # incremental
    python -m xpbd_b200.build --force

The library is plain C ABI (``include/xpbd_b200.h``); nothing here depends on
PyTorch.  Flags: ``-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo``,
``--fmad=false`` (no contraction of multiply-add, so fp32 results round like a
plain evaluation of the same expressions), C++17, static CUDA runtime.
"""

from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libxpbd_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
         "-shared", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    cmd = [NVCC] + ARCH + FLAGS + list(extra) + ["-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp"] + sources()
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed to build libxpbd_b200.so")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose or a.ptxas_info, extra=extra))
