"""Build librtkb200.so in-tree with nvcc for sm_100a.

``python -m rtk_b200.build`` compiles every CUDA/C++ source under
``rtk_b200/csrc`` into ``rtk_b200/librtkb200.so`` (one shared library, static
CUDA runtime, relocatable device code so kernels share the device status word).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "librtkb200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    csrc = os.path.join(PKG, "csrc")
    return sorted(glob.glob(os.path.join(csrc, "*.cu")) + glob.glob(os.path.join(csrc, "*.cpp")))


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    srcs = sources()
    deps = srcs + glob.glob(os.path.join(PKG, "csrc", "*.h")) + glob.glob(os.path.join(PKG, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    if os.path.exists(LIB) and not extra:
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    host_cc = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-rdc=true", "-ccbin", host_cc,
           "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc"),
           "-shared", "-o", LIB + ".tmp", *srcs, "-lcudart_static", "-ldl", "-lrt", "-lpthread", "-lz"]
    if extra:
        cmd[1:1] = extra
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None
    print(build(verbose=v or bool(extra), extra=extra))
