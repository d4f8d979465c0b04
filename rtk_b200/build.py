"""Build librtkb200.so in-tree with nvcc for sm_100a.

``python -m rtk_b200.build`` compiles every CUDA/C++ source under
``rtk_b200/csrc`` into ``rtk_b200/librtkb200.so`` (one shared library, static
CUDA runtime, relocatable device code so kernels share the device status word).
Each source compiles to its own object under ``rtk_b200/_build`` (in parallel,
and again only when it or a header changed); one nvcc call links them.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "librtkb200.so")
OBJ_DIR = os.path.join(PKG, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    csrc = os.path.join(PKG, "csrc")
    return sorted(glob.glob(os.path.join(csrc, "*.cu")) + glob.glob(os.path.join(csrc, "*.cpp")))


def headers():
    return glob.glob(os.path.join(PKG, "csrc", "*.h")) + glob.glob(os.path.join(PKG, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _common(host_cc):
    return [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-rdc=true", "-ccbin", host_cc,
            "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr",
            "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "csrc")]


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    return r.returncode, r.stdout + r.stderr


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    srcs = sources()
    hdr_time = max((os.path.getmtime(h) for h in headers()), default=0.0)
    if os.path.exists(LIB) and not extra:
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in srcs) and hdr_time <= t:
            return LIB
    host_cc = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    os.makedirs(OBJ_DIR, exist_ok=True)
    common = _common(host_cc)
    if extra:
        common[1:1] = extra
    jobs, objs = [], []
    for s in srcs:
        o = os.path.join(OBJ_DIR, os.path.basename(s) + ".o")
        objs.append(o)
        stale = extra or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time)
        if stale:
            jobs.append([*common, "-dc", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for cmd, (rc, out) in zip(jobs, ex.map(_compile, jobs)):
            if verbose:
                print(" ".join(cmd))
                if out:
                    print(out)
            if rc != 0:
                raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out)
    link = [*_common(host_cc), "-shared", "-o", LIB + ".tmp", *objs, "-lcudart_static", "-ldl", "-lrt", "-lpthread",
            "-lz"]
    if verbose:
        print(" ".join(link))
    rc, out = _compile(link)
    if rc != 0:
        raise RuntimeError("nvcc link failed:\n" + out)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None
    print(build(verbose=v or bool(extra), extra=extra))
