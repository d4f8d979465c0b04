"""RTK's own CUDA FDK back projector (CUDA_reconstruct_conebeam from
src/rtkCudaFDKBackProjectionImageFilter.cu), built from an RTK source tree by
oracle/rtk_cuda/Makefile into oracle/_ref/librtkcudafdk.so.

TEST INFRASTRUCTURE ONLY: the reference's CUDA kernel is timed beside the
product and checked against the FP64 oracle (a pin of the half-pixel,
normalisation and weighting conventions, at the precision of its
texture-filtered interpolation).  The product never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "librtkcudafdk.so")
_lib = None


def build(rtk_src: str | None = None) -> str | None:
    """Builds the library when an RTK source tree is given (or found at the
    default location); returns its path, or None when neither the library nor
    the sources exist."""
    src = rtk_src or os.environ.get("RTK_SRC", "/root/reference")
    if os.path.isdir(os.path.join(src, "src")):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "rtk_cuda"), f"RTK_SRC={src}"], check=True)
    return LIB_PATH if os.path.exists(LIB_PATH) else None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        L.rtkcuda_fdk_backproject.restype = C.c_int
        L.rtkcuda_fdk_backproject.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float),
                                               C.c_void_p, C.c_void_p, C.c_void_p]
        L.rtkcuda_last_error.restype = C.c_char_p
        L.rtkcuda_slab_size.restype = C.c_int
        _lib = L
    return _lib


def filter_matrices(O, g, vol, proj) -> np.ndarray:
    """The float matrices CudaFDKBackProjectionImageFilter::GPUGenerateData
    builds (src/rtkCudaFDKBackProjectionImageFilter.cxx:45-97): RTK's
    index-to-index matrix of each projection (the oracle's restatement of
    GetIndexToIndexProjectionMatrix), corrected for the volume region's index
    and for the stack's index with the 0.5 texel offset of a 2-D texture, and
    normalised by its perspective value at the rotation centre."""
    i2p = O.index_to_physical(vol)
    rot_centre = np.linalg.solve(i2p[:3, :3], -i2p[:3, 3])  # continuous index of the physical origin
    vidx = np.array(vol.index, dtype=np.float64)
    rot_centre = rot_centre - vidx
    mvol = np.eye(4)
    mvol[:3, 3] = vidx
    mproj = np.eye(3)
    mproj[0, 2] = -proj.index[0] + 0.5
    mproj[1, 2] = -proj.index[1] + 0.5
    out = np.zeros((proj.size[2], 12), dtype=np.float32)
    for s in range(proj.size[2]):
        m, _ = O.bp_matrix(g, vol, proj, proj.index[2] + s, False)
        m = mproj @ m @ mvol
        persp = m[2, 3] + m[2, :3] @ rot_centre
        out[s] = (m / persp).reshape(12).astype(np.float32)
    return out


def fdk_backproject(proj_size, vol_size, matrices, d_vol_in: int, d_vol_out: int, d_proj: int) -> None:
    """Runs the filter's slab loop over CUDA_reconstruct_conebeam on device
    pointers (synchronous, on the legacy default stream, as RTK does)."""
    L = lib()
    ps = (C.c_int * 3)(*proj_size)
    vs = (C.c_int * 3)(*vol_size)
    m = np.ascontiguousarray(matrices, dtype=np.float32)
    rc = L.rtkcuda_fdk_backproject(ps, vs, m.ctypes.data_as(C.POINTER(C.c_float)), C.c_void_p(d_vol_in),
                                   C.c_void_p(d_vol_out), C.c_void_p(d_proj))
    if rc != 0:
        raise RuntimeError("RTK CUDA back projection: " + L.rtkcuda_last_error().decode())
