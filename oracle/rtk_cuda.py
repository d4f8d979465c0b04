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
        I3 = C.POINTER(C.c_int)
        F = C.POINTER(C.c_float)
        L.rtkcuda_fdk_weight.restype = C.c_int
        L.rtkcuda_fdk_weight.argtypes = [I3, I3, C.c_void_p, C.c_void_p, F, F, F, F]
        L.rtkcuda_parker_weight.restype = C.c_int
        L.rtkcuda_parker_weight.argtypes = [I3, I3, C.c_void_p, C.c_void_p, F, C.c_float, C.c_float, C.c_float,
                                            C.c_float, C.c_float]
        L.rtkcuda_displaced_weight.restype = C.c_int
        L.rtkcuda_displaced_weight.argtypes = [I3, I3, I3, I3, C.c_void_p, C.c_void_p, F, C.c_float, C.c_int,
                                               C.c_float, C.c_float, C.c_float]
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


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def _i(v):
    return (C.c_int * len(v))(*[int(x) for x in v])


def _check(rc):
    if rc != 0:
        raise RuntimeError("RTK CUDA filter: " + lib().rtkcuda_last_error().decode())


# geometry parameter columns of the oracle's Geometry.parameters
_SID, _SDD, _GA, _POX, _POY, _OOP, _IP, _SOX, _SOY = range(9)


def fdk_weight(O, g, proj, d_in: int, d_out: int) -> None:
    """RTK's CUDA FDK weighting (kernel_weight_projection) on a whole stack,
    with the per-projection table CudaFDKWeightProjectionFilter::GPUGenerateData
    builds (src/rtkCudaFDKWeightProjectionFilter.cxx:31-110): the angular gaps
    of the source angles times the ramp factor (0.5 for a parallel beam,
    |sdd| / (2 sid^2) |source position| otherwise), and the tilt angles."""
    gaps = g.angular_gaps(g.source_angles())
    tilt = g.tilt_angles()
    k0, n = proj.index[2], proj.size[2]
    tab = np.zeros((n, 7))
    for s in range(n):
        k = k0 + s
        p = g.parameters(k)
        fac = gaps[k]
        if p[_SDD] == 0.0:
            fac *= 0.5
        else:
            sp = g.source_position(k)[:3]
            fac *= abs(p[_SDD]) / (2.0 * p[_SID] * p[_SID]) * np.linalg.norm(sp)
        tab[s] = (p[_SDD], p[_SID], p[_POX], p[_POY], p[_SOY], fac, tilt[k])
    t, tp = _f(tab)
    D = np.asarray(proj.direction).reshape(3, 3)
    o, op = _f([proj.origin[0], proj.origin[1]])
    r, rp = _f([D[0, 0] * proj.spacing[0], D[1, 0] * proj.spacing[0]])
    c, cp = _f([D[0, 1] * proj.spacing[1], D[1, 1] * proj.spacing[1]])
    _check(lib().rtkcuda_fdk_weight(_i(proj.index[:2]), _i(proj.size), C.c_void_p(d_in), C.c_void_p(d_out), tp, op,
                                    rp, cp))


def parker_weight(O, g, proj, d_in: int, d_out: int, threshold=np.pi / 9) -> bool:
    """RTK's CUDA Parker short-scan weighting (kernel_parker_weight) with the
    table and angles CudaParkerShortScanImageFilter::GPUGenerateData passes
    (src/rtkCudaParkerShortScanImageFilter.cxx:68-108); delta and the first
    angle from the oracle's restatement of the filter's short-scan detection.
    Returns False (nothing done) for a full scan."""
    short, delta, first = O.parker_params(g, threshold)
    if not short:
        return False
    k0, n = proj.index[2], proj.size[2]
    ga = g.gantry_angles()
    tab = np.zeros((n, 5))
    for s in range(n):
        p = g.parameters(k0 + s)
        tab[s] = (p[_SDD], p[_SOX], p[_POX], p[_SID], ga[k0 + s])
    t, tp = _f(tab)
    D = np.asarray(proj.direction).reshape(3, 3)
    _check(lib().rtkcuda_parker_weight(_i(proj.index[:2]), _i(proj.size), C.c_void_p(d_in), C.c_void_p(d_out), tp,
                                       delta, first, proj.origin[0], D[0, 0] * proj.spacing[0],
                                       D[0, 1] * proj.spacing[1]))
    return True


def displaced_weight(O, g, proj, d_in: int, d_out: int, pad=True):
    """RTK's CUDA displaced-detector weighting (kernel_displaced_weight) with
    the table, corners and regions CudaDisplacedDetectorImageFilter::GPUGenerateData
    passes (src/rtkCudaDisplacedDetectorImageFilter.cxx:30-140); the output
    region (padded on the truncated side) and the corners from the oracle's
    restatement of the filter's GenerateOutputInformation.  Returns the output
    region's (index0, size0); d_out must hold that many columns."""
    st, i0, s0, inf, sup = O.displaced_detector_region(g, proj, pad)
    if st <= 0:
        raise ValueError("no displaced-detector weighting for this geometry")
    k0, n = proj.index[2], proj.size[2]
    tab = np.zeros((n, 4))
    for s in range(n):
        p = g.parameters(k0 + s)
        tab[s] = (p[_SDD], p[_SOX], p[_POX], p[_SID])
    t, tp = _f(tab)
    D = np.asarray(proj.direction).reshape(3, 3)
    theta = min(-inf, sup)
    _check(lib().rtkcuda_displaced_weight(_i(proj.index), _i(proj.size), _i((i0, proj.index[1], proj.index[2])),
                                          _i((s0, proj.size[1], proj.size[2])), C.c_void_p(d_in), C.c_void_p(d_out), tp,
                                          theta, int(sup + inf > 0.0), proj.origin[0], D[0, 0] * proj.spacing[0],
                                          D[0, 1] * proj.spacing[1]))
    return i0, s0
