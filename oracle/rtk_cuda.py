"""RTK's own CUDA code, built unchanged from an RTK source tree by
oracle/rtk_cuda/Makefile: the FDK back projector (CUDA_reconstruct_conebeam,
src/rtkCudaFDKBackProjectionImageFilter.cu), the projection weighting
filters and the ramp filter (CUDA_padding, CUDA_fft_convolution) in
oracle/_ref/librtkcudafdk.so; the ray-casting forward projector,
the voxel-based back projector, the Laplacian, TV denoising and the
conjugate-gradient update in oracle/_ref/librtkcudaiter.so.

TEST INFRASTRUCTURE ONLY: the reference's CUDA kernels are timed beside the
product and checked against the FP64 oracle (pins of the half-pixel,
normalisation and weighting conventions, at the precision of their
texture-filtered interpolation where they use textures).  The product never
loads them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "librtkcudafdk.so")
ITER_LIB_PATH = os.path.join(HERE, "_ref", "librtkcudaiter.so")
_lib = None
_ilib = None


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


def iter_available() -> bool:
    return os.path.exists(ITER_LIB_PATH)


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
        L.rtkcuda_fft_ramp.restype = C.c_int
        L.rtkcuda_fft_ramp.argtypes = [I3, C.c_int, C.c_int, F, C.c_int, F, C.c_int, C.c_void_p, C.c_void_p]
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


def fft_ramp(O, proj, params, d_in: int, d_out: int) -> int:
    """RTK's CUDA ramp filter (CudaFFTRampImageFilter, whose GPUGenerateData
    is CudaFFTProjectionsConvolutionImageFilter's) on a whole stack: the
    padded width and height from the oracle's restatement of
    GetPaddedImageRegion, the kernel spectrum from the oracle's restatement of
    FFTRampImageFilter::UpdateFFTProjectionsConvolutionKernel (real: the
    spatial kernel is even; with HannCutFrequencyY the 1-D kernel replicated
    over the padded height times the vertical window, the 2-D kernel) scaled by
    1 / (padded pixel count) as the CUDA filter does, and the mirror weights as
    UpdateTruncationMirrorWeights computes them
    (include/rtkFFTProjectionsConvolutionImageFilter.hxx:345-355, float, from
    the extent floor(t * nu)).  Returns the padded width."""
    nu, nv, n = proj.size
    padded = O.ramp_padded_size(nu, params)
    K = O.ramp_kernel(padded, proj.spacing[0], params)
    if params.hann_cut_y > 0.0:
        H = O.ramp_padded_size_y(nv, params)
        wy = O.ramp_window_y(H, params)
        rows = np.array([wy[min(j, H - j)] for j in range(H)])
        K2 = rows[:, None] * K[None, :]
    else:
        H = nv
        K2 = K[None, :]
    K2 = K2 / (float(padded) * H * n)
    spec = np.zeros(K2.shape + (2,))
    spec[..., 0] = K2
    k, kp = _f(spec)
    ext = int(np.floor(params.truncation_correction * nu))
    i = np.arange(ext + 1, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        w = np.sin((ext - i) * np.pi / (2 * ext - 2)) ** 0.75
    mw, mwp = _f(w)
    _check(lib().rtkcuda_fft_ramp(_i(proj.size), padded, H, kp, K2.shape[0], mwp, ext + 1, C.c_void_p(d_in),
                                  C.c_void_p(d_out)))
    return padded


# ---- librtkcudaiter.so: projectors, Laplacian, TV denoising, CG update


def ilib():
    global _ilib
    if _ilib is None:
        L = C.CDLL(ITER_LIB_PATH)
        I3 = C.POINTER(C.c_int)
        F = C.POINTER(C.c_float)
        V = C.c_void_p
        L.rtkcuda_forward_project.restype = C.c_int
        L.rtkcuda_forward_project.argtypes = [I3, I3, F, F, V, V, V, C.c_float, F, F, F]
        L.rtkcuda_back_project.restype = C.c_int
        L.rtkcuda_back_project.argtypes = [I3, I3, F, V, V, V]
        L.rtkcuda_ray_cast_back_project.restype = C.c_int
        L.rtkcuda_ray_cast_back_project.argtypes = [I3, I3, F, F, V, V, V, C.c_float, F, F, F]
        L.rtkcuda_laplacian.restype = C.c_int
        L.rtkcuda_laplacian.argtypes = [I3, F, V, V]
        L.rtkcuda_total_variation.restype = C.c_int
        L.rtkcuda_total_variation.argtypes = [I3, F, V, V, C.c_float, C.c_float, C.c_int]
        for name in ("rtkcuda_cg_copy", "rtkcuda_cg_subtract"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = [C.c_size_t, V, V]
        L.rtkcuda_cg_update.restype = C.c_int
        L.rtkcuda_cg_update.argtypes = [C.c_size_t, V, V, V, V]
        L.rtkcuda_iter_last_error.restype = C.c_char_p
        _ilib = L
    return _ilib


def _icheck(rc):
    if rc != 0:
        raise RuntimeError("RTK CUDA: " + ilib().rtkcuda_iter_last_error().decode())


def forward_matrices(O, g, vol, proj):
    """What CudaForwardProjectionImageFilter::GPUGenerateData passes for a
    flat panel (include/rtkCudaForwardProjectionImageFilter.hxx:60-167):
    per projection, detector index -> volume texture coordinates (the
    volume's physical-to-index matrix shifted by 0.5 to the texel-corner
    convention, times the oracle's projection-coordinates-to-fixed-system
    matrix and the stack's index-to-physical matrix), the source in the same
    coordinates, the box from the first to the last voxel centre, the spacing
    and the default step (the smallest spacing).  Volume and stack regions
    start at index 0 here."""
    if any(vol.index) or any(proj.index[:2]):
        raise ValueError("regions starting at index 0 only")
    pp2i = np.linalg.inv(O.index_to_physical(vol))
    pp2i[:3, 3] += 0.5
    i2p = O.index_to_physical(proj)
    n = proj.size[2]
    mats = np.zeros((n, 12), dtype=np.float32)
    src = np.zeros((n, 3), dtype=np.float32)
    for s in range(n):
        k = proj.index[2] + s
        mats[s] = (pp2i @ g.proj_coords_to_fixed(k) @ i2p)[:3].reshape(12)
        src[s] = (pp2i @ g.source_position(k))[:3]
    bmin = [0.5, 0.5, 0.5]
    bmax = [0.5 + vol.size[i] - 1.0 for i in range(3)]
    return mats, src, bmin, bmax, list(vol.spacing), float(min(vol.spacing))


def forward_project(O, g, vol, proj, d_vol: int, d_proj_in: int, d_proj_out: int, t_step=None) -> None:
    """RTK's CUDA ray-casting forward projection (kernel_forwardProject:
    trilinear texture samples every t_step mm between the box faces) of the
    FP32 volume at d_vol, added to d_proj_in, into d_proj_out; the filter's
    slab loop over CUDA_forward_project."""
    mats, src, bmin, bmax, sp, step = forward_matrices(O, g, vol, proj)
    m, mp = _f(mats)
    s, sp_ = _f(src)
    a, ap = _f(bmin)
    b, bp = _f(bmax)
    c, cp = _f(sp)
    _icheck(ilib().rtkcuda_forward_project(_i(proj.size), _i(vol.size), mp, sp_, C.c_void_p(d_proj_in),
                                           C.c_void_p(d_proj_out), C.c_void_p(d_vol),
                                           float(step if t_step is None else t_step), ap, bp, cp))


def ray_cast_back_matrices(O, g, vol, proj):
    """What CudaRayCastBackProjectionImageFilter::GPUGenerateData passes for
    a flat panel (src/rtkCudaRayCastBackProjectionImageFilter.cxx:57-156): per
    projection, detector index -> volume index (voxel centres: the volume's
    physical-to-index matrix, the oracle's projection-coordinates-to-fixed-system
    matrix, the stack's index-to-physical matrix), the source in volume
    indices, the box from the first to the last voxel index, the spacing and
    the default step (the smallest spacing).  Regions start at index 0."""
    if any(vol.index) or any(proj.index[:2]):
        raise ValueError("regions starting at index 0 only")
    pp2i = np.linalg.inv(O.index_to_physical(vol))
    i2p = O.index_to_physical(proj)
    n = proj.size[2]
    mats = np.zeros((n, 12), dtype=np.float32)
    src = np.zeros((n, 3), dtype=np.float32)
    for s in range(n):
        k = proj.index[2] + s
        mats[s] = (pp2i @ g.proj_coords_to_fixed(k) @ i2p)[:3].reshape(12)
        src[s] = (pp2i @ g.source_position(k))[:3]
    return mats, src, [0.0, 0.0, 0.0], [vol.size[i] - 1.0 for i in range(3)], list(vol.spacing), \
        float(min(vol.spacing))


def ray_cast_back_project(O, g, vol, proj, d_vol_in: int, d_vol_out: int, d_proj: int, t_step=None) -> None:
    """RTK's CUDA ray-cast back projector (kernel_ray_cast_back_project, the
    adjoint of its ray-casting forward projector: steps of the smallest
    spacing along each ray, trilinear atomic splats) over 16-projection
    slabs."""
    mats, src, bmin, bmax, sp, step = ray_cast_back_matrices(O, g, vol, proj)
    m, mp = _f(mats)
    q, qp = _f(src)
    b0, b1, s0 = _f(bmin), _f(bmax), _f(sp)  # (array, pointer) pairs, alive for the call
    _icheck(ilib().rtkcuda_ray_cast_back_project(_i(proj.size), _i(vol.size), mp, qp, C.c_void_p(d_vol_in),
                                                 C.c_void_p(d_vol_out), C.c_void_p(d_proj),
                                                 float(t_step or step), b0[1], b1[1], s0[1]))


def back_project(O, g, vol, proj, d_vol_in: int, d_vol_out: int, d_proj: int) -> None:
    """RTK's CUDA voxel-based back projection (kernel_backProject: bilinear
    texture reads at each voxel's projection, no distance weight) with the
    filter's matrices (include/rtkCudaBackProjectionImageFilter.hxx:51-134:
    the same texel-centred, rotation-centre-normalised index-to-index
    matrices as the FDK filter's)."""
    m, mp = _f(filter_matrices(O, g, vol, proj))
    _icheck(ilib().rtkcuda_back_project(_i(proj.size), _i(vol.size), mp, C.c_void_p(d_vol_in), C.c_void_p(d_vol_out),
                                        C.c_void_p(d_proj)))


def laplacian(vol, d_in: int, d_out: int) -> None:
    """CUDA_laplacian (src/rtkCudaLaplacianImageFilter.cu): gradient then
    divergence kernels of src/rtkCudaFirstOrderKernels.cu."""
    sp, spp = _f(vol.spacing)
    _icheck(ilib().rtkcuda_laplacian(_i(vol.size), spp, C.c_void_p(d_in), C.c_void_p(d_out)))


def total_variation_denoising(vol, d_in: int, d_out: int, gamma: float, niter: int) -> None:
    """CUDA_total_variation (src/rtkCudaTotalVariationDenoisingBPDQImageFilter.cu)
    on all three dimensions, with beta = 0.9 / 2^3 x the smallest spacing as
    DenoisingBPDQImageFilter::GenerateOutputInformation sets it
    (include/rtkDenoisingBPDQImageFilter.hxx:69-86)."""
    sp, spp = _f(vol.spacing)
    beta = 0.9 / 8.0 * min(vol.spacing)
    _icheck(ilib().rtkcuda_total_variation(_i(vol.size), spp, C.c_void_p(d_in), C.c_void_p(d_out), float(gamma),
                                           float(beta), int(niter)))


def conjugate_gradient(n: int, apply_operator, d_b: int, d_x: int, d_r: int, d_p: int, d_ap: int, niter: int) -> None:
    """CudaConjugateGradientImageFilter::GPUGenerateData
    (include/rtkCudaConjugateGradientImageFilter.hxx:58-105) on FP32 device
    vectors of n elements: x holds X0 on entry and the iterate on return;
    apply_operator(src, dst) computes dst = A src (device pointers) and must
    have finished when it returns (RTK's update runs on the legacy default
    stream)."""
    L = ilib()
    apply_operator(d_x, d_ap)
    _icheck(L.rtkcuda_cg_copy(n, C.c_void_p(d_b), C.c_void_p(d_r)))
    _icheck(L.rtkcuda_cg_subtract(n, C.c_void_p(d_r), C.c_void_p(d_ap)))
    _icheck(L.rtkcuda_cg_copy(n, C.c_void_p(d_r), C.c_void_p(d_p)))
    for _ in range(niter):
        apply_operator(d_p, d_ap)
        _icheck(L.rtkcuda_cg_update(n, C.c_void_p(d_x), C.c_void_p(d_r), C.c_void_p(d_p), C.c_void_p(d_ap)))
