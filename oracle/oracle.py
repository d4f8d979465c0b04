"""ctypes loader for the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker.  The product package
``rtk_b200`` never imports this module.

Every array is float64 and C-contiguous; images use ITK's row-major x-fastest
layout (volume [z][y][x], projection stack [projection][v][u]).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


class OrcImage(C.Structure):
    _fields_ = [
        ("size", C.c_int * 3),
        ("index", C.c_int * 3),
        ("origin", C.c_double * 3),
        ("spacing", C.c_double * 3),
        ("direction", C.c_double * 9),
    ]


class OrcRampParams(C.Structure):
    _fields_ = [
        ("hann_cut", C.c_double),
        ("cosine_cut", C.c_double),
        ("hamming", C.c_double),
        ("ramlak_cut", C.c_double),
        ("shepplogan_cut", C.c_double),
        ("truncation_correction", C.c_double),
        ("greatest_prime_factor", C.c_int),
        ("zero_pad_factor", C.c_int),
        ("hann_cut_y", C.c_double),
        ("zero_pad_factor_y", C.c_int),
    ]


def build() -> str:
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        D = C.POINTER(C.c_double)
        F = C.POINTER(C.c_float)
        I = C.POINTER(C.c_int)
        G = C.c_void_p
        IM = C.POINTER(OrcImage)
        sig = {
            "orc_geometry_new": (G, []),
            "orc_geometry_free": (None, [G]),
            "orc_geometry_add_projection": (C.c_int, [G] + [C.c_double] * 9),
            "orc_geometry_add_projection_rad": (C.c_int, [G] + [C.c_double] * 9),
            "orc_geometry_size": (C.c_int, [G]),
            "orc_geometry_matrix": (None, [G, C.c_int, D]),
            "orc_geometry_source_position": (None, [G, C.c_int, D]),
            "orc_geometry_proj_coords_to_fixed": (None, [G, C.c_int, D]),
            "orc_geometry_parameters": (None, [G, C.c_int, D]),
            "orc_geometry_source_angles": (None, [G, D]),
            "orc_geometry_gantry_angles": (None, [G, D]),
            "orc_geometry_tilt_angles": (None, [G, D]),
            "orc_geometry_angular_gaps": (None, [G, D, D]),
            "orc_geometry_angular_gaps_with_next": (None, [G, D, D]),
            "orc_geometry_to_untilted": (C.c_double, [G, C.c_int, C.c_double]),
            "orc_index_to_physical": (None, [IM, D]),
            "orc_physical_to_index": (None, [IM, D]),
            "orc_bp_matrix": (C.c_int, [G, IM, IM, C.c_int, C.c_int, D]),
            "orc_bp_project": (C.c_int, [G, IM, IM, C.c_int, C.c_int, D, D]),
            "orc_backproject": (None, [G, IM, IM, D, D, D, C.c_int, C.c_int]),
            "orc_joseph_forward": (None, [G, IM, D, IM, D, D, C.c_int]),
            "orc_joseph_back": (None, [G, IM, D, D, IM, D]),
            "orc_joseph_sample_count": (C.c_double, [G, IM, IM, C.c_int]),
            "orc_fdk_weight": (None, [G, IM, D, D]),
            "orc_parker_weight": (C.c_int, [G, IM, C.c_double, D, D]),
            "orc_displaced_detector_region": (C.c_int, [G, IM, C.c_int, I, I, D, D]),
            "orc_displaced_detector": (C.c_int, [G, IM, C.c_int, D, D]),
            "orc_ramp_padded_size": (C.c_int, [C.c_int, C.POINTER(OrcRampParams)]),
            "orc_ramp_padded_size_y": (C.c_int, [C.c_int, C.POINTER(OrcRampParams)]),
            "orc_ramp_window_y": (None, [C.c_int, C.POINTER(OrcRampParams), D]),
            "orc_ramp_kernel": (None, [C.c_int, C.c_double, C.POINTER(OrcRampParams), D]),
            "orc_ramp_filter": (None, [IM, C.POINTER(OrcRampParams), D, D, C.c_int]),
            "orc_cg_joseph": (None, [G, IM, IM, D, D, D, C.c_double, C.c_double, C.c_int, D, D, C.c_int]),
            "orc_parker_params": (C.c_int, [G, C.c_double, D, D]),
            "orc_cg": (None, [G, IM, IM, D, D, D, C.c_double, C.c_double, C.c_int, D, D, C.c_int, C.c_int]),
            "orc_joseph_back_mt": (None, [G, IM, D, D, IM, D, C.c_int]),
            "orc_laplacian": (None, [IM, D, D]),
            "orc_ray_box": (None, [G, IM, IM, D, C.c_int]),
            "orc_sart": (None, [G, IM, IM, D, D, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double,
                                C.POINTER(C.c_int), C.c_int]),
            "orc_de_pierro": (None, [IM, D, D, D, C.c_double, D]),
            "orc_ray_box_corners": (None, [G, IM, D, D, D, C.c_int]),
            "orc_i0_estimation": (None, [C.POINTER(C.c_ushort), C.c_long, C.c_int, C.c_uint, D]),
            "orc_raw_to_attenuation": (None, [C.POINTER(C.c_ushort), C.c_long, C.c_double, C.c_double, C.POINTER(C.c_float)]),
            "orc_geometry_set_radius_cylindrical": (None, [G, C.c_double]),
            "orc_tv_denoising_bpdq": (None, [IM, D, D, C.c_double, C.c_int, C.POINTER(C.c_int)]),
            "orc_total_variation": (C.c_double, [IM, D]),
            "orc_regularized_cg": (None, [G, IM, IM, D, D, D, D, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                          C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_double, C.c_int]),
            "orc_osem": (None, [G, IM, IM, D, D, C.c_int, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int), C.c_int]),
            "orc_project_ellipsoids": (None, [G, IM, C.c_int, D, D, C.c_int]),
            "orc_draw_ellipsoids": (None, [IM, C.c_int, D, D, C.c_int]),
            "orc_fdk_backproject_f32_rtk": (C.c_int, [G, IM, IM, F, F, C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def nthreads() -> int:
    return max(1, os.cpu_count() or 1)


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def image(size, spacing=(1.0, 1.0, 1.0), origin=None, index=(0, 0, 0), direction=None) -> OrcImage:
    """ITK image description; origin defaults to centring the image on 0."""
    im = OrcImage()
    for a in range(3):
        im.size[a] = int(size[a])
        im.index[a] = int(index[a])
        im.spacing[a] = float(spacing[a])
        im.origin[a] = float(origin[a]) if origin is not None else -0.5 * (size[a] - 1) * spacing[a]
    d = np.eye(3) if direction is None else np.asarray(direction, dtype=np.float64).reshape(3, 3)
    for q in range(9):
        im.direction[q] = float(d.flat[q])
    return im


def shape_of(im: OrcImage):
    return (im.size[2], im.size[1], im.size[0])


def index_to_physical(im: OrcImage):
    m = np.zeros(16)
    lib().orc_index_to_physical(C.byref(im), _d(m))
    return m.reshape(4, 4)


class Geometry:
    """FP64 restatement of rtk::ThreeDCircularProjectionGeometry."""

    def __init__(self):
        self._g = lib().orc_geometry_new()

    def __del__(self):
        try:
            if self._g:
                lib().orc_geometry_free(self._g)
                self._g = None
        except Exception:
            pass

    def set_radius_cylindrical(self, radius):
        lib().orc_geometry_set_radius_cylindrical(self._g, float(radius))

    def add_projection(self, sid, sdd, gantry_deg, pox=0.0, poy=0.0, oop_deg=0.0, ip_deg=0.0, sox=0.0, soy=0.0):
        rc = lib().orc_geometry_add_projection(self._g, sid, sdd, gantry_deg, pox, poy, oop_deg, ip_deg, sox, soy)
        if rc != 0:
            raise ValueError("cannot mix parallel and divergent projections")

    def __len__(self):
        return lib().orc_geometry_size(self._g)

    def matrix(self, i):
        m = np.zeros(12)
        lib().orc_geometry_matrix(self._g, i, _d(m))
        return m.reshape(3, 4)

    def source_position(self, i):
        s = np.zeros(4)
        lib().orc_geometry_source_position(self._g, i, _d(s))
        return s

    def parameters(self, i):
        """(sid, sdd, gantry, pox, poy, oop, ip, sox, soy, source angle) of projection i."""
        p = np.zeros(10)
        lib().orc_geometry_parameters(self._g, i, _d(p))
        return p

    def proj_coords_to_fixed(self, i):
        m = np.zeros(16)
        lib().orc_geometry_proj_coords_to_fixed(self._g, i, _d(m))
        return m.reshape(4, 4)

    def _vec(self, fn):
        out = np.zeros(len(self))
        fn(self._g, _d(out))
        return out

    def source_angles(self):
        return self._vec(lib().orc_geometry_source_angles)

    def gantry_angles(self):
        return self._vec(lib().orc_geometry_gantry_angles)

    def tilt_angles(self):
        return self._vec(lib().orc_geometry_tilt_angles)

    def angular_gaps(self, angles):
        a = np.ascontiguousarray(angles, dtype=np.float64)
        out = np.zeros(len(self))
        lib().orc_geometry_angular_gaps(self._g, _d(a), _d(out))
        return out

    def to_untilted(self, i, x):
        return lib().orc_geometry_to_untilted(self._g, i, x)


def bp_matrix(g: Geometry, vol: OrcImage, proj: OrcImage, i: int, fdk: bool):
    m = np.zeros(12)
    mode = lib().orc_bp_matrix(g._g, C.byref(vol), C.byref(proj), i, int(fdk), _d(m))
    return m.reshape(3, 4), mode


def bp_project(g: Geometry, vol: OrcImage, proj: OrcImage, k: int, fdk: bool, physical):
    """(u, v, weight) of a physical point in projection k by the oracle's own
    ray/detector-plane derivation, and RTK's path mode."""
    x = np.ascontiguousarray(physical, dtype=np.float64)
    out = np.zeros(3)
    mode = lib().orc_bp_project(g._g, C.byref(vol), C.byref(proj), k, int(fdk), _d(x), _d(out))
    return out, mode


def backproject(g, vol, proj, proj_data, vol_in=None, fdk=True, threads=None):
    p = np.ascontiguousarray(proj_data, dtype=np.float64)
    vin = np.zeros(shape_of(vol)) if vol_in is None else np.ascontiguousarray(vol_in, dtype=np.float64)
    out = np.empty(shape_of(vol))
    lib().orc_backproject(g._g, C.byref(vol), C.byref(proj), _d(p), _d(vin), _d(out), int(fdk),
                          threads or nthreads())
    return out


def joseph_forward(g, vol, vol_data, proj, proj_in=None, threads=None):
    v = np.ascontiguousarray(vol_data, dtype=np.float64)
    pin = np.zeros(shape_of(proj)) if proj_in is None else np.ascontiguousarray(proj_in, dtype=np.float64)
    out = np.empty(shape_of(proj))
    lib().orc_joseph_forward(g._g, C.byref(vol), _d(v), C.byref(proj), _d(pin), _d(out), threads or nthreads())
    return out


def joseph_back(g, vol, proj, proj_data, vol_in=None, threads=1):
    """RTK's single-threaded Joseph back projection (threads > 1: the same sum
    split over threads by projection)."""
    p = np.ascontiguousarray(proj_data, dtype=np.float64)
    vin = np.zeros(shape_of(vol)) if vol_in is None else np.ascontiguousarray(vol_in, dtype=np.float64)
    out = np.empty(shape_of(vol))
    if threads == 1:
        lib().orc_joseph_back(g._g, C.byref(vol), _d(vin), _d(out), C.byref(proj), _d(p))
    else:
        lib().orc_joseph_back_mt(g._g, C.byref(vol), _d(vin), _d(out), C.byref(proj), _d(p), threads or nthreads())
    return out


def joseph_sample_count(g, vol, proj, threads=None) -> float:
    return lib().orc_joseph_sample_count(g._g, C.byref(vol), C.byref(proj), threads or nthreads())


def fdk_weight(g, proj, data):
    d = np.ascontiguousarray(data, dtype=np.float64)
    out = np.empty_like(d)
    lib().orc_fdk_weight(g._g, C.byref(proj), _d(d), _d(out))
    return out


def parker_weight(g, proj, data, threshold=np.pi / 9):
    d = np.ascontiguousarray(data, dtype=np.float64)
    out = np.empty_like(d)
    short = lib().orc_parker_weight(g._g, C.byref(proj), threshold, _d(d), _d(out))
    return out, bool(short)


def parker_params(g, threshold=np.pi / 9):
    """(short scan?, delta, first angle) of ParkerShortScanImageFilter."""
    d, f = C.c_double(), C.c_double()
    short = lib().orc_parker_params(g._g, threshold, C.byref(d), C.byref(f))
    return bool(short), d.value, f.value


def displaced_detector_region(g, proj, pad=True):
    i0, s0 = C.c_int(), C.c_int()
    inf, sup = C.c_double(), C.c_double()
    st = lib().orc_displaced_detector_region(g._g, C.byref(proj), int(pad), C.byref(i0), C.byref(s0),
                                             C.byref(inf), C.byref(sup))
    return st, i0.value, s0.value, inf.value, sup.value


def displaced_detector(g, proj, data, pad=True):
    st, i0, s0, _, _ = displaced_detector_region(g, proj, pad)
    if st < 0:
        raise ValueError("Cannot account for detector displacement larger than 50% of panel size.")
    d = np.ascontiguousarray(data, dtype=np.float64)
    out = np.zeros((proj.size[2], proj.size[1], s0))
    lib().orc_displaced_detector(g._g, C.byref(proj), int(pad), _d(d), _d(out))
    return out, i0, s0


def ramp_params(hann=0.0, cosine=0.0, hamming=0.0, ramlak=0.0, shepplogan=0.0, truncation=0.0, gpf=2, pad=2,
                hann_y=0.0, pad_y=2):
    p = OrcRampParams()
    p.hann_cut, p.cosine_cut, p.hamming = hann, cosine, hamming
    p.ramlak_cut, p.shepplogan_cut, p.truncation_correction = ramlak, shepplogan, truncation
    p.greatest_prime_factor, p.zero_pad_factor = gpf, pad
    p.hann_cut_y, p.zero_pad_factor_y = hann_y, pad_y
    return p


def ramp_padded_size(nu, params):
    return lib().orc_ramp_padded_size(nu, C.byref(params))


def ramp_padded_size_y(nv, params):
    return lib().orc_ramp_padded_size_y(nv, C.byref(params))


def ramp_window_y(padded_y, params):
    w = np.zeros(padded_y // 2 + 1)
    lib().orc_ramp_window_y(padded_y, C.byref(params), _d(w))
    return w


def ramp_kernel(padded, spacing, params):
    k = np.zeros(padded // 2 + 1)
    lib().orc_ramp_kernel(padded, spacing, C.byref(params), _d(k))
    return k


def ramp_filter(proj, data, params, threads=None):
    d = np.ascontiguousarray(data, dtype=np.float64)
    out = np.empty_like(d)
    lib().orc_ramp_filter(C.byref(proj), C.byref(params), _d(d), _d(out), threads or nthreads())
    return out


def laplacian(vol, x):
    d = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(d)
    lib().orc_laplacian(C.byref(vol), _d(d), _d(out))
    return out


def ray_box(g, vol, proj, threads=None):
    out = np.empty(shape_of(proj))
    lib().orc_ray_box(g._g, C.byref(vol), C.byref(proj), _d(out), threads or nthreads())
    return out


def sart(g, vol, proj, proj_data, niter, order, x0=None, lam=0.3, positivity=False, subset=1,
         displaced_detector=True, threshold=1e-5, threads=None):
    p = np.ascontiguousarray(proj_data, dtype=np.float64)
    x = np.zeros(shape_of(vol)) if x0 is None else np.array(x0, dtype=np.float64, copy=True, order="C")
    o = np.ascontiguousarray(order, dtype=np.int32)
    lib().orc_sart(g._g, C.byref(vol), C.byref(proj), _d(p), _d(x), int(niter), float(lam), int(positivity),
                   int(subset), int(displaced_detector), float(threshold),
                   o.ctypes.data_as(C.POINTER(C.c_int)), threads or nthreads())
    return x


def de_pierro(vol, xk, update, norm, beta):
    """DePierroRegularizationImageFilter; norm None = a volume of ones."""
    a = np.ascontiguousarray(xk, dtype=np.float64)
    u = np.ascontiguousarray(update, dtype=np.float64)
    n = None if norm is None else np.ascontiguousarray(norm, dtype=np.float64)
    out = np.empty(shape_of(vol))
    lib().orc_de_pierro(C.byref(vol), _d(a), _d(u), _d(n), float(beta), _d(out))
    return out


def osem(g, vol, proj, proj_data, niter, order, x0, subset=1, beta=0.0, joseph_bp=False, threads=None):
    """OSEMConeBeamReconstructionFilter (Joseph forward projector; voxel-based or Joseph back projector)."""
    p = np.ascontiguousarray(proj_data, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True, order="C")
    o = np.ascontiguousarray(order, dtype=np.int32)
    lib().orc_osem(g._g, C.byref(vol), C.byref(proj), _d(p), _d(x), int(niter), int(subset), float(beta),
                   int(joseph_bp), o.ctypes.data_as(C.POINTER(C.c_int)), threads or nthreads())
    return x


def _dims(dims):
    return (C.c_int * 3)(*[int(bool(d)) for d in dims])


def tv_denoising_bpdq(vol, f, gamma, niter, dims=(True, True, True)):
    """TotalVariationDenoisingBPDQImageFilter."""
    a = np.ascontiguousarray(f, dtype=np.float64)
    out = np.empty(shape_of(vol))
    lib().orc_tv_denoising_bpdq(C.byref(vol), _d(a), _d(out), float(gamma), int(niter), _dims(dims))
    return out


def total_variation(vol, x):
    """TotalVariationImageFilter."""
    return lib().orc_total_variation(C.byref(vol), _d(np.ascontiguousarray(x, dtype=np.float64)))


def regularized_cg(g, vol, proj, proj_data, x0, main_iterations=10, cg_iterations=4, weights=None, tikhonov=0.0,
                   gamma=0.0, positivity=True, tv=True, gamma_tv=5e-5, tv_iterations=10, tv_dims=(True, True, True),
                   soft_threshold=False, soft_threshold_value=1e-3, mask=None, threads=None):
    """RegularizedConjugateGradientConeBeamReconstructionFilter (Joseph pair)."""
    p = np.ascontiguousarray(proj_data, dtype=np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True, order="C")
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
    lib().orc_regularized_cg(g._g, C.byref(vol), C.byref(proj), _d(p), _d(w), _d(m), _d(x), int(main_iterations),
                             int(cg_iterations), float(tikhonov), float(gamma), int(positivity), int(tv),
                             float(gamma_tv), int(tv_iterations), _dims(tv_dims), int(soft_threshold),
                             float(soft_threshold_value), threads or nthreads())
    return x


def i0_estimation(raw, bit_shift=2, dyn_threshold=20):
    """I0EstimationProjectionFilter on a uint16 array: dict of i0, i0_fwhm, imin, imax, low_bound, high_bound."""
    r = np.ascontiguousarray(raw, dtype=np.uint16)
    out = np.zeros(6)
    lib().orc_i0_estimation(r.ctypes.data_as(C.POINTER(C.c_ushort)), r.size, int(bit_shift), int(dyn_threshold),
                            _d(out))
    return dict(zip(("i0", "i0_fwhm", "imin", "imax", "low_bound", "high_bound"), out.tolist()))


def raw_to_attenuation(raw, i0=65535.0, idark=0.0):
    """LUTbasedVariableI0RawToAttenuationImageFilter (float32 out)."""
    r = np.ascontiguousarray(raw, dtype=np.uint16)
    out = np.empty(r.shape, dtype=np.float32)
    lib().orc_raw_to_attenuation(r.ctypes.data_as(C.POINTER(C.c_ushort)), r.size, float(i0), float(idark),
                                 out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def ray_box_corners(g, proj, bmin, bmax, threads=None):
    """RayBoxIntersectionImageFilter with SetBoxMin / SetBoxMax."""
    out = np.empty(shape_of(proj))
    lo = np.ascontiguousarray(bmin, dtype=np.float64)
    hi = np.ascontiguousarray(bmax, dtype=np.float64)
    lib().orc_ray_box_corners(g._g, C.byref(proj), _d(lo), _d(hi), _d(out), threads or nthreads())
    return out


def iterative_fdk(g, vol, proj, proj_data, x0, niter=3, lam=0.3, positivity=False, ramp=None, displaced=True,
                  short_scan=True, threshold=np.pi / 9):
    """IterativeFDKConeBeamReconstructionFilter::GenerateData
    (include/rtkIterativeFDKConeBeamReconstructionFilter.hxx:171-218), composed from the oracle's
    filters: x += FDK(p), then niter - 1 times x += FDK(lambda (p - JosephFP(x)) / raybox) with the
    ray box from the volume's origin to origin + size x spacing (0 below 1e-5); FDK = displaced
    detector (padded on the truncated side), Parker, FDK weights, ramp, FDK back projection."""
    params = ramp or ramp_params()

    def fdk(q):
        qo = proj
        if displaced:
            q, i0, s0 = displaced_detector(g, proj, q)
            qo = image((s0, proj.size[1], proj.size[2]), tuple(proj.spacing), origin=tuple(proj.origin),
                       index=(i0, proj.index[1], proj.index[2]), direction=np.asarray(proj.direction).reshape(3, 3))
        if short_scan:
            q, _ = parker_weight(g, qo, q, threshold)
        q = fdk_weight(g, qo, q)
        q = ramp_filter(qo, q, params)
        return backproject(g, vol, qo, q, fdk=True)

    p = np.ascontiguousarray(proj_data, dtype=np.float64)
    origin = np.asarray(vol.origin)
    rb = ray_box_corners(g, proj, origin, origin + np.asarray(vol.size) * np.asarray(vol.spacing))
    x = np.array(x0, dtype=np.float64, copy=True) + fdk(p)
    if positivity:
        x = np.maximum(x, 0.0)
    for _ in range(1, niter):
        fp = joseph_forward(g, vol, x, proj)
        with np.errstate(divide="ignore", invalid="ignore"):
            e = np.where(rb < 1e-5, 0.0, lam * (p - fp) / rb)
        x = x + fdk(e)
        if positivity:
            x = np.maximum(x, 0.0)
    return x


def water_precorrection(data, coefficients):
    """WaterPrecorrectionImageFilter::DynamicThreadedGenerateData
    (include/rtkWaterPrecorrectionImageFilter.hxx:14-62) on float32 data: with at least 3
    coefficients out = float(c0 + c1 v), then out = float(out + c_j v^j) with v^j in float; with
    two (not the identity) float(c0 + c1 v); one non-zero: c0; otherwise the input (in place)."""
    v = np.asarray(data, dtype=np.float32)
    c = [float(x) for x in coefficients]
    if len(c) >= 3:
        out = (c[0] + c[1] * v.astype(np.float64)).astype(np.float32)
        bpow = (v * v).astype(np.float32)
        for cj in c[2:]:
            out = (out.astype(np.float64) + cj * bpow.astype(np.float64)).astype(np.float32)
            bpow = (bpow * v).astype(np.float32)
        return out
    if len(c) == 2 and (c[0] != 0.0 or c[1] != 1.0):
        return (c[0] + c[1] * v.astype(np.float64)).astype(np.float32)
    if len(c) == 1 and c[0] != 0.0:
        return np.full(v.shape, np.float32(c[0]))
    return v.copy()


def cg_joseph(g, vol, proj, proj_data, niter, x0=None, weights=None, tikhonov=0.0, gamma=0.0, mask=None,
              threads=None, backprojector="joseph"):
    """RTK's CG reconstruction with the Joseph forward projector and the
    chosen back projector ("joseph", or "voxel" for the voxel-based one)."""
    p = np.ascontiguousarray(proj_data, dtype=np.float64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
    x = np.zeros(shape_of(vol)) if x0 is None else np.array(x0, dtype=np.float64, copy=True, order="C")
    res = np.zeros(niter + 1)
    bp = {"joseph": 0, "voxel": 1}[backprojector]
    lib().orc_cg(g._g, C.byref(vol), C.byref(proj), _d(p), _d(w), _d(m), tikhonov, gamma, niter, _d(x), _d(res), bp,
                 threads or nthreads())
    return x, res


def project_ellipsoids(g, proj, ell, threads=None):
    e = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 16)
    out = np.empty(shape_of(proj))
    lib().orc_project_ellipsoids(g._g, C.byref(proj), e.shape[0], _d(e), _d(out), threads or nthreads())
    return out


def draw_ellipsoids(vol, ell, threads=None):
    e = np.ascontiguousarray(ell, dtype=np.float64).reshape(-1, 16)
    out = np.empty(shape_of(vol))
    lib().orc_draw_ellipsoids(C.byref(vol), e.shape[0], _d(e), _d(out), threads or nthreads())
    return out


def fdk_backproject_f32_rtk(g, vol, proj, proj_data_f32, vol_inout_f32, threads=None):
    """RTK's CPU FDK backprojector with RTK's data types (the timed CPU baseline)."""
    p = np.ascontiguousarray(proj_data_f32, dtype=np.float32)
    assert vol_inout_f32.dtype == np.float32 and vol_inout_f32.flags.c_contiguous
    rc = lib().orc_fdk_backproject_f32_rtk(g._g, C.byref(vol), C.byref(proj),
                                           p.ctypes.data_as(C.POINTER(C.c_float)),
                                           vol_inout_f32.ctypes.data_as(C.POINTER(C.c_float)),
                                           threads or nthreads())
    if rc != 0:
        raise RuntimeError("CPU baseline needs the optimised-Y path (circular geometry)")


# ---- field of view and the offset-field-of-view displaced detector ----------


def fov_radius(g, proj, kind):
    """rtk::FieldOfViewImageFilter::ComputeFOVRadius
    (include/rtkFieldOfViewImageFilter.hxx:41-187): per projection, the lines
    from the source through the corner pixels of the first (corners 0, 1) and
    last (2, 3) detector columns, in the rotation plane (x, z), bound
    half-planes a x + b z <= c, oriented so that the other side's corners lie
    inside (:110-131); the largest disc (x, z, r) at distance r inside every
    half-plane of the kind (0 RADIUSINF: first column, 1 RADIUSSUP: last, 2
    RADIUSBOTH) maximises r.  RTK hands the programme to lp_solve; the oracle
    solves the same programme with scipy's HiGHS (geometries without
    collimation jaws: AddCollimationConstraints adds nothing then).  Returns
    (x, z, r), or None where lp_solve reports no solution."""
    from scipy.optimize import linprog

    i2p = index_to_physical(proj)
    rows, rhs = [], []
    for k in range(len(g)):
        s = g.source_position(k)
        p2f = g.proj_coords_to_fixed(k)
        a, b, c, cor = [], [], [], []
        for q in range(4):
            iu = proj.index[0] + (q // 2) * (proj.size[0] - 1)
            iv = proj.index[1] + (q % 2) * (proj.size[1] - 1)
            pos = p2f @ (i2p @ np.array([iu, iv, k, 1.0]))
            cor.append((pos[0], pos[2]))
            a.append(pos[2] - s[2])
            b.append(s[0] - pos[0])
            c.append(s[0] * pos[2] - pos[0] * s[2])
        if a[0] * cor[2][0] + b[0] * cor[2][1] >= c[0] and a[1] * cor[3][0] + b[1] * cor[3][1] >= c[1]:
            flip = (0, 1)
        elif a[2] * cor[0][0] + b[2] * cor[0][1] >= c[2] and a[3] * cor[1][0] + b[3] * cor[1][1] >= c[3]:
            flip = (2, 3)
        else:
            raise ValueError("Error computing the FOV, unhandled detector rotation.")
        for q in flip:
            a[q], b[q], c[q] = -a[q], -b[q], -c[q]
        for q in range(4):
            if (q < 2 and kind != 1) or (q >= 2 and kind != 0):
                rows.append([a[q], b[q], np.hypot(a[q], b[q])])
                rhs.append(c[q])
    res = linprog([0.0, 0.0, -1.0], A_ub=np.array(rows), b_ub=np.array(rhs),
                  bounds=[(None, None), (None, None), (0, None)], method="highs")
    if res.status != 0:
        return None
    return float(res.x[0]), float(res.x[1]), float(res.x[2])


def displaced_detector_offset_fov_region(g, proj):
    """DisplacedDetectorForOffsetFieldOfViewImageFilter::GenerateOutputInformation
    (include/rtkDisplacedDetectorForOffsetFieldOfViewImageFilter.hxx:36-118):
    returns (weighted, out index0, out size0, disc (x, z, r), shift)."""
    fov = fov_radius(g, proj, 2)
    if fov is None:
        raise ValueError("Cannot account for too large detector displacements")
    inf, sup = fov_radius(g, proj, 0), fov_radius(g, proj, 1)
    ri = inf[2] if inf else float("nan")
    rs = sup[2] if sup else float("nan")
    nu = proj.size[0]
    if 200.0 * abs(ri - rs) / (ri + rs) < 10.0:
        return False, proj.index[0], nu, fov, 0
    if rs > ri:
        return True, proj.index[0] - nu, 2 * nu, fov, nu
    return True, proj.index[0], 2 * nu, fov, 0


def displaced_detector_offset_fov(g, proj, data):
    """DisplacedDetectorForOffsetFieldOfViewImageFilter::DynamicThreadedGenerateData
    (:122-270) on a whole stack: returns (out, out index0, out size0)."""
    weighted, i0, s0, (cx, cz, R), shift = displaced_detector_offset_fov_region(g, proj)
    d = np.asarray(data, dtype=np.float64)
    if not weighted:
        return d.copy(), i0, s0
    n, nv, nu = d.shape
    out = np.zeros((n, nv, s0))
    for s in range(n):
        k = proj.index[2] + s
        sp = g.source_position(k)
        opp = -1.0 / (sp[0] * sp[0] + sp[2] * sp[2])
        scx, scz = cx - sp[0], cz - sp[2]
        inv = 1.0 / np.sqrt(scx * scx + scz * scz)
        ang = np.arctan2(scz * inv, scx * inv) - np.arctan2(sp[2] * opp, sp[0] * opp)
        if ang > np.pi:
            ang -= 2 * np.pi
        if ang < -np.pi:
            ang += 2 * np.pi
        t2 = np.arcsin(R / np.sqrt((cx - sp[0]) ** 2 + (cz - sp[2]) ** 2))
        t1 = -t2 + ang
        t2 = t2 + ang
        prm = g.parameters(k)
        sid = np.sqrt(prm[0] ** 2 + prm[7] ** 2)
        l1, l2 = np.tan(t1) * sid, np.tan(t2) * sid
        invsid = 1.0 / sid
        pod = np.pi / 2 * np.sqrt(scx * scx + scz * scz) / R
        w = np.empty(nu)
        for i in range(nu):
            x = proj.origin[0] + proj.spacing[0] * (proj.index[0] + i)
            l = g.to_untilted(k, x)
            f = np.sin(np.sin(np.arctan(l * invsid) - ang) * pod)
            if shift:
                w[i] = 0.0 if l <= l1 else (2.0 if l >= l2 else f + 1.0)
            else:
                w[i] = 2.0 if l <= l1 else (0.0 if l >= l2 else 1.0 - f)
        out[s, :, shift:shift + nu] = d[s] * w[None, :]
    return out, i0, s0
