"""Functional entry points over the C ABI on torch CUDA tensors.

Each function takes float32, C-contiguous CUDA tensors (ITK layout, shape
z, y, x), enqueues the kernels on the current torch stream (or ``stream``) and
returns without synchronising.  Errors raise ``RtkbError``.
"""
from __future__ import annotations

import ctypes as C
import json
import os

from ._capi import check, load
from .image import shape_of


def _torch():
    import torch

    return torch


def _ptr(t):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a CUDA tensor (there is no CPU path)")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError("expected a contiguous float32 tensor")
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    torch = _torch()
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def _check_shape(t, desc, what):
    if tuple(t.shape) != shape_of(desc):
        raise ValueError(f"{what}: shape {tuple(t.shape)} does not match description {shape_of(desc)}")


def _ptr_bf16(t):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a CUDA tensor (there is no CPU path)")
    if t.dtype != torch.bfloat16 or not t.is_contiguous():
        raise TypeError("expected a contiguous bfloat16 tensor")
    return C.c_void_p(t.data_ptr())


def _backproject(fn, geometry, vol_desc, proj_desc, proj, vol_in, out, stream, fn_bf16=None):
    """Backprojection from a float32 stack, or from a bfloat16 stack (BF16
    storage variant) when proj.dtype is torch.bfloat16."""
    torch = _torch()
    _check_shape(proj, proj_desc, "projections")
    _check_shape(vol_in, vol_desc, "volume")
    if out is None:
        out = torch.empty_like(vol_in)
    _check_shape(out, vol_desc, "output")
    if proj.dtype == torch.bfloat16:
        if fn_bf16 is None:
            raise TypeError("this projector has no bfloat16 variant")
        fn, pp = fn_bf16, _ptr_bf16(proj)
    else:
        pp = _ptr(proj)
    check(fn(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), pp, _ptr(vol_in), _ptr(out), _stream(stream)))
    return out


def to_bf16(x, out=None, stream=None):
    """bfloat16 copy of a float32 CUDA tensor (round to nearest even), by the
    library's own kernel."""
    torch = _torch()
    if out is None:
        out = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device)
    if out.shape != x.shape:
        raise ValueError("shape mismatch")
    check(load().rtkb_convert_to_bf16(_ptr(x), _ptr_bf16(out), x.numel(), _stream(stream)))
    return out


def fdk_backproject(geometry, vol_desc, proj_desc, proj, vol_in, out=None, stream=None):
    """rtk::FDKBackProjectionImageFilter: out = vol_in + FDK backprojection
    (proj float32, or bfloat16 for the BF16 storage variant)."""
    L = load()
    return _backproject(L.rtkb_fdk_backproject, geometry, vol_desc, proj_desc, proj, vol_in, out, stream,
                        L.rtkb_fdk_backproject_bf16)


def voxel_backproject(geometry, vol_desc, proj_desc, proj, vol_in, out=None, stream=None):
    """rtk::BackProjectionImageFilter (voxel-based): out = vol_in + backprojection
    (proj float32, or bfloat16 for the BF16 storage variant)."""
    L = load()
    return _backproject(L.rtkb_voxel_backproject, geometry, vol_desc, proj_desc, proj, vol_in, out, stream,
                        L.rtkb_voxel_backproject_bf16)


def joseph_forward_project(geometry, vol_desc, proj_desc, vol, proj_in, out=None, stream=None):
    """rtk::JosephForwardProjectionImageFilter: out = proj_in + Joseph line integrals of vol."""
    torch = _torch()
    _check_shape(vol, vol_desc, "volume")
    _check_shape(proj_in, proj_desc, "projections")
    if out is None:
        out = torch.empty_like(proj_in)
    _check_shape(out, proj_desc, "output")
    check(load().rtkb_joseph_forward_project(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), _ptr(vol),
                                             _ptr(proj_in), _ptr(out), _stream(stream)))
    return out


def joseph_back_project(geometry, vol_desc, proj_desc, proj, vol_in, out=None, stream=None):
    """rtk::JosephBackProjectionImageFilter: out = vol_in + Joseph backprojection of proj."""
    return _backproject(load().rtkb_joseph_back_project, geometry, vol_desc, proj_desc, proj, vol_in, out, stream)


def joseph_sample_count(geometry, vol_desc, proj_desc, stream=None) -> float:
    """Bilinear samples one Joseph forward projection takes (synchronises)."""
    n = C.c_double()
    check(load().rtkb_joseph_sample_count(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), C.byref(n),
                                          _stream(stream)))
    return n.value


def ramp_params(hann=0.0, cosine=0.0, hamming=0.0, ramlak=0.0, shepplogan=0.0, truncation=0.0, gpf=2, pad=2,
                hann_y=0.0, pad_y=2):
    """rtkb_ramp_params: RTK's FFTRampImageFilter windows (HannCutFrequency,
    CosineCutFrequency, HammingFrequency, RamLakCutFrequency,
    SheppLoganCutFrequency; HannCutFrequencyY as hann_y), TruncationCorrection,
    GreatestPrimeFactor and ZeroPadFactors (pad, pad_y)."""
    from ._capi import RampParams

    p = RampParams()
    p.hann_cut, p.cosine_cut, p.hamming = hann, cosine, hamming
    p.ramlak_cut, p.shepplogan_cut, p.truncation_correction = ramlak, shepplogan, truncation
    p.greatest_prime_factor, p.zero_pad_factor = gpf, pad
    p.hann_cut_y, p.zero_pad_factor_y = hann_y, pad_y
    return p


def _unary(fn, desc, inp, out, out_shape=None):
    torch = _torch()
    _check_shape(inp, desc, "projections")
    if out is None:
        out = torch.empty(out_shape or tuple(inp.shape), device=inp.device, dtype=torch.float32)
    return out


def fdk_weight(geometry, proj_desc, proj, out=None, stream=None):
    """rtk::FDKWeightProjectionFilter."""
    out = _unary(None, proj_desc, proj, out)
    check(load().rtkb_fdk_weight(geometry.handle, C.byref(proj_desc), _ptr(proj), _ptr(out), _stream(stream)))
    return out


def parker_short_scan(geometry, proj_desc, proj, threshold=3.141592653589793 / 9, out=None, stream=None):
    """rtk::ParkerShortScanImageFilter; returns (out, is_short_scan)."""
    out = _unary(None, proj_desc, proj, out)
    short = C.c_int(0)
    check(load().rtkb_parker_short_scan(geometry.handle, C.byref(proj_desc), threshold, _ptr(proj), _ptr(out),
                                        _stream(stream), C.byref(short)))
    return out, bool(short.value)


def displaced_detector_region(geometry, proj_desc, pad=True):
    from ._capi import ImageDesc

    out = ImageDesc()
    w = C.c_int(0)
    check(load().rtkb_displaced_detector_region(geometry.handle, C.byref(proj_desc), int(pad), C.byref(out),
                                                C.byref(w)))
    return out, bool(w.value)


def displaced_detector(geometry, proj_desc, proj, pad=True, stream=None, out=None):
    """rtk::DisplacedDetectorImageFilter; returns (out, out_desc)."""
    od, _ = displaced_detector_region(geometry, proj_desc, pad)
    out = _unary(None, proj_desc, proj, out, shape_of(od))
    check(load().rtkb_displaced_detector(geometry.handle, C.byref(proj_desc), int(pad), _ptr(proj), _ptr(out),
                                         _stream(stream)))
    return out, od


def displaced_detector_offset_fov_region(geometry, proj_desc):
    """Output image of rtk::DisplacedDetectorForOffsetFieldOfViewImageFilter
    and whether it weights: (out_desc, weighted)."""
    from ._capi import ImageDesc

    out = ImageDesc()
    w = C.c_int(0)
    check(load().rtkb_displaced_detector_offset_fov_region(geometry.handle, C.byref(proj_desc), C.byref(out),
                                                           C.byref(w)))
    return out, bool(w.value)


def displaced_detector_offset_fov(geometry, proj_desc, proj, stream=None, out=None):
    """rtk::DisplacedDetectorForOffsetFieldOfViewImageFilter (the displaced-detector
    weighting RTK's CPU rtkfdk chains: padding and weights from the stack's
    field of view); returns (out, out_desc)."""
    od, _ = displaced_detector_offset_fov_region(geometry, proj_desc)
    out = _unary(None, proj_desc, proj, out, shape_of(od))
    check(load().rtkb_displaced_detector_offset_fov(geometry.handle, C.byref(proj_desc), _ptr(proj), _ptr(out),
                                                    _stream(stream)))
    return out, od


FOV_RADIUS_INF, FOV_RADIUS_SUP, FOV_RADIUS_BOTH = 0, 1, 2


def field_of_view_radius(geometry, proj_desc, kind=FOV_RADIUS_BOTH):
    """rtk::FieldOfViewImageFilter::ComputeFOVRadius (host only): (x, z, r) of
    the largest disc in the rotation plane every projection sees."""
    x, z, r = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
    check(load().rtkb_field_of_view_radius(geometry.handle, C.byref(proj_desc), int(kind), C.byref(x), C.byref(z),
                                           C.byref(r)))
    return x.value, z.value, r.value


def ramp_kernel(nu, spacing, params):
    import numpy as np

    padded = C.c_int(0)
    check(load().rtkb_ramp_kernel(nu, spacing, C.byref(params), C.byref(padded), None))
    k = np.zeros(padded.value // 2 + 1)
    check(load().rtkb_ramp_kernel(nu, spacing, C.byref(params), C.byref(padded),
                                  k.ctypes.data_as(C.POINTER(C.c_double))))
    return padded.value, k


def ramp_filter(proj_desc, proj, params=None, out=None, stream=None):
    """rtk::FFTRampImageFilter (row-wise ramp filtering)."""
    params = params or ramp_params()
    out = _unary(None, proj_desc, proj, out)
    check(load().rtkb_ramp_filter(C.byref(proj_desc), C.byref(params), _ptr(proj), _ptr(out), _stream(stream)))
    return out


def _displaced_mode(displaced):
    """rtkb_fdk_preprocess_params.displaced_detector: False 0, True 1
    (DisplacedDetectorImageFilter), "offset_fov" 2 (its ForOffsetFieldOfView
    variant)."""
    return 2 if displaced == "offset_fov" else int(bool(displaced))


def _displaced_region(geometry, proj_desc, displaced, pad):
    if _displaced_mode(displaced) == 2:
        return displaced_detector_offset_fov_region(geometry, proj_desc)[0]
    return displaced_detector_region(geometry, proj_desc, pad)[0]


def fdk_preprocess(geometry, proj_desc, proj, ramp=None, displaced=False, pad=True, short_scan=False,
                   threshold=3.141592653589793 / 9, stream=None, out=None):
    """Displaced detector + Parker + FDK weighting + ramp in one pass.
    displaced: False, True (DisplacedDetectorImageFilter) or "offset_fov"
    (DisplacedDetectorForOffsetFieldOfViewImageFilter).  Returns (filtered
    stack, its description)."""
    from ._capi import FdkPreprocessParams

    p = FdkPreprocessParams()
    p.displaced_detector, p.pad_on_truncated_side = _displaced_mode(displaced), int(pad)
    p.short_scan = int(short_scan)
    p.angular_gap_threshold = threshold
    p.ramp = ramp or ramp_params()
    od = proj_desc
    if displaced:
        od = _displaced_region(geometry, proj_desc, displaced, pad)
    out = _unary(None, proj_desc, proj, out, shape_of(od))
    from ._capi import ImageDesc

    got = ImageDesc()
    check(load().rtkb_fdk_preprocess(geometry.handle, C.byref(proj_desc), C.byref(p), C.byref(got), _ptr(proj),
                                     _ptr(out), _stream(stream)))
    return out, got


def fdk_preprocess_batch(problems, ramp=None, displaced=False, pad=True, short_scan=False,
                         threshold=3.141592653589793 / 9, stream=None):
    """rtkb_fdk_preprocess_batch: fdk_preprocess of every (geometry,
    proj_desc, proj, out) in `problems` (out None: allocated) in one launch per
    padded row length.  Returns [(filtered stack, its description)]."""
    from ._capi import FdkPreprocessParams, FdkPreprocessProblem

    p = FdkPreprocessParams()
    p.displaced_detector, p.pad_on_truncated_side = _displaced_mode(displaced), int(pad)
    p.short_scan = int(short_scan)
    p.angular_gap_threshold = threshold
    p.ramp = ramp or ramp_params()
    arr = (FdkPreprocessProblem * max(1, len(problems)))()
    outs = []
    for k, (geometry, proj_desc, proj, out) in enumerate(problems):
        od = proj_desc
        if displaced:
            od = _displaced_region(geometry, proj_desc, displaced, pad)
        out = _unary(None, proj_desc, proj, out, shape_of(od))
        arr[k].geometry, arr[k].proj = geometry.handle, proj_desc
        arr[k].d_in, arr[k].d_out = _ptr(proj), _ptr(out)
        outs.append(out)
    check(load().rtkb_fdk_preprocess_batch(arr, len(problems), C.byref(p), _stream(stream)))
    return [(o, arr[k].out) for k, o in enumerate(outs)]


def trim_memory_pool() -> int:
    """Return the library's unused reserved scratch memory (current device) to
    the driver; returns the bytes still reserved."""
    n = C.c_longlong()
    check(load().rtkb_trim_memory_pool(C.byref(n)))
    return n.value


def memory_pool_reserved() -> int:
    """Bytes the library's scratch pool holds on the current device."""
    n = C.c_longlong()
    check(load().rtkb_memory_pool_reserved(C.byref(n)))
    return n.value


def device_status(stream=None) -> int:
    """Synchronises the stream and returns (and clears) the kernels' status word."""
    st = C.c_int(0)
    check(load().rtkb_device_status(_stream(stream), C.byref(st)))
    return st.value


def laplacian(vol_desc, x, out=None, stream=None):
    """rtk::LaplacianImageFilter (CudaLaplacianImageFilter): out = Laplacian(x)
    with a zero-flux Neumann boundary, spacing-scaled."""
    _check_shape(x, vol_desc, "volume")
    if out is None:
        out = _torch().empty_like(x)
    _check_shape(out, vol_desc, "output")
    check(load().rtkb_laplacian(C.byref(vol_desc), _ptr(x), _ptr(out), _stream(stream)))
    return out


def ray_box_lengths(geometry, vol_desc, proj_desc, out=None, stream=None):
    """rtk::RayBoxIntersectionImageFilter (box of the volume, SetBoxFromImage(vol,
    false)): per-pixel ray length in mm."""
    if out is None:
        out = _torch().empty(shape_of(proj_desc), device="cuda", dtype=_torch().float32)
    _check_shape(out, proj_desc, "output")
    check(load().rtkb_ray_box_lengths(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), _ptr(out),
                                      _stream(stream)))
    return out


def sart(geometry, vol_desc, proj_desc, proj, x, niter=3, lam=0.3, positivity=False, subset=1,
         displaced_detector=True, threshold=1e-5, order=None, seed=0, stream=None):
    """rtk::SARTConeBeamReconstructionFilter (Joseph forward, voxel-based back
    projection), in place on x; order: processing order of the stack's
    projections (a permutation), or None for a seeded shuffle."""
    import numpy as np

    from ._capi import SartParams

    _check_shape(proj, proj_desc, "projections")
    _check_shape(x, vol_desc, "volume")
    p = SartParams()
    p.niter, p.lam, p.positivity = int(niter), float(lam), int(positivity)
    p.projections_per_subset, p.disable_displaced_detector = int(subset), int(not displaced_detector)
    p.division_threshold, p.seed = float(threshold), int(seed)
    keep = None
    if order is not None:
        keep = np.ascontiguousarray(order, dtype=np.int32)
        if keep.size != proj_desc.size[2]:
            raise ValueError("order must list every projection of the stack")
        p.order = keep.ctypes.data_as(C.POINTER(C.c_int))
    check(load().rtkb_sart(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), _ptr(proj), _ptr(x), C.byref(p),
                           _stream(stream)))
    return x


def osem(geometry, vol_desc, proj_desc, proj, x, niter=3, subset=1, beta=0.0, store_normalization=True,
         backprojector="voxel", order=None, seed=0, stream=None):
    """rtk::OSEMConeBeamReconstructionFilter (Joseph forward projection;
    backprojector "voxel", RTK's default, or "joseph") with De Pierro's
    regularisation weight beta, in place on x; order: processing order of
    the stack's projections (a permutation), or None for a seeded shuffle."""
    import numpy as np

    from ._capi import OsemParams

    codes = {"voxel": 0, "joseph": 1}
    if backprojector not in codes:
        raise ValueError(f"backprojector must be one of {sorted(codes)}")
    _check_shape(proj, proj_desc, "projections")
    _check_shape(x, vol_desc, "volume")
    p = OsemParams()
    p.niter, p.projections_per_subset, p.beta = int(niter), int(subset), float(beta)
    p.store_normalization, p.backprojector, p.seed = int(store_normalization), codes[backprojector], int(seed)
    keep = None
    if order is not None:
        keep = np.ascontiguousarray(order, dtype=np.int32)
        if keep.size != proj_desc.size[2]:
            raise ValueError("order must list every projection of the stack")
        p.order = keep.ctypes.data_as(C.POINTER(C.c_int))
    check(load().rtkb_osem(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), _ptr(proj), _ptr(x), C.byref(p),
                           _stream(stream)))
    return x


def de_pierro_regularization(vol_desc, xk, update, norm=None, beta=0.01, out=None, stream=None):
    """rtk::DePierroRegularizationImageFilter: inputs x_k, the ML-EM update and
    the normalisation volume (None: ones); returns the regularisation factor."""
    _check_shape(xk, vol_desc, "x_k")
    _check_shape(update, vol_desc, "update")
    if norm is not None:
        _check_shape(norm, vol_desc, "normalisation")
    if out is None:
        out = _torch().empty_like(xk)
    _check_shape(out, vol_desc, "output")
    check(load().rtkb_de_pierro_regularization(C.byref(vol_desc), _ptr(xk), _ptr(update),
                                               None if norm is None else _ptr(norm), float(beta), _ptr(out),
                                               _stream(stream)))
    return out


def _dims3(dims):
    return (C.c_int * 3)(*[int(bool(d)) for d in dims])


def regularized_cg(geometry, vol_desc, proj_desc, proj, x, weights=None, main_loop_iterations=10, cg_iterations=4,
                   tikhonov=0.0, gamma=0.0, positivity=True, tv=True, gamma_tv=5e-5, tv_iterations=10,
                   tv_dimensions=(True, True, True), soft_threshold_on_image=False, soft_threshold=1e-3,
                   displaced_detector=True, support_mask=None, stream=None):
    """rtk::RegularizedConjugateGradientConeBeamReconstructionFilter (Joseph
    pair; CG, positivity, TV denoising, soft threshold), in place on x."""
    from ._capi import RegularizedCgParams

    _check_shape(proj, proj_desc, "projections")
    _check_shape(x, vol_desc, "volume")
    if weights is not None:
        _check_shape(weights, proj_desc, "weights")
    p = RegularizedCgParams()
    p.main_loop_iterations, p.cg_iterations = int(main_loop_iterations), int(cg_iterations)
    p.tikhonov, p.gamma, p.positivity, p.tv = float(tikhonov), float(gamma), int(positivity), int(tv)
    p.gamma_tv, p.tv_iterations = float(gamma_tv), int(tv_iterations)
    dims = _dims3(tv_dimensions)
    p.tv_dimensions = C.cast(dims, C.POINTER(C.c_int))
    p.soft_threshold_on_image, p.soft_threshold = int(soft_threshold_on_image), float(soft_threshold)
    p.disable_displaced_detector = int(not displaced_detector)
    if support_mask is not None:
        _check_shape(support_mask, vol_desc, "support mask")
        p.support_mask = _ptr(support_mask).value
    check(load().rtkb_regularized_cg(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), _ptr(proj),
                                     None if weights is None else _ptr(weights), _ptr(x), C.byref(p),
                                     _stream(stream)))
    return x


def tv_denoising_bpdq(vol_desc, x, gamma, niter, dimensions=(True, True, True), out=None, stream=None):
    """rtk::TotalVariationDenoisingBPDQImageFilter (out may be x)."""
    _check_shape(x, vol_desc, "volume")
    if out is None:
        out = _torch().empty_like(x)
    _check_shape(out, vol_desc, "output")
    check(load().rtkb_tv_denoising_bpdq(C.byref(vol_desc), _ptr(x), _ptr(out), float(gamma), int(niter),
                                        _dims3(dimensions), _stream(stream)))
    return out


def total_variation(vol_desc, x, stream=None) -> float:
    """rtk::TotalVariationImageFilter (waits for the stream)."""
    _check_shape(x, vol_desc, "volume")
    v = C.c_double()
    check(load().rtkb_total_variation(C.byref(vol_desc), _ptr(x), C.byref(v), _stream(stream)))
    return v.value


def _ptr_u16(t):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a CUDA tensor (there is no CPU path)")
    if t.dtype not in (torch.uint16, torch.int16) or not t.is_contiguous():
        raise TypeError("expected a contiguous 16-bit tensor of raw counts")
    return C.c_void_p(t.data_ptr())


def i0_estimation(desc, raw, bit_shift=2, dyn_threshold=20, stream=None):
    """rtk::I0EstimationProjectionFilter on a 16-bit raw image (uint16 CUDA
    tensor): returns a dict with i0, i0_fwhm, imin, imax, low_bound, high_bound."""
    from ._capi import I0Estimate

    _check_shape(raw, desc, "raw image")
    r = I0Estimate()
    check(load().rtkb_i0_estimation(C.byref(desc), _ptr_u16(raw), int(bit_shift), int(dyn_threshold), C.byref(r),
                                    _stream(stream)))
    return {k: getattr(r, k) for k, _ in r._fields_}


def raw_to_attenuation(desc, raw, i0=65535.0, idark=0.0, out=None, stream=None):
    """rtk::LUTbasedVariableI0RawToAttenuationImageFilter: line integrals
    log(I0 - IDark) - log(raw - IDark) of a uint16 CUDA tensor (float32 out)."""
    _check_shape(raw, desc, "raw image")
    if out is None:
        out = _torch().empty(tuple(raw.shape), device="cuda", dtype=_torch().float32)
    _check_shape(out, desc, "output")
    check(load().rtkb_raw_to_attenuation(C.byref(desc), _ptr_u16(raw), float(i0), float(idark), _ptr(out),
                                         _stream(stream)))
    return out


def iterative_fdk(geometry, vol_desc, proj_desc, proj, x, niter=3, lam=0.3, positivity=False, ramp=None,
                  displaced=True, pad=True, short_scan=True, threshold=3.141592653589793 / 9, stream=None):
    """rtk::IterativeFDKConeBeamReconstructionFilter (Joseph forward projection),
    in place on x (x0 in, result out)."""
    from ._capi import IterativeFdkParams

    _check_shape(proj, proj_desc, "projections")
    _check_shape(x, vol_desc, "volume")
    p = IterativeFdkParams()
    p.niter, p.lam, p.positivity = int(niter), float(lam), int(positivity)
    p.fdk.displaced_detector, p.fdk.pad_on_truncated_side, p.fdk.short_scan = int(displaced), int(pad), int(short_scan)
    p.fdk.angular_gap_threshold = threshold
    p.fdk.ramp = ramp or ramp_params()
    check(load().rtkb_iterative_fdk(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), _ptr(proj), _ptr(x),
                                    C.byref(p), _stream(stream)))
    return x


def water_precorrection(desc, proj, coefficients, out=None, stream=None):
    """rtk::WaterPrecorrectionImageFilter: out = sum_j c_j proj^j (out may be proj)."""
    _check_shape(proj, desc, "projections")
    if out is None:
        out = _torch().empty_like(proj)
    _check_shape(out, desc, "output")
    c = (C.c_double * max(1, len(coefficients)))(*[float(v) for v in coefficients])
    check(load().rtkb_water_precorrection(C.byref(desc), _ptr(proj), _ptr(out), c, len(coefficients),
                                          _stream(stream)))
    return out


def _backprojector_code(bp):
    """RTK's back projector choice of its iterative filters: "joseph"
    (BP_JOSEPH) or "voxel" (BP_VOXELBASED, rtkconjugategradient's default)."""
    codes = {"voxel": 0, "voxelbased": 0, "joseph": 1}  # RTK's BackProjectionType values
    if bp not in codes:
        raise ValueError(f"backprojector must be one of {sorted(codes)}")
    return codes[bp]


def _storage_code(storage):
    # "bf16": r, p, A p and the projection temporary stored as BF16;
    # "bf16_direction": p and the projection temporary BF16, r and A p FP32
    codes = {"fp32": 0, "bf16": 1, "bf16_direction": 2}
    if storage not in codes:
        raise ValueError(f"storage must be one of {sorted(codes)}")
    return codes[storage]


class ConjugateGradient:
    """Plan of rtk::ConjugateGradientConeBeamReconstructionFilter (Joseph
    forward projector; Joseph or voxel-based back projector, RTK's SetBackProjectionFilter
    choice; FP64 scalars on the device, one CUDA graph per iteration).
    storage="bf16" stores the normal-equation vectors and the
    projection-domain temporary as bfloat16 (FP32 arithmetic, FP64 dots and
    step sizes; Joseph back projector)."""

    def __init__(self, geometry, vol_desc, proj_desc, tikhonov=0.0, use_cuda_graph=True, storage="fp32",
                 gamma=0.0, backprojector="joseph"):
        from ._capi import CgParams

        self._lib = load()
        self.geometry = geometry
        self.vol_desc, self.proj_desc = vol_desc, proj_desc
        p = CgParams()
        p.tikhonov, p.use_cuda_graph, p.storage = tikhonov, int(use_cuda_graph), _storage_code(storage)
        p.gamma = gamma
        p.backprojector = _backprojector_code(backprojector)
        h = C.c_void_p()
        check(self._lib.rtkb_cg_create(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), C.byref(p),
                                       C.byref(h)))
        self._h = h
        self._keep = []

    def start(self, proj, x, weights=None, displaced_detector=True, stream=None):
        _check_shape(proj, self.proj_desc, "projections")
        _check_shape(x, self.vol_desc, "volume")
        if weights is not None:
            _check_shape(weights, self.proj_desc, "weights")
        self._keep = [proj, x, weights]
        check(self._lib.rtkb_cg_start(self._h, _ptr(proj), _ptr(weights) if weights is not None else None,
                                      int(displaced_detector), _ptr(x), _stream(stream)))
        return self

    def set_support_mask(self, mask):
        """ConjugateGradientConeBeamReconstructionFilter::SetSupportMask (a
        float32 volume, kept referenced; None removes it); before start."""
        if mask is not None:
            _check_shape(mask, self.vol_desc, "support mask")
        check(self._lib.rtkb_cg_set_support_mask(self._h, None if mask is None else _ptr(mask)))
        self._mask = mask

    def finish(self, stream=None):
        """The filter's output multiplication by the support mask (no-op without one)."""
        check(self._lib.rtkb_cg_finish(self._h, _stream(stream)))

    def start_rhs(self, b, x, stream=None):
        """Start CG on A x = b for a given right-hand side volume b."""
        _check_shape(b, self.vol_desc, "right-hand side")
        _check_shape(x, self.vol_desc, "volume")
        self._keep = [b, x]
        check(self._lib.rtkb_cg_start_rhs(self._h, _ptr(b), _ptr(x), _stream(stream)))
        return self

    def iterate(self, n=1, stream=None):
        check(self._lib.rtkb_cg_iterate(self._h, int(n), _stream(stream)))

    def set_preconditioner(self, net, history=8):
        """Flexible PCG with a learned preconditioner (a rtk_b200.learned.UNet;
        None removes it), re-orthogonalising against `history` directions.
        Call before start()."""
        self._net = net
        check(self._lib.rtkb_cg_set_preconditioner(self._h, net.handle if net is not None else None,
                                                   int(history)))

    def preconditioner_status(self):
        """(network still in use, iteration at which plain CG took over or -1)."""
        a, f = C.c_int(), C.c_int()
        check(self._lib.rtkb_cg_preconditioner_status(self._h, C.byref(a), C.byref(f)))
        return bool(a.value), f.value

    def apply_operator(self, x, out, stream=None):
        """out = A x (normal operator of the plan; W = 1 before start())."""
        _check_shape(x, self.vol_desc, "volume")
        _check_shape(out, self.vol_desc, "volume")
        check(self._lib.rtkb_cg_apply_operator(self._h, _ptr(x), _ptr(out), _stream(stream)))
        return out

    def save_state(self, stream=None, device="cuda"):
        """Checkpoint of the recurrence (rtkb_cg_save_state): a uint8 tensor on
        `device` holding the scalars, R, P and the iteration count; the iterate
        x is the caller's tensor and is saved by the caller."""
        n = C.c_longlong()
        check(self._lib.rtkb_cg_state_bytes(self._h, C.byref(n)))
        buf = _torch().empty(n.value, dtype=_torch().uint8, device=device)
        check(self._lib.rtkb_cg_save_state(self._h, C.c_void_p(buf.data_ptr()), _stream(stream)))
        return buf

    def load_state(self, buf, stream=None):
        """Resume from save_state()'s checkpoint (rtkb_cg_load_state); call
        after start() on the saved iterate."""
        if buf.dtype != _torch().uint8 or not buf.is_contiguous():
            raise TypeError("expected the contiguous uint8 tensor save_state() returned")
        check(self._lib.rtkb_cg_load_state(self._h, C.c_void_p(buf.data_ptr()), _stream(stream)))

    def residual(self, stream=None):
        """(||r_k||^2, ||r_0||^2, k) -- synchronises the stream."""
        rr, rr0, it = C.c_double(), C.c_double(), C.c_int()
        check(self._lib.rtkb_cg_residual(self._h, C.byref(rr), C.byref(rr0), C.byref(it), _stream(stream)))
        return rr.value, rr0.value, it.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rtkb_cg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ConjugateGradientBatch:
    """Batched CG (rtkb_cg_batch_*): many independent problems, each a tuple
    (geometry, vol_desc, proj_desc, proj, x[, weights[, displaced_detector]]);
    iterate(n) runs n iterations of every problem as one CUDA graph launch."""

    def __init__(self, problems, tikhonov=0.0, storage="fp32", gamma=0.0, backprojector="joseph"):
        from ._capi import CgBatchProblem, CgParams

        self._lib = load()
        arr = (CgBatchProblem * len(problems))()
        self._keep = list(problems)
        for i, prob in enumerate(problems):
            g, vd, pd, proj, x = prob[:5]
            w = prob[5] if len(prob) > 5 else None
            dd = prob[6] if len(prob) > 6 else True
            _check_shape(proj, pd, "projections")
            _check_shape(x, vd, "volume")
            if w is not None:
                _check_shape(w, pd, "weights")
            q = arr[i]
            q.geometry, q.vol, q.proj = g.handle, vd, pd
            q.d_proj, q.d_x = _ptr(proj).value, _ptr(x).value
            q.d_weights = _ptr(w).value if w is not None else None
            q.displaced_detector = int(dd)
        self._arr = arr
        p = CgParams()
        p.tikhonov, p.use_cuda_graph, p.storage, p.gamma = tikhonov, 0, _storage_code(storage), gamma
        p.backprojector = _backprojector_code(backprojector)
        h = C.c_void_p()
        check(self._lib.rtkb_cg_batch_create(arr, len(problems), C.byref(p), C.byref(h)))
        self._h = h
        self.n = len(problems)

    def start(self, stream=None):
        check(self._lib.rtkb_cg_batch_start(self._h, self._arr, _stream(stream)))

    def iterate(self, n, stream=None):
        check(self._lib.rtkb_cg_batch_iterate(self._h, int(n), _stream(stream)))

    def residual(self, i, stream=None):
        """(||r_k||^2, ||r_0||^2, k) of problem i -- synchronises the stream."""
        plan = self._lib.rtkb_cg_batch_plan(self._h, int(i))
        if not plan:
            raise IndexError(i)
        rr, rr0, it = C.c_double(), C.c_double(), C.c_int()
        check(self._lib.rtkb_cg_residual(C.c_void_p(plan), C.byref(rr), C.byref(rr0), C.byref(it), _stream(stream)))
        return rr.value, rr0.value, it.value

    def close(self):
        if getattr(self, "_h", None):
            _torch().cuda.synchronize()
            self._lib.rtkb_cg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def conjugate_gradient(geometry, vol_desc, proj_desc, proj, x, niter, rel_residual=0.0, weights=None,
                       displaced_detector=True, tikhonov=0.0, use_cuda_graph=True, stream=None, storage="fp32",
                       gamma=0.0, backprojector="joseph"):
    """Whole CG reconstruction in place on x; returns (iterations, relative residual)."""
    from ._capi import CgParams

    p = CgParams()
    p.tikhonov, p.use_cuda_graph, p.storage = tikhonov, int(use_cuda_graph), _storage_code(storage)
    p.gamma = gamma
    p.backprojector = _backprojector_code(backprojector)
    it, rel = C.c_int(), C.c_double()
    check(load().rtkb_conjugate_gradient(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), C.byref(p),
                                         _ptr(proj), _ptr(weights) if weights is not None else None,
                                         int(displaced_detector), _ptr(x), int(niter), float(rel_residual),
                                         C.byref(it), C.byref(rel), _stream(stream)))
    return it.value, rel.value


def _host_ptr(t, what):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or t.is_cuda:
        raise TypeError(f"{what}: expected a host (CPU) tensor")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError(f"{what}: expected a contiguous float32 tensor")
    return C.c_void_p(t.data_ptr())


def fdk_backproject_host(geometry, vol_desc, proj_desc, proj, vol_in=None, out=None, chunk=0, stream=None):
    """rtkb_fdk_backproject_host: FDK backprojection of a host (CPU) stack into a
    host volume, the stack streamed to the GPU in subsets growing from
    chunk / 12 to `chunk` projections (0: a quarter of the stack), each copy
    overlapping the backprojection of the previous subset; the volume comes
    back slab by slab while the last subset is backprojected.  vol_in None
    means a zero volume.
    Asynchronous on `stream`: synchronise it before reading `out`.  Pinned
    tensors (pin_memory=True) give full copy bandwidth and overlap."""
    torch = _torch()
    _check_shape(proj, proj_desc, "projections")
    if vol_in is not None:
        _check_shape(vol_in, vol_desc, "volume")
    if out is None:
        out = torch.empty(shape_of(vol_desc), dtype=torch.float32, pin_memory=True)
    _check_shape(out, vol_desc, "output")
    vin = _host_ptr(vol_in, "volume") if vol_in is not None else None
    check(load().rtkb_fdk_backproject_host(geometry.handle, C.byref(vol_desc), C.byref(proj_desc),
                                           _host_ptr(proj, "projections"), vin, _host_ptr(out, "output"),
                                           int(chunk), _stream(stream)))
    return out


def fdk_backproject_static_scratch(geometry, vol_desc, proj_desc, proj, vol_in, out=None, stream=None):
    """rtkb_fdk_backproject_static_scratch: FDK backprojection that allocates no
    device memory (stacks of at most 2048 projections; see include/rtkb200.h)."""
    return _backproject(load().rtkb_fdk_backproject_static_scratch, geometry, vol_desc, proj_desc, proj, vol_in,
                        out, stream)


def project_ellipsoids(geometry, proj_desc, ellipsoids, out=None, stream=None):
    """Analytic projections of ellipsoids (16 doubles each: centre, semi-axes,
    rotation local->world row-major, density) onto the described stack."""
    import numpy as np

    torch = _torch()
    e = np.ascontiguousarray(ellipsoids, dtype=np.float64).reshape(-1, 16)
    if out is None:
        out = torch.empty(shape_of(proj_desc), device="cuda", dtype=torch.float32)
    _check_shape(out, proj_desc, "output")
    check(load().rtkb_project_ellipsoids(geometry.handle, C.byref(proj_desc), e.shape[0],
                                         e.ctypes.data_as(C.POINTER(C.c_double)), _ptr(out), _stream(stream)))
    return out


def _problem_array(problems):
    from ._capi import BpProblem

    torch = _torch()
    arr = (BpProblem * len(problems))()
    keep = []
    for k, (geometry, vol_desc, proj_desc, proj, vol_in, out) in enumerate(problems):
        _check_shape(proj, proj_desc, "projections")
        _check_shape(vol_in, vol_desc, "volume")
        _check_shape(out, vol_desc, "output")
        arr[k].geometry = geometry.handle
        arr[k].vol = vol_desc
        arr[k].proj = proj_desc
        arr[k].d_proj = _ptr(proj).value
        arr[k].d_vol_in = _ptr(vol_in).value
        arr[k].d_vol_out = _ptr(out).value
        keep.append((proj, vol_in, out))
    return arr, keep


def backproject_batch(problems, fdk=True, config=-1, stream=None):
    """Batched FDK (or voxel) backprojection of independent problems in one
    persistent launch.  problems: [(geometry, vol_desc, proj_desc, proj,
    vol_in, out)], float32 CUDA tensors.  Returns the configuration used."""
    arr, _ = _problem_array(problems)
    used = C.c_int(-1)
    L = load()
    fn = L.rtkb_fdk_backproject_batch if fdk else L.rtkb_voxel_backproject_batch
    check(fn(arr, len(problems), int(config), C.byref(used), _stream(stream)))
    return used.value


def _tune_key(problems, fdk, device_name):
    """Autotuner cache key: the kernel, the device and every problem's volume
    and stack sizes (the tile configuration depends on nothing else)."""
    shapes = sorted((tuple(int(v) for v in p[1].size), tuple(int(v) for v in p[2].size)) for p in problems)
    return json.dumps({"kernel": "fdk_backproject" if fdk else "voxel_backproject", "device": device_name,
                       "problems": shapes}, sort_keys=True)


def _cache_get(path, key):
    try:
        with open(path) as f:
            return json.load(f).get(key)
    except (OSError, ValueError):
        return None


def _cache_put(path, key, value):
    """Adds one entry to the JSON cache file (written to a temporary file and
    renamed, so a reader never sees a partial file)."""
    try:
        with open(path) as f:
            data = json.load(f)
    except (OSError, ValueError):
        data = {}
    data[key] = value
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def backproject_autotune(problems, fdk=True, repeats=2, stream=None, cache=None):
    """The project's autotuner: times every backprojector configuration on the
    batch and returns (best configuration, its ms, [ms per configuration]).
    cache: path of a JSON file of earlier results keyed by kernel, device and
    problem sizes; a hit returns the stored result without timing anything."""
    key = None
    if cache is not None:
        key = _tune_key(problems, fdk, _torch().cuda.get_device_name())
        hit = _cache_get(cache, key)
        if hit is not None:
            return hit["config"], hit["ms"], hit["ms_per_config"]
    arr, _ = _problem_array(problems)
    times = (C.c_double * 16)(*([-1.0] * 16))  # one entry per configuration (fewer than 16)
    best, best_ms = C.c_int(), C.c_double()
    check(load().rtkb_backproject_autotune(arr, len(problems), int(fdk), int(repeats), C.byref(best),
                                           C.byref(best_ms), times, _stream(stream)))
    result = (best.value, best_ms.value, [t for t in times if t >= 0.0])
    if cache is not None:
        _cache_put(cache, key, {"config": result[0], "ms": result[1], "ms_per_config": result[2]})
    return result


JOSEPH_BAND_ROWS = (8, 16, 32, 64)


def joseph_band_rows(forward=None, back=None):
    """Current detector rows per band of the Joseph projectors' grids; sets
    them first when given (rtkb_joseph_set_band_rows)."""
    f, b = C.c_int(), C.c_int()
    check(load().rtkb_joseph_get_band_rows(C.byref(f), C.byref(b)))
    if forward is not None or back is not None:
        f.value, b.value = forward or f.value, back or b.value
        check(load().rtkb_joseph_set_band_rows(f.value, b.value))
    return f.value, b.value


def joseph_autotune(geometry, vol_desc, proj_desc, vol, proj, repeats=2, stream=None, cache=None, apply=True):
    """Autotuner of the Joseph pair's band height: times the forward projection
    of `vol` and the back projection of `proj` (neither is modified; outputs go
    to scratch tensors) for every band of JOSEPH_BAND_ROWS with CUDA events,
    and returns {"forward": rows, "back": rows, "forward_ms": [...],
    "back_ms": [...]}, applied with rtkb_joseph_set_band_rows unless
    apply=False.  cache: JSON file keyed by kernel, device and sizes, as for
    backproject_autotune."""
    torch = _torch()
    key = None
    if cache is not None:
        shapes = [tuple(int(v) for v in vol_desc.size), tuple(int(v) for v in proj_desc.size)]
        key = json.dumps({"kernel": "joseph_pair", "device": torch.cuda.get_device_name(), "problems": [shapes]},
                         sort_keys=True)
        hit = _cache_get(cache, key)
        if hit is not None:
            if apply:
                joseph_band_rows(hit["forward"], hit["back"])
            return hit
    saved = joseph_band_rows()
    st = stream if stream is not None else torch.cuda.current_stream()
    pout = torch.empty_like(proj)
    pzero = torch.zeros_like(proj)
    vout = torch.empty_like(vol)
    vzero = torch.zeros_like(vol)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        best = None
        for _ in range(max(1, repeats)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            fn()
            e1.record(st)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        return best

    fwd_ms, back_ms = [], []
    try:
        for rows in JOSEPH_BAND_ROWS:
            joseph_band_rows(rows, rows)
            fwd_ms.append(timed(lambda: joseph_forward_project(geometry, vol_desc, proj_desc, vol, pzero, out=pout,
                                                               stream=st)))
            back_ms.append(timed(lambda: joseph_back_project(geometry, vol_desc, proj_desc, proj, vzero, out=vout,
                                                             stream=st)))
    finally:
        joseph_band_rows(*saved)
    res = {"forward": JOSEPH_BAND_ROWS[fwd_ms.index(min(fwd_ms))], "back": JOSEPH_BAND_ROWS[back_ms.index(min(back_ms))],
           "forward_ms": fwd_ms, "back_ms": back_ms}
    if apply:
        joseph_band_rows(res["forward"], res["back"])
    if cache is not None:
        _cache_put(cache, key, res)
    return res


class BackprojectionBatch:
    """Prepared batch (rtkb_bp_batch_*): host work done once, each execute()
    is one persistent launch over all problems.  The tensors of `problems`
    are kept alive with the batch."""

    def __init__(self, problems, fdk=True, config=-1):
        self._lib = load()
        arr, self._keep = _problem_array(problems)
        h = C.c_void_p()
        check(self._lib.rtkb_bp_batch_create(arr, len(problems), int(fdk), int(config), C.byref(h)))
        self._h = h
        self.config = self._lib.rtkb_bp_batch_config(h)

    def execute(self, stream=None):
        check(self._lib.rtkb_bp_batch_execute(self._h, _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            torch = _torch()
            torch.cuda.synchronize()
            self._lib.rtkb_bp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def backproject_config(force=-1):
    """Autotuner hook of the tiled backprojector (rtkb_backproject_config):
    force >= 0 selects that configuration for later calls on this host thread,
    -1 restores the footprint heuristic.  Returns (configuration of the last
    tiled launch on this thread or -1, number of configurations)."""
    last, count = C.c_int(), C.c_int()
    check(load().rtkb_backproject_config(int(force), C.byref(last), C.byref(count)))
    return last.value, count.value


def backproject_schedule(schedule, sweep_shift=4):
    """Tile schedule of the tiled backprojector (rtkb_bp_set_schedule): 0 every
    tile walks the stack from projection 0 (run-to-run identical sums), 1 the
    projection sweep (chunks of 2^sweep_shift projections; tiles in flight
    share projections in L2, summation order varies at FP32 rounding)."""
    check(load().rtkb_bp_set_schedule(int(schedule), int(sweep_shift)))
