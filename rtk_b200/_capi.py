"""ctypes binding of librtkb200.so (the C ABI declared in include/rtkb200.h).

The library is built in-tree by ``rtk_b200.build``.  Loading fails loudly when
it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "librtkb200.so")
HEADER_PATH = os.path.join(os.path.dirname(_PKG), "include", "rtkb200.h")

RTKB_OK = 0
RTKB_ERR_INVALID_ARGUMENT = 1
RTKB_ERR_CUDA = 2
RTKB_ERR_UNSUPPORTED = 3
RTKB_ERR_TIMEOUT = 4
RTKB_ERR_OUT_OF_MEMORY = 5


class ImageDesc(C.Structure):
    """rtkb_image_desc: itk::ImageBase metadata of a 3-D image."""

    _fields_ = [
        ("size", C.c_int * 3),
        ("index", C.c_int * 3),
        ("origin", C.c_double * 3),
        ("spacing", C.c_double * 3),
        ("direction", C.c_double * 9),
    ]


class RampParams(C.Structure):
    """rtkb_ramp_params (rtk::FFTRampImageFilter settings)."""

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


class FdkPreprocessProblem(C.Structure):
    """rtkb_fdk_preprocess_problem."""

    _fields_ = [("geometry", C.c_void_p), ("proj", ImageDesc), ("d_in", C.c_void_p), ("d_out", C.c_void_p),
                ("out", ImageDesc)]


class FdkPreprocessParams(C.Structure):
    """rtkb_fdk_preprocess_params."""

    _fields_ = [
        ("displaced_detector", C.c_int),
        ("pad_on_truncated_side", C.c_int),
        ("short_scan", C.c_int),
        ("angular_gap_threshold", C.c_double),
        ("ramp", RampParams),
    ]


class RtkbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rtkb error {code}: {msg}")
        self.code = code


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_F = C.POINTER(C.c_float)
_V = C.c_void_p
_G = C.c_void_p
_IM = C.POINTER(ImageDesc)

# name -> (restype, argtypes)
SIGNATURES = {
    "rtkb_last_error": (C.c_char_p, []),
    "rtkb_version": (C.c_char_p, []),
    "rtkb_device_status": (C.c_int, [_V, _I]),
    "rtkb_geometry_new": (_G, []),
    "rtkb_geometry_free": (None, [_G]),
    "rtkb_geometry_add_projection": (C.c_int, [_G] + [C.c_double] * 9),
    "rtkb_geometry_add_projection_in_radians": (C.c_int, [_G] + [C.c_double] * 9),
    "rtkb_geometry_number_of_projections": (C.c_int, [_G]),
    "rtkb_geometry_get_matrix": (C.c_int, [_G, C.c_int, _D]),
    "rtkb_geometry_get_source_position": (C.c_int, [_G, C.c_int, _D]),
    "rtkb_geometry_get_projection_coordinates_to_fixed_system_matrix": (C.c_int, [_G, C.c_int, _D]),
    "rtkb_geometry_get_parameters": (C.c_int, [_G, C.c_int, _D]),
    "rtkb_geometry_to_untilted_coordinate_at_isocenter": (C.c_double, [_G, C.c_int, C.c_double]),
    "rtkb_geometry_set_radius_cylindrical_detector": (C.c_int, [_G, C.c_double]),
    "rtkb_backprojection_matrices": (C.c_int, [_G, _IM, _IM, C.c_int, C.c_int, C.c_int, _D, _I]),
    "rtkb_fdk_backproject": (C.c_int, [_G, _IM, _IM, _V, _V, _V, _V]),
    "rtkb_fdk_backproject_host": (C.c_int, [_G, _IM, _IM, _V, _V, _V, C.c_int, _V]),
    "rtkb_voxel_backproject": (C.c_int, [_G, _IM, _IM, _V, _V, _V, _V]),
    "rtkb_backproject_matrices": (C.c_int, [_I, _I, C.c_int, _D, _I, C.c_int, _V, _V, _V, _V]),
    "rtkb_probe_smem_gather": (C.c_int, [C.c_int, C.c_int, _V, _V]),
    "rtkb_backproject_config": (C.c_int, [C.c_int, _I, _I]),
    "rtkb_bp_set_schedule": (C.c_int, [C.c_int, C.c_int]),
    "rtkb_joseph_set_band_rows": (C.c_int, [C.c_int, C.c_int]),
    "rtkb_joseph_get_band_rows": (C.c_int, [_I, _I]),
    "rtkb_joseph_forward_project": (C.c_int, [_G, _IM, _IM, _V, _V, _V, _V]),
    "rtkb_joseph_back_project": (C.c_int, [_G, _IM, _IM, _V, _V, _V, _V]),
    "rtkb_fdk_weight": (C.c_int, [_G, _IM, _V, _V, _V]),
    "rtkb_parker_short_scan": (C.c_int, [_G, _IM, C.c_double, _V, _V, _V, _I]),
    "rtkb_displaced_detector_region": (C.c_int, [_G, _IM, C.c_int, _IM, _I]),
    "rtkb_displaced_detector": (C.c_int, [_G, _IM, C.c_int, _V, _V, _V]),
    "rtkb_displaced_detector_offset_fov_region": (C.c_int, [_G, _IM, _IM, _I]),
    "rtkb_displaced_detector_offset_fov": (C.c_int, [_G, _IM, _V, _V, _V]),
    "rtkb_field_of_view_radius": (C.c_int, [_G, _IM, C.c_int, _D, _D, _D]),
    "rtkb_ramp_kernel": (C.c_int, [C.c_int, C.c_double, C.POINTER(RampParams), _I, _D]),
    "rtkb_ramp_filter": (C.c_int, [_IM, C.POINTER(RampParams), _V, _V, _V]),
    "rtkb_fdk_preprocess": (C.c_int, [_G, _IM, C.POINTER(FdkPreprocessParams), _IM, _V, _V, _V]),
    "rtkb_fdk_preprocess_batch": (C.c_int, [C.POINTER(FdkPreprocessProblem), C.c_int, C.POINTER(FdkPreprocessParams),
                                            _V]),
}

_lib = None


def header_symbols() -> list[str]:
    """Names of every function declared in include/rtkb200.h."""
    txt = open(HEADER_PATH).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rtkb_[a-z0-9_]+)\s*\(", txt)))


def load(path: str = LIB_PATH):
    """Load librtkb200.so and attach signatures; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m rtk_b200.build` (no CPU fallback exists)")
    L = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code: int) -> None:
    if code != RTKB_OK:
        msg = load().rtkb_last_error()
        raise RtkbError(code, msg.decode() if msg else "")


class CgParams(C.Structure):
    """rtkb_cg_params."""

    _fields_ = [("tikhonov", C.c_double), ("use_cuda_graph", C.c_int), ("storage", C.c_int), ("gamma", C.c_double),
                ("backprojector", C.c_int)]


SIGNATURES.update({
    "rtkb_cg_create": (C.c_int, [_G, _IM, _IM, C.POINTER(CgParams), C.POINTER(C.c_void_p)]),
    "rtkb_cg_start": (C.c_int, [_V, _V, _V, C.c_int, _V, _V]),
    "rtkb_cg_iterate": (C.c_int, [_V, C.c_int, _V]),
    "rtkb_cg_residual": (C.c_int, [_V, _D, _D, _I, _V]),
    "rtkb_cg_destroy": (None, [_V]),
    "rtkb_conjugate_gradient": (C.c_int, [_G, _IM, _IM, C.POINTER(CgParams), _V, _V, C.c_int, _V, C.c_int,
                                          C.c_double, _I, _D, _V]),
})

SIGNATURES.update({
    "rtkb_fdk_backproject_static_scratch": (C.c_int, [_G, _IM, _IM, _V, _V, _V, _V]),
})

SIGNATURES.update({
    "rtkb_geometry_set_collimation_of_last_projection": (C.c_int, [_G, C.c_double, C.c_double, C.c_double,
                                                                   C.c_double]),
    "rtkb_geometry_read_xml": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "rtkb_geometry_write_xml": (C.c_int, [_G, C.c_char_p]),
    "rtkb_image_read_mha": (C.c_int, [C.c_char_p, _IM, _V, C.c_longlong]),
    "rtkb_laplacian": (C.c_int, [_IM, _V, _V, _V]),
    "rtkb_ray_box_lengths": (C.c_int, [_G, _IM, _IM, _V, _V]),
    "rtkb_sart": (C.c_int, [_G, _IM, _IM, _V, _V, C.c_void_p, _V]),
    "rtkb_osem": (C.c_int, [_G, _IM, _IM, _V, _V, C.c_void_p, _V]),
    "rtkb_water_precorrection": (C.c_int, [_IM, _V, _V, C.POINTER(C.c_double), C.c_int, _V]),
    "rtkb_iterative_fdk": (C.c_int, [_G, _IM, _IM, _V, _V, C.c_void_p, _V]),
    "rtkb_cg_set_support_mask": (C.c_int, [C.c_void_p, _V]),
    "rtkb_cg_finish": (C.c_int, [C.c_void_p, _V]),
    "rtkb_i0_estimation": (C.c_int, [_IM, _V, C.c_int, C.c_uint, C.c_void_p, _V]),
    "rtkb_raw_to_attenuation": (C.c_int, [_IM, _V, C.c_double, C.c_double, _V, _V]),
    "rtkb_regularized_cg": (C.c_int, [_G, _IM, _IM, _V, _V, _V, C.c_void_p, _V]),
    "rtkb_tv_denoising_bpdq": (C.c_int, [_IM, _V, _V, C.c_double, C.c_int, C.POINTER(C.c_int), _V]),
    "rtkb_total_variation": (C.c_int, [_IM, _V, C.POINTER(C.c_double), _V]),
    "rtkb_trim_memory_pool": (C.c_int, [C.POINTER(C.c_longlong)]),
    "rtkb_set_wait_limit": (C.c_int, [C.c_uint, C.POINTER(C.c_uint)]),
    "rtkb_wait_self_test": (C.c_int, [_V]),
    "rtkb_inject_allocation_failures": (C.c_int, [C.c_int]),
    "rtkb_memory_pool_reserved": (C.c_int, [C.POINTER(C.c_longlong)]),
    "rtkb_de_pierro_regularization": (C.c_int, [_IM, _V, _V, _V, C.c_double, _V, _V]),
    "rtkb_image_write_mha": (C.c_int, [C.c_char_p, _IM, _V, C.c_int]),
})

class CgBatchProblem(C.Structure):
    """rtkb_cg_batch_problem."""

    _fields_ = [("geometry", C.c_void_p), ("vol", ImageDesc), ("proj", ImageDesc), ("d_proj", C.c_void_p),
                ("d_weights", C.c_void_p), ("displaced_detector", C.c_int), ("d_x", C.c_void_p)]


SIGNATURES.update({
    "rtkb_cg_batch_create": (C.c_int, [C.POINTER(CgBatchProblem), C.c_int, C.POINTER(CgParams),
                                       C.POINTER(C.c_void_p)]),
    "rtkb_cg_batch_start": (C.c_int, [_V, C.POINTER(CgBatchProblem), _V]),
    "rtkb_cg_batch_iterate": (C.c_int, [_V, C.c_int, _V]),
    "rtkb_cg_batch_plan": (C.c_void_p, [_V, C.c_int]),
    "rtkb_cg_batch_destroy": (None, [_V]),
})

SIGNATURES.update({
    "rtkb_project_ellipsoids": (C.c_int, [_G, _IM, C.c_int, _D, _V, _V]),
})

SIGNATURES.update({
    "rtkb_cg_apply_operator": (C.c_int, [_V, _V, _V, _V]),
    "rtkb_cg_state_bytes": (C.c_int, [_V, C.POINTER(C.c_longlong)]),
    "rtkb_cg_save_state": (C.c_int, [_V, _V, _V]),
    "rtkb_cg_load_state": (C.c_int, [_V, _V, _V]),
    "rtkb_cg_start_rhs": (C.c_int, [_V, _V, _V, _V]),
    "rtkb_joseph_sample_count": (C.c_int, [_G, _IM, _IM, _D, _V]),
    "rtkb_fdk_backproject_bf16": (C.c_int, [_G, _IM, _IM, _V, _V, _V, _V]),
    "rtkb_voxel_backproject_bf16": (C.c_int, [_G, _IM, _IM, _V, _V, _V, _V]),
    "rtkb_convert_to_bf16": (C.c_int, [_V, _V, C.c_longlong, _V]),
    "rtkb_cg_set_preconditioner": (C.c_int, [_V, _V, C.c_int]),
    "rtkb_cg_preconditioner_status": (C.c_int, [_V, _I, _I]),
    "rtkb_unet_create": (C.c_int, [C.c_ulonglong, C.POINTER(C.c_void_p)]),
    "rtkb_unet_num_parameters": (C.c_longlong, [_V]),
    "rtkb_unet_get_parameters": (C.c_int, [_V, _F, C.c_longlong]),
    "rtkb_unet_set_parameters": (C.c_int, [_V, _F, C.c_longlong]),
    "rtkb_unet_get_gradients": (C.c_int, [_V, _F, C.c_longlong]),
    "rtkb_unet_reserve": (C.c_int, [_V, C.c_int, C.c_int, C.c_int, C.c_int]),
    "rtkb_unet_forward": (C.c_int, [_V, C.c_int, C.c_int, C.c_int, C.c_int, _V, _V, C.c_int, _V]),
    "rtkb_unet_train_step": (C.c_int, [_V, C.c_int, C.c_int, C.c_int, C.c_int, _V, _V, C.c_int, C.c_double,
                                       C.c_int, _D, _V]),
    "rtkb_unet_destroy": (None, [_V]),
    "rtkb_unet_set_conv_pipeline": (C.c_int, [C.c_int]),
    "rtkb_unet_set_wgrad_kernel": (C.c_int, [C.c_int]),
})


class BpProblem(C.Structure):
    """rtkb_bp_problem."""

    _fields_ = [("geometry", C.c_void_p), ("vol", ImageDesc), ("proj", ImageDesc), ("d_proj", C.c_void_p),
                ("d_vol_in", C.c_void_p), ("d_vol_out", C.c_void_p)]


SIGNATURES.update({
    "rtkb_fdk_backproject_batch": (C.c_int, [C.POINTER(BpProblem), C.c_int, C.c_int, _I, _V]),
    "rtkb_voxel_backproject_batch": (C.c_int, [C.POINTER(BpProblem), C.c_int, C.c_int, _I, _V]),
    "rtkb_backproject_autotune": (C.c_int, [C.POINTER(BpProblem), C.c_int, C.c_int, C.c_int, _I, _D, _D, _V]),
    "rtkb_bp_batch_create": (C.c_int, [C.POINTER(BpProblem), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "rtkb_bp_batch_execute": (C.c_int, [_V, _V]),
    "rtkb_bp_batch_config": (C.c_int, [_V]),
    "rtkb_bp_batch_destroy": (None, [_V]),
})


class SartParams(C.Structure):
    """rtkb_sart_params."""

    _fields_ = [("niter", C.c_int), ("lam", C.c_double), ("positivity", C.c_int),
                ("projections_per_subset", C.c_int), ("disable_displaced_detector", C.c_int),
                ("division_threshold", C.c_double), ("order", C.POINTER(C.c_int)), ("seed", C.c_ulonglong)]


class OsemParams(C.Structure):
    """rtkb_osem_params."""

    _fields_ = [("niter", C.c_int), ("projections_per_subset", C.c_int), ("beta", C.c_double),
                ("store_normalization", C.c_int), ("backprojector", C.c_int), ("order", C.POINTER(C.c_int)),
                ("seed", C.c_ulonglong)]


class RegularizedCgParams(C.Structure):
    """rtkb_regularized_cg_params."""

    _fields_ = [("main_loop_iterations", C.c_int), ("cg_iterations", C.c_int), ("tikhonov", C.c_double),
                ("gamma", C.c_double), ("positivity", C.c_int), ("tv", C.c_int), ("gamma_tv", C.c_double),
                ("tv_iterations", C.c_int), ("tv_dimensions", C.POINTER(C.c_int)),
                ("soft_threshold_on_image", C.c_int), ("soft_threshold", C.c_double),
                ("disable_displaced_detector", C.c_int), ("support_mask", C.c_void_p)]


class I0Estimate(C.Structure):
    """rtkb_i0_estimate."""

    _fields_ = [("i0", C.c_double), ("i0_fwhm", C.c_double), ("imin", C.c_double), ("imax", C.c_double),
                ("low_bound", C.c_double), ("high_bound", C.c_double)]


class IterativeFdkParams(C.Structure):
    """rtkb_iterative_fdk_params."""

    _fields_ = [("niter", C.c_int), ("lam", C.c_double), ("positivity", C.c_int), ("fdk", FdkPreprocessParams)]
