"""The C ABI library loads without a GPU, exports every symbol declared in
include/rtkb200.h, and validates arguments before touching the device."""
import ctypes as C
import subprocess

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(rtkb):
    from rtk_b200 import _capi

    declared = _capi.header_symbols()
    assert len(declared) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    lib = rtkb.load()
    for s in declared:
        assert getattr(lib, s) is not None
    # every declared function has a ctypes signature in the binding
    assert set(declared) <= set(_capi.SIGNATURES), set(declared) - set(_capi.SIGNATURES)


def test_version(rtkb):
    assert b"sm_100a" in rtkb.load().rtkb_version()


def test_invalid_arguments_fail_before_device_work(rtkb):
    lib = rtkb.load()
    vd = rtkb.make_desc((8, 8, 8))
    pd = rtkb.make_desc((16, 16, 4))
    # no geometry
    rc = lib.rtkb_fdk_backproject(None, C.byref(vd), C.byref(pd), None, None, None, None)
    assert rc == rtkb._capi.RTKB_ERR_INVALID_ARGUMENT
    assert b"Geometry" in lib.rtkb_last_error()
    # geometry shorter than the stack
    g = rtkb.geometry.circular(2, 1000.0, 1500.0)
    rc = lib.rtkb_fdk_backproject(g.handle, C.byref(vd), C.byref(pd), None, None, None, None)
    assert rc == rtkb._capi.RTKB_ERR_INVALID_ARGUMENT
    assert b"Mismatch" in lib.rtkb_last_error()
    # zero spacing
    bad = rtkb.make_desc((8, 8, 8), (1.0, 0.0, 1.0))
    g4 = rtkb.geometry.circular(4, 1000.0, 1500.0)
    rc = lib.rtkb_voxel_backproject(g4.handle, C.byref(bad), C.byref(pd), None, None, None, None)
    assert rc == rtkb._capi.RTKB_ERR_INVALID_ARGUMENT
    # cylindrical detectors are rejected like RTK's voxel-based backprojector
    g4.SetRadiusCylindricalDetector(1500.0)
    rc = lib.rtkb_fdk_backproject(g4.handle, C.byref(vd), C.byref(pd), None, None, None, None)
    assert rc == rtkb._capi.RTKB_ERR_UNSUPPORTED


def test_matrix_entry_rejects_non_finite(rtkb):
    lib = rtkb.load()
    vs = (C.c_int * 3)(4, 4, 4)
    ps = (C.c_int * 3)(8, 8, 1)
    m = np.full(12, np.nan)
    modes = np.array([2], dtype=np.int32)
    dummy = C.c_void_p(16)
    rc = lib.rtkb_backproject_matrices(vs, ps, 1, m.ctypes.data_as(C.POINTER(C.c_double)),
                                       modes.ctypes.data_as(C.POINTER(C.c_int)), 1, dummy, dummy, dummy, None)
    assert rc == rtkb._capi.RTKB_ERR_INVALID_ARGUMENT


def test_ops_refuse_cpu_tensors(rtkb):
    torch = pytest.importorskip("torch")
    g = rtkb.geometry.circular(4, 1000.0, 1500.0)
    vd = rtkb.make_desc((8, 8, 8))
    pd = rtkb.make_desc((16, 16, 4))
    with pytest.raises(TypeError, match="CUDA"):
        rtkb.ops.fdk_backproject(g, vd, pd, torch.zeros(4, 16, 16), torch.zeros(8, 8, 8))


def test_i0_estimation_refuses_an_empty_image(rtkb):
    """RTK's histogram search reads past the histogram only when every bin is
    empty, i.e. for an image without pixels; the entry point refuses those
    before any device work."""
    lib = rtkb.load()
    empty = rtkb.make_desc((0, 16, 1))
    out = rtkb._capi.I0Estimate()
    rc = lib.rtkb_i0_estimation(C.byref(empty), C.c_void_p(16), 2, 20, C.byref(out), None)
    assert rc == rtkb._capi.RTKB_ERR_INVALID_ARGUMENT
    assert b"positive" in lib.rtkb_last_error()
