"""Helpers shared by the GPU parity tests."""
from __future__ import annotations

import numpy as np

# FP32 projections and volumes against the FP64 oracle: relative L2 error bound
# stated for this path (FP32 storage, FP32 arithmetic with FP64 geometry).
REL_L2_TOL = 1e-5


def rel_l2(a, ref) -> float:
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((a - ref).ravel()) / (den if den > 0 else 1.0))


def to_gpu(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def to_np(t) -> np.ndarray:
    import torch

    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def pair_geometry(rtkb, oracle, params):
    """Same projections in the product geometry and the oracle geometry."""
    gl = rtkb.ThreeDCircularProjectionGeometry()
    go = oracle.Geometry()
    for p in params:
        gl.AddProjection(*p)
        go.add_projection(*p)
    return gl, go


def pair_image(rtkb, oracle, size, spacing, origin=None, index=(0, 0, 0), direction=None):
    return (rtkb.make_desc(size, spacing, origin, index, direction),
            oracle.image(size, spacing, origin, index, direction))
