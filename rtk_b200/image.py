"""Images: a float32 buffer plus itk::ImageBase metadata (rtkb_image_desc)."""
from __future__ import annotations

import numpy as np

from ._capi import ImageDesc, check, load


def make_desc(size, spacing=(1.0, 1.0, 1.0), origin=None, index=(0, 0, 0), direction=None) -> ImageDesc:
    """Describe an ITK image; the origin defaults to centring it on 0 (as RTK's
    ConstantImageSource users usually do)."""
    d = ImageDesc()
    for a in range(3):
        d.size[a] = int(size[a])
        d.index[a] = int(index[a])
        d.spacing[a] = float(spacing[a])
        d.origin[a] = float(origin[a]) if origin is not None else -0.5 * (int(size[a]) - 1) * float(spacing[a])
    dm = np.eye(3) if direction is None else np.asarray(direction, dtype=np.float64).reshape(3, 3)
    for q in range(9):
        d.direction[q] = float(dm.flat[q])
    return d


def shape_of(d: ImageDesc):
    """numpy/torch shape (z, y, x) of a described image."""
    return (d.size[2], d.size[1], d.size[0])


class Image:
    """A 3-D float32 image: ``data`` (torch tensor on the GPU, shape z, y, x) and
    its ITK metadata ``desc``."""

    def __init__(self, data, desc: ImageDesc):
        if tuple(data.shape) != shape_of(desc):
            raise ValueError(f"data shape {tuple(data.shape)} does not match size {shape_of(desc)}")
        self.data = data
        self.desc = desc

    def GetLargestPossibleRegion(self):  # noqa: N802
        return tuple(self.desc.index), tuple(self.desc.size)

    def GetSpacing(self):  # noqa: N802
        return tuple(self.desc.spacing)

    def GetOrigin(self):  # noqa: N802
        return tuple(self.desc.origin)


def read_image(filename):
    """A MetaImage file (.mha / .mhd, any scalar element type) as (float32
    numpy array of shape (z, y, x), ImageDesc), as itk::ImageFileReader with
    MetaImageIO gives it to RTK."""
    import ctypes as C

    lib = load()
    d = ImageDesc()
    check(lib.rtkb_image_read_mha(str(filename).encode(), C.byref(d), None, 0))
    a = np.empty(shape_of(d), dtype=np.float32)
    check(lib.rtkb_image_read_mha(str(filename).encode(), C.byref(d), a.ctypes.data_as(C.c_void_p), a.size))
    return a, d


def write_image(filename, data, desc: ImageDesc, compress=False) -> None:
    """Write a float32 image (numpy array or torch tensor, shape (z, y, x)) as a
    MetaImage file (.mha, or .mhd with its .raw / .zraw beside it)."""
    import ctypes as C

    a = data.detach().cpu().numpy() if hasattr(data, "detach") else np.asarray(data)
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.shape != shape_of(desc):
        raise ValueError(f"data shape {a.shape} does not match size {shape_of(desc)}")
    check(load().rtkb_image_write_mha(str(filename).encode(), C.byref(desc), a.ctypes.data_as(C.c_void_p),
                                      int(compress)))
