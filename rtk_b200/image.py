"""Images: a float32 buffer plus itk::ImageBase metadata (rtkb_image_desc)."""
from __future__ import annotations

import numpy as np

from ._capi import ImageDesc


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
