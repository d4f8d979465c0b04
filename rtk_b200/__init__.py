"""rtk_b200 -- B200-native (sm_100a) implementation of RTK's projector pair, FDK
and conjugate-gradient reconstructions.

The product is the C ABI library ``librtkb200.so`` (include/rtkb200.h): CUDA
kernels for sm_100a plus FP64 host geometry in C++.  This package is its thin
Python binding, mirroring the names of RTK's Python wrapping (``itk.RTK``):
``ThreeDCircularProjectionGeometry``, ``FDKBackProjectionImageFilter`` ...
PyTorch provides device memory and streams only.
"""
from ._capi import RtkbError, load  # noqa: F401
from .geometry import ThreeDCircularProjectionGeometry  # noqa: F401
from .image import Image, ImageDesc, make_desc  # noqa: F401
from . import ops  # noqa: F401

__version__ = "0.1.0"
