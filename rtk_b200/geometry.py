"""rtk.ThreeDCircularProjectionGeometry over the C ABI (FP64 geometry in C++).

Method names and argument meaning follow
src/rtkThreeDCircularProjectionGeometry.cxx (AddProjection :56-77 in degrees,
AddProjectionInRadians :79-153, getters :407-663).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._capi import check, load


class ThreeDCircularProjectionGeometry:
    def __init__(self):
        self._lib = load()
        self._g = self._lib.rtkb_geometry_new()
        if not self._g:
            raise MemoryError("rtkb_geometry_new failed")

    @classmethod
    def New(cls):  # noqa: N802  (ITK naming)
        return cls()

    def __del__(self):
        g = getattr(self, "_g", None)
        if g:
            try:
                self._lib.rtkb_geometry_free(g)
            except Exception:
                pass
            self._g = None

    @property
    def handle(self):
        return self._g

    # ---- construction ----
    def AddProjection(self, sid, sdd, gantryAngle, projOffsetX=0.0, projOffsetY=0.0,  # noqa: N802,N803
                      outOfPlaneAngle=0.0, inPlaneAngle=0.0, sourceOffsetX=0.0, sourceOffsetY=0.0):  # noqa: N803
        check(self._lib.rtkb_geometry_add_projection(self._g, sid, sdd, gantryAngle, projOffsetX, projOffsetY,
                                                     outOfPlaneAngle, inPlaneAngle, sourceOffsetX, sourceOffsetY))

    def AddProjectionInRadians(self, sid, sdd, gantryAngle, projOffsetX=0.0, projOffsetY=0.0,  # noqa: N802,N803
                               outOfPlaneAngle=0.0, inPlaneAngle=0.0, sourceOffsetX=0.0,  # noqa: N803
                               sourceOffsetY=0.0):  # noqa: N803
        check(self._lib.rtkb_geometry_add_projection_in_radians(self._g, sid, sdd, gantryAngle, projOffsetX,
                                                                projOffsetY, outOfPlaneAngle, inPlaneAngle,
                                                                sourceOffsetX, sourceOffsetY))

    def SetRadiusCylindricalDetector(self, r):  # noqa: N802
        check(self._lib.rtkb_geometry_set_radius_cylindrical_detector(self._g, r))

    def SetCollimationOfLastProjection(self, uinf, usup, vinf, vsup):  # noqa: N802
        check(self._lib.rtkb_geometry_set_collimation_of_last_projection(self._g, uinf, usup, vinf, vsup))

    # ---- getters ----
    def __len__(self):
        return self._lib.rtkb_geometry_number_of_projections(self._g)

    def GetNumberOfProjections(self):  # noqa: N802
        return len(self)

    def GetMatrix(self, i):  # noqa: N802
        m = np.zeros(12)
        check(self._lib.rtkb_geometry_get_matrix(self._g, i, m.ctypes.data_as(C.POINTER(C.c_double))))
        return m.reshape(3, 4)

    def GetMatrices(self):  # noqa: N802
        return [self.GetMatrix(i) for i in range(len(self))]

    def GetSourcePosition(self, i):  # noqa: N802
        s = np.zeros(4)
        check(self._lib.rtkb_geometry_get_source_position(self._g, i, s.ctypes.data_as(C.POINTER(C.c_double))))
        return s

    def GetProjectionCoordinatesToFixedSystemMatrix(self, i):  # noqa: N802
        m = np.zeros(16)
        check(self._lib.rtkb_geometry_get_projection_coordinates_to_fixed_system_matrix(
            self._g, i, m.ctypes.data_as(C.POINTER(C.c_double))))
        return m.reshape(4, 4)

    def _param(self, which):
        out = np.zeros(max(1, len(self)))
        check(self._lib.rtkb_geometry_get_parameters(self._g, which, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[: len(self)]

    def GetGantryAngles(self):  # noqa: N802
        return self._param(0)

    def GetSourceAngles(self):  # noqa: N802
        return self._param(1)

    def GetTiltAngles(self):  # noqa: N802
        return self._param(2)

    def GetOutOfPlaneAngles(self):  # noqa: N802
        return self._param(3)

    def GetInPlaneAngles(self):  # noqa: N802
        return self._param(4)

    def GetSourceToIsocenterDistances(self):  # noqa: N802
        return self._param(5)

    def GetSourceToDetectorDistances(self):  # noqa: N802
        return self._param(6)

    def GetProjectionOffsetsX(self):  # noqa: N802
        return self._param(7)

    def GetProjectionOffsetsY(self):  # noqa: N802
        return self._param(8)

    def GetSourceOffsetsX(self):  # noqa: N802
        return self._param(9)

    def GetSourceOffsetsY(self):  # noqa: N802
        return self._param(10)

    def GetAngularGapsOfSourceAngles(self):  # noqa: N802
        return self._param(11)

    def GetCollimationUInf(self):  # noqa: N802
        return self._param(12)

    def GetCollimationUSup(self):  # noqa: N802
        return self._param(13)

    def GetCollimationVInf(self):  # noqa: N802
        return self._param(14)

    def GetCollimationVSup(self):  # noqa: N802
        return self._param(15)

    def ToUntiltedCoordinateAtIsocenter(self, i, tilted):  # noqa: N802
        return self._lib.rtkb_geometry_to_untilted_coordinate_at_isocenter(self._g, i, tilted)


def read_geometry(filename) -> ThreeDCircularProjectionGeometry:
    """rtk::ReadGeometry: a geometry from an RTK XML geometry file."""
    g = ThreeDCircularProjectionGeometry.__new__(ThreeDCircularProjectionGeometry)
    g._lib = load()
    h = C.c_void_p()
    check(g._lib.rtkb_geometry_read_xml(str(filename).encode(), C.byref(h)))
    g._g = h.value
    return g


def write_geometry(geometry, filename) -> None:
    """rtk::ThreeDCircularProjectionGeometryXMLFileWriter: write an RTK XML geometry file."""
    check(geometry._lib.rtkb_geometry_write_xml(geometry.handle, str(filename).encode()))


def circular(n_proj, sid, sdd, arc_deg=360.0, first_deg=0.0, **kw) -> ThreeDCircularProjectionGeometry:
    """n_proj projections uniform over arc_deg (RTK's rtksimulatedgeometry)."""
    g = ThreeDCircularProjectionGeometry()
    for i in range(n_proj):
        g.AddProjection(sid, sdd, first_deg + i * arc_deg / n_proj, **kw)
    return g
