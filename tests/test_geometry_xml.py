"""RTK's geometry file (rtkb_geometry_read_xml / rtkb_geometry_write_xml):
src/rtkThreeDCircularProjectionGeometryXMLFileReader.cxx and ...Writer.cxx,
format in documentation/docs/Geometry.md:180-222.  The round-trip cases and
the 1e-13 tolerance are those of RTK's test/rtkgeometryfiletest.cxx; the
documented example file is tests/golden/geometry_example.xml (made by
tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import rtk_b200 as rtkb
from rtk_b200.geometry import read_geometry, write_geometry

HERE = os.path.dirname(os.path.abspath(__file__))
GETTERS = ["GetGantryAngles", "GetOutOfPlaneAngles", "GetInPlaneAngles", "GetSourceToIsocenterDistances",
           "GetSourceOffsetsX", "GetSourceOffsetsY", "GetSourceToDetectorDistances", "GetProjectionOffsetsX",
           "GetProjectionOffsetsY"]


def _write_read_check(g, path):
    write_geometry(g, path)
    r = read_geometry(path)
    assert len(r) == len(g)
    for name in GETTERS:
        np.testing.assert_allclose(getattr(r, name)(), getattr(g, name)(), rtol=0, atol=1e-13, err_msg=name)
    for i in range(len(g)):
        np.testing.assert_allclose(r.GetMatrix(i), g.GetMatrix(i), rtol=1e-12, atol=1e-9)
    return r


def test_rtkgeometryfiletest_cases(tmp_path):
    path = str(tmp_path / "g.xml")
    g = rtkb.ThreeDCircularProjectionGeometry()
    g.AddProjection(615., 548., 36., 1.3, 1.57, 15.4, 13.48, 5.42, 7.56)
    _write_read_check(g, path)
    g = rtkb.ThreeDCircularProjectionGeometry()
    for _ in range(5):
        g.AddProjection(615., 548., 36., 1.3, 1.57, 15.4, 13.48, 5.42, 7.56)
    _write_read_check(g, path)
    # equal parameters are written once, before the projections
    txt = open(path).read()
    assert txt.count("<SourceToIsocenterDistance>") == 1 and txt.count("<GantryAngle>") == 5
    g = rtkb.ThreeDCircularProjectionGeometry()
    g.AddProjection(615., 15., -8., 1.3, 1.57, 15.4, 13.48, 5.42, 7.56)
    g.AddProjection(354., 873., 3218., 354.4, 6587.1, .483, 384.4, 6874.4, 384.4)
    g.AddProjection(1869., 6987., 684., 681., -45.1, 6548.1, 6547., .214, .217)
    g.AddProjection(1532., 3218., 98732., -184.5, 548.1, -659.4, 123.4, 87.4, -15476.)
    g.AddProjection(578., 68., 9879., -38.4, 2158.4, -158.4, -43.3, 3218.4, 325.4)
    _write_read_check(g, path)
    assert open(path).read().count("<SourceToIsocenterDistance>") == 5


def test_defaults_are_not_written_and_collimation_round_trips(tmp_path):
    path = str(tmp_path / "g.xml")
    g = rtkb.geometry.circular(4, 1000.0, 1536.0)
    write_geometry(g, path)
    txt = open(path).read()
    assert '<RTKThreeDCircularGeometry version="3">' in txt
    for absent in ("ProjectionOffsetX", "InPlaneAngle", "SourceOffsetY", "Collimation", "RadiusCylindrical"):
        assert absent not in txt
    g.SetCollimationOfLastProjection(-10.0, 12.5, -3.0, 4.0)
    g.SetRadiusCylindricalDetector(1536.0)
    r = _write_read_check(g, path)
    assert np.all(r.GetCollimationUInf()[:3] == np.finfo(np.float64).max)
    assert r.GetCollimationUInf()[3] == -10.0 and r.GetCollimationVSup()[3] == 4.0
    assert "<RadiusCylindricalDetector>1536</RadiusCylindricalDetector>" in open(path).read()


def test_reads_the_documented_example():
    kat = json.load(open(os.path.join(HERE, "golden", "geometry_kat.json")))
    g = read_geometry(os.path.join(HERE, "golden", "geometry_example.xml"))
    assert len(g) == 2
    np.testing.assert_allclose(g.GetSourceToIsocenterDistances(), 1000.0)
    np.testing.assert_allclose(g.GetSourceToDetectorDistances(), 1536.0)
    for i, p in enumerate(kat["projections"]):
        np.testing.assert_allclose(np.degrees(g.GetGantryAngles()[i]), p["gantry_angle"], atol=1e-9)
        np.testing.assert_allclose(g.GetProjectionOffsetsX()[i], p["proj_offset_x"], atol=1e-12)
        # the reader already required agreement to 0.001; the recomputed matrix is much closer
        np.testing.assert_allclose(g.GetMatrix(i).ravel(), p["matrix"], rtol=1e-9, atol=1e-6)


def _example_text():
    return open(os.path.join(HERE, "golden", "geometry_example.xml")).read()


def test_inconsistent_matrix_is_an_error(tmp_path):
    bad = _example_text().replace("-117056.503295898", "-117056.553295898", 1)
    path = tmp_path / "bad.xml"
    path.write_text(bad)
    with pytest.raises(rtkb.RtkbError, match="not consistent"):
        read_geometry(str(path))


def test_versions_alias_and_inherited_parameters(tmp_path):
    path = tmp_path / "v.xml"
    path.write_text(_example_text().replace('version="3"', 'version="1"'))
    with pytest.raises(rtkb.RtkbError, match="Incompatible version"):
        read_geometry(str(path))
    # version 2 files read as version 3; <Angle> is GantryAngle's older name; a
    # parameter set before the projections applies to every following one
    path.write_text('<?xml version="1.0"?>\n<!DOCTYPE RTKGEOMETRY>\n<RTKThreeDCircularGeometry version="2">\n'
                    "<SourceToIsocenterDistance>800</SourceToIsocenterDistance>\n"
                    "<SourceToDetectorDistance>1200</SourceToDetectorDistance>\n"
                    "<ProjectionOffsetY>2.5</ProjectionOffsetY>\n"
                    "<Projection><Angle>10</Angle></Projection>\n"
                    "<Projection><GantryAngle>20</GantryAngle><ProjectionOffsetX>-3</ProjectionOffsetX>"
                    "</Projection>\n</RTKThreeDCircularGeometry>\n")
    g = read_geometry(str(path))
    np.testing.assert_allclose(np.degrees(g.GetGantryAngles()), [10.0, 20.0])
    np.testing.assert_allclose(g.GetProjectionOffsetsY(), [2.5, 2.5])
    np.testing.assert_allclose(g.GetProjectionOffsetsX(), [0.0, -3.0])
    np.testing.assert_allclose(g.GetSourceToIsocenterDistances(), [800.0, 800.0])


def test_missing_file_and_empty_geometry(tmp_path):
    with pytest.raises(rtkb.RtkbError):
        read_geometry(str(tmp_path / "none.xml"))
    with pytest.raises(rtkb.RtkbError, match="empty"):
        write_geometry(rtkb.ThreeDCircularProjectionGeometry(), str(tmp_path / "e.xml"))
