"""Geometry: the oracle and the product's FP64 host geometry against RTK's
published known-answer matrices (documentation/docs/Geometry.md) and against
each other on irregular geometries (tilts, offsets, non-trivial image
directions and region indices)."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "geometry_kat.json")


def _kat():
    with open(GOLDEN) as f:
        return json.load(f)


def _check_matrix(m, ref):
    ref = np.asarray(ref).reshape(3, 4)
    scale = np.maximum(np.abs(ref), 1.0)
    assert np.all(np.abs(m - ref) / scale < 1e-10), (m, ref)


def test_oracle_geometry_kat(oracle):
    kat = _kat()
    g = oracle.Geometry()
    for p in kat["projections"]:
        g.add_projection(kat["sid"], kat["sdd"], p["gantry_angle"], p["proj_offset_x"], p["proj_offset_y"])
    for i, p in enumerate(kat["projections"]):
        _check_matrix(g.matrix(i), p["matrix"])


def test_product_geometry_kat(rtkb):
    kat = _kat()
    g = rtkb.ThreeDCircularProjectionGeometry()
    for p in kat["projections"]:
        g.AddProjection(kat["sid"], kat["sdd"], p["gantry_angle"], p["proj_offset_x"], p["proj_offset_y"])
    for i, p in enumerate(kat["projections"]):
        _check_matrix(g.GetMatrix(i), p["matrix"])


def _irregular(rng, n, lib_geom, orc_geom):
    params = []
    for _ in range(n):
        p = (rng.uniform(500, 1200), rng.uniform(1200, 1700), rng.uniform(-400, 400), rng.uniform(-60, 60),
             rng.uniform(-30, 30), rng.uniform(-20, 20), rng.uniform(-30, 30), rng.uniform(-20, 20),
             rng.uniform(-20, 20))
        lib_geom.AddProjection(*p)
        orc_geom.add_projection(*p)
        params.append(p)
    return params


def test_product_geometry_matches_oracle(rtkb, oracle):
    rng = np.random.default_rng(1)
    gl = rtkb.ThreeDCircularProjectionGeometry()
    go = oracle.Geometry()
    _irregular(rng, 40, gl, go)
    for i in range(40):
        np.testing.assert_allclose(gl.GetMatrix(i), go.matrix(i), rtol=1e-13, atol=1e-9)
        np.testing.assert_allclose(gl.GetSourcePosition(i), go.source_position(i), rtol=1e-13, atol=1e-9)
        np.testing.assert_allclose(gl.GetProjectionCoordinatesToFixedSystemMatrix(i), go.proj_coords_to_fixed(i),
                                   rtol=1e-13, atol=1e-9)
        for x in (-100.0, 0.0, 37.5):
            assert abs(gl.ToUntiltedCoordinateAtIsocenter(i, x) - go.to_untilted(i, x)) < 1e-9
    np.testing.assert_allclose(gl.GetSourceAngles(), go.source_angles(), atol=1e-12)
    np.testing.assert_allclose(gl.GetTiltAngles(), go.tilt_angles(), atol=1e-12)
    np.testing.assert_allclose(gl.GetGantryAngles(), go.gantry_angles(), atol=1e-12)
    np.testing.assert_allclose(gl.GetAngularGapsOfSourceAngles(), go.angular_gaps(go.source_angles()), atol=1e-12)


def test_angular_gaps_uniform(rtkb):
    g = rtkb.geometry.circular(90, 1000.0, 1500.0)
    np.testing.assert_allclose(g.GetAngularGapsOfSourceAngles(), np.full(90, 2 * np.pi / 90), atol=1e-12)


def test_parallel_divergent_mix_is_rejected(rtkb):
    g = rtkb.ThreeDCircularProjectionGeometry()
    g.AddProjection(1000.0, 1500.0, 0.0)
    with pytest.raises(rtkb.RtkbError, match="parallel projection"):
        g.AddProjection(1000.0, 0.0, 10.0)


def _eval(m, x):
    h = m @ np.append(x, 1.0)
    return h[0] / h[2], h[1] / h[2], 1.0 / (h[2] * h[2])


@pytest.mark.parametrize("kind", ["irregular", "circular", "parallel"])
@pytest.mark.parametrize("direction", ["identity", "perpendicular", "oblique"])
def test_backprojection_matrices_against_ray_plane_intersection(rtkb, oracle, direction, kind):
    """RTK's composed volume-index -> projection-index matrix
    (include/rtkBackProjectionImageFilter.hxx:535-595, FDK normalisation
    include/rtkFDKBackProjectionImageFilter.hxx:80-104), as the product builds
    it and as the oracle restates it, evaluated at voxel indices, against the
    oracle's independent derivation: the ray from the source through the
    voxel's physical position meets the detector plane (source position and
    detector frame), then the stack's physical-to-index map.  Volume and
    stack regions start at non-zero indices; directions are non-trivial."""
    import ctypes as C

    rng = np.random.default_rng(7)
    gl = rtkb.ThreeDCircularProjectionGeometry()
    go = oracle.Geometry()
    if kind == "irregular":
        _irregular(rng, 12, gl, go)
    else:
        for i in range(12):
            p = (1000.0, 0.0 if kind == "parallel" else 1536.0, i * 30.0 + 3.0, 12.0, -7.0, 0.0, 0.0, 5.0, -3.0)
            gl.AddProjection(*p)
            go.add_projection(*p)
    d = {"identity": np.eye(3), "perpendicular": np.array([[0, 1, 0], [-1, 0, 0], [0, 0, 1.0]]),
         "oblique": np.array([[np.cos(0.7), -np.sin(0.7), 0], [np.sin(0.7), np.cos(0.7), 0], [0, 0, 1.0]])}[direction]
    vd = rtkb.make_desc((20, 18, 16), (1.5, 1.2, 1.1), origin=(-13.0, -9.0, -8.0), index=(3, -2, 5), direction=d)
    pd = rtkb.make_desc((40, 30, 12), (1.3, 1.1, 1.0), origin=(-25.0, -16.0, 0.0), index=(-7, 4, 0))
    vo = oracle.image((20, 18, 16), (1.5, 1.2, 1.1), origin=(-13.0, -9.0, -8.0), index=(3, -2, 5), direction=d)
    po = oracle.image((40, 30, 12), (1.3, 1.1, 1.0), origin=(-25.0, -16.0, 0.0), index=(-7, 4, 0))
    i2p = oracle.index_to_physical(vo)
    idx = [np.array(v, dtype=np.float64) for v in ((3, -2, 5), (22, 15, 20), (10, 4, 11), (3, 15, 5))]
    for fdk in (0, 1):
        out = np.zeros(12 * 12)
        modes = np.zeros(12, dtype=np.int32)
        rtkb._capi.check(rtkb.load().rtkb_backprojection_matrices(
            gl.handle, C.byref(vd), C.byref(pd), 0, 12, fdk, out.ctypes.data_as(C.POINTER(C.c_double)),
            modes.ctypes.data_as(C.POINTER(C.c_int))))
        for i in range(12):
            m_orc, mode_orc = oracle.bp_matrix(go, vo, po, i, bool(fdk))
            m_prod = out[12 * i:12 * i + 12].reshape(3, 4)
            for x in idx:
                phys = (i2p @ np.append(x, 1.0))[:3]
                want, mode = oracle.bp_project(go, vo, po, i, bool(fdk), phys)
                for m in (m_prod, m_orc):
                    u, v, w2 = _eval(m, x)
                    assert abs(u - want[0]) < 1e-9 and abs(v - want[1]) < 1e-9, (u, v, want)
                    if fdk:
                        assert abs(w2 - want[2]) < 1e-12 * max(1.0, want[2]), (w2, want[2])
            assert modes[i] == mode and mode_orc == mode
            if kind != "irregular" and direction != "oblique":
                assert mode != 0  # circular and parallel stacks take RTK's optimised paths
