"""MetaImage files (rtkb_image_read_mha / rtkb_image_write_mha): the header
keys of ITK's MetaIO as RTK's applications write them, data inline (.mha) or
beside the header (.mhd + .raw / .zraw), zlib compression, byte order and the
scalar element types, converted to float32 on reading."""
import zlib

import numpy as np
import pytest

import rtk_b200 as rtkb
from rtk_b200.image import make_desc, read_image, write_image


def _desc_equal(a, b, origin_shift=(0.0, 0.0, 0.0)):
    assert tuple(a.size) == tuple(b.size)
    np.testing.assert_allclose(tuple(a.spacing), tuple(b.spacing))
    np.testing.assert_allclose(np.array(tuple(a.origin)), np.array(tuple(b.origin)) + origin_shift, atol=1e-12)
    np.testing.assert_allclose(tuple(a.direction), tuple(b.direction), atol=1e-15)


@pytest.mark.parametrize("ext,compress", [(".mha", False), (".mha", True), (".mhd", False), (".mhd", True)])
def test_round_trip(tmp_path, ext, compress):
    rng = np.random.default_rng(0)
    d = make_desc((13, 7, 5), (0.5, 0.75, 2.0), origin=(-3.0, 1.5, 10.0))
    a = rng.standard_normal((5, 7, 13)).astype(np.float32)
    path = tmp_path / ("vol" + ext)
    write_image(path, a, d, compress=compress)
    b, e = read_image(path)
    assert b.dtype == np.float32 and np.array_equal(a, b)
    _desc_equal(e, d)
    assert tuple(e.index) == (0, 0, 0)
    if ext == ".mhd":
        assert (tmp_path / ("vol" + (".zraw" if compress else ".raw"))).exists()


def test_index_and_direction(tmp_path):
    """A region with a non-zero index is written at the physical position of
    its first voxel; TransformMatrix lists the axis directions (the columns of
    the row-major direction matrix)."""
    c, s = np.cos(0.3), np.sin(0.3)
    rot = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    d = make_desc((4, 3, 2), (1.0, 2.0, 3.0), origin=(1.0, 2.0, 3.0), index=(2, -1, 5), direction=rot)
    a = np.arange(24, dtype=np.float32).reshape(2, 3, 4)
    path = tmp_path / "r.mha"
    write_image(path, a, d)
    header = open(path, "rb").read().split(b"ElementDataFile")[0].decode()
    tm = [float(x) for x in header.split("TransformMatrix =")[1].splitlines()[0].split()]
    np.testing.assert_allclose(np.array(tm).reshape(3, 3), rot.T, atol=1e-15)
    b, e = read_image(path)
    assert np.array_equal(a, b)
    first = np.array([1.0, 2.0, 3.0]) + rot @ (np.array([1.0, 2.0, 3.0]) * np.array([2, -1, 5]))
    np.testing.assert_allclose(tuple(e.origin), first, atol=1e-12)
    np.testing.assert_allclose(np.array(tuple(e.direction)).reshape(3, 3), rot, atol=1e-15)


def _header(ndims, dims, etype, msb=False, compressed=False, datafile="LOCAL"):
    return ("ObjectType = Image\nNDims = %d\nBinaryData = True\nBinaryDataByteOrderMSB = %s\nCompressedData = %s\n"
            "ElementSpacing = %s\nDimSize = %s\nElementType = %s\nElementDataFile = %s\n"
            % (ndims, "True" if msb else "False", "True" if compressed else "False",
               " ".join(["1"] * ndims), " ".join(str(x) for x in dims), etype, datafile)).encode()


@pytest.mark.parametrize("etype,dtype", [("MET_USHORT", ">u2"), ("MET_SHORT", "<i2"), ("MET_DOUBLE", ">f8"),
                                          ("MET_UCHAR", "u1"), ("MET_INT", "<i4"), ("MET_UINT", ">u4")])
def test_element_types_byte_orders_and_compression(tmp_path, etype, dtype):
    rng = np.random.default_rng(1)
    vals = rng.integers(0, 200, size=(3, 4, 5)).astype(dtype)
    msb = dtype.startswith(">")
    for compressed in (False, True):
        payload = vals.tobytes()
        if compressed:
            payload = zlib.compress(payload)
        path = tmp_path / f"t{int(compressed)}.mha"
        path.write_bytes(_header(3, (5, 4, 3), etype, msb, compressed) + payload)
        b, e = read_image(path)
        assert np.array_equal(b, vals.astype(np.float32))
        assert tuple(e.size) == (5, 4, 3)


def test_two_dimensional_detached_and_errors(tmp_path):
    vals = np.arange(12, dtype="<f4").reshape(3, 4)
    (tmp_path / "p.raw").write_bytes(vals.tobytes())
    (tmp_path / "p.mhd").write_bytes(_header(2, (4, 3), "MET_FLOAT", datafile="p.raw"))
    b, e = read_image(tmp_path / "p.mhd")
    assert tuple(e.size) == (4, 3, 1) and np.array_equal(b[0], vals)
    (tmp_path / "x.mha").write_bytes(_header(3, (2, 2, 2), "MET_LONG_LONG") + bytes(64))
    with pytest.raises(rtkb.RtkbError, match="unsupported ElementType"):
        read_image(tmp_path / "x.mha")
    (tmp_path / "s.mha").write_bytes(_header(3, (4, 4, 4), "MET_FLOAT") + bytes(16))
    with pytest.raises(rtkb.RtkbError, match="shorter"):
        read_image(tmp_path / "s.mha")
    with pytest.raises(rtkb.RtkbError, match=".mha or .mhd"):
        write_image(tmp_path / "v.nii", np.zeros((1, 1, 1), np.float32), make_desc((1, 1, 1)))
