"""An FDK reconstruction driven by RTK's files: a geometry XML file and a
MetaImage projection stack written, read back (rtkb_geometry_read_xml,
rtkb_image_read_mha), reconstructed on the GPU, the volume written and read
again -- equal to the same reconstruction from the in-memory objects."""
import numpy as np
import pytest
import torch

import rtk_b200 as rtkb
from rtk_b200.geometry import read_geometry, write_geometry
from rtk_b200.image import make_desc, read_image, write_image
from tests import phantoms

pytestmark = pytest.mark.gpu


def _fdk(g, pdesc, p, vdesc):
    filtered, fdesc = rtkb.ops.fdk_preprocess(g, pdesc, p, rtkb.ops.ramp_params(hann=1.0))
    zero = torch.zeros((vdesc.size[2], vdesc.size[1], vdesc.size[0]), device="cuda")
    return rtkb.ops.fdk_backproject(g, vdesc, fdesc, filtered, zero)


def test_fdk_from_files_equals_in_memory(tmp_path):
    g = rtkb.geometry.circular(60, 1000.0, 1500.0, projOffsetX=3.0)
    pdesc = make_desc((128, 96, 60), (1.5, 1.5, 1.0))
    p = rtkb.ops.project_ellipsoids(g, pdesc, phantoms.shepp_logan(80.0))
    vdesc = make_desc((64, 64, 64), (2.0,) * 3)
    ref = _fdk(g, pdesc, p, vdesc)

    write_geometry(g, tmp_path / "geometry.xml")
    write_image(tmp_path / "projections.mha", p, pdesc, compress=True)
    g2 = read_geometry(tmp_path / "geometry.xml")
    p2, pdesc2 = read_image(tmp_path / "projections.mha")
    vol = _fdk(g2, pdesc2, torch.from_numpy(p2).cuda(), vdesc)
    write_image(tmp_path / "volume.mha", vol, vdesc)
    v2, vdesc2 = read_image(tmp_path / "volume.mha")
    assert rtkb.ops.device_status() == 0
    # the volume file holds exactly what was reconstructed; the geometry read
    # back from 15-digit text may differ from the original in the last bit of
    # an angle, so the reconstructions agree to FP32 rounding
    assert np.array_equal(v2, vol.cpu().numpy())
    r = ref.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(v2 - r) / np.linalg.norm(r) < 1e-6
    assert tuple(vdesc2.size) == (64, 64, 64)
    assert float(np.abs(v2).max()) > 0
