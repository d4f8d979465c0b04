"""CPU checks of the oracle's SART pieces (test infrastructure): the ray-box
length of RayBoxIntersectionImageFilter on rays whose answer is known."""
import numpy as np

from oracle import oracle as O


def test_ray_box_central_ray_is_the_box_extent():
    O.build()
    g = O.Geometry()
    g.add_projection(1000.0, 1500.0, 0.0)   # source on +z, detector plane at z = -500
    g.add_projection(1000.0, 1500.0, 90.0)  # source on +x
    vol = O.image((11, 7, 9), (2.0, 3.0, 4.0), origin=(-10.0, -9.0, -16.0))
    proj = O.image((5, 5, 2), (1.0, 1.0, 1.0), origin=(-2.0, -2.0, 0.0))
    rb = O.ray_box(g, vol, proj)
    # the centre pixel's ray runs along z (angle 0) or x (angle 90) through the box
    # SetBoxFromImage(vol, false) spans: (size - 1) x spacing
    np.testing.assert_allclose(rb[0, 2, 2], 8 * 4.0, rtol=1e-12)
    np.testing.assert_allclose(rb[1, 2, 2], 10 * 2.0, rtol=1e-12)
    assert np.all(rb >= 0)
