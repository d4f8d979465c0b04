"""The benchmark configurations as seeded synthetic inputs, shared by the
parity tests, the fixture scripts under tests/golden and bench.py.

  C1  plain FDK: Shepp-Logan (RTK's ellipsoids scaled to a 200 mm field,
      PhantomScale 100), 180 projections over 360 deg, SID 1000, SDD 1500,
      256 x 256 detector at 1.0 mm, pre-log Poisson noise at I0 = 1e5 (mu_ref
      0.01879 / mm, rtknoise's default), Hann ramp, 128^3 at 1.6 mm.
  C2  projector pair: 20 random ellipsoids, 720 projections of 1024 x 768 at
      0.388 mm, SID 1000, SDD 1536, 512^3 at 0.5 mm; displaced-detector
      (ProjectionOffsetX 80 mm) and 200 deg Parker short-scan variants with
      the same 720 projections.
  C3  CG: 256^3 at 1 mm, 360 projections of 512 x 384 at 0.8 mm, SID 1000,
      SDD 1536, 20 random ellipsoids, Poisson noise at I0 = 5e4.

No public dataset is named for these configurations; everything is generated
here from fixed seeds (the build's seed 20261203 plus the configuration
index)."""
from __future__ import annotations

import numpy as np

from tests import phantoms

SEED = 20261203

C1 = {"n": 180, "arc": 360.0, "sid": 1000.0, "sdd": 1500.0, "det": (256, 256), "pix": 1.0,
      "vol": (128, 128, 128), "vox": 1.6, "i0": 1e5, "mu_ref": 0.01879, "phantom_scale": 100.0}
C2 = {"n": 720, "sid": 1000.0, "sdd": 1536.0, "det": (1024, 768), "pix": 0.388, "vol": (512, 512, 512), "vox": 0.5,
      "displaced_offset": 80.0, "short_arc": 200.0}
C3 = {"n": 360, "sid": 1000.0, "sdd": 1536.0, "det": (512, 384), "pix": 0.8, "vol": (256, 256, 256), "vox": 1.0,
      "i0": 5e4}


def circular_params(n, sid, sdd, arc=360.0, pox=0.0, poy=0.0):
    """AddProjection arguments of n projections evenly spaced over arc."""
    return [(sid, sdd, i * arc / n, pox, poy) for i in range(n)]


def c1_projections(O, g, proj):
    """C1's noisy line integrals (FP64 values of float32 data) from the
    oracle's analytic projector of the Shepp-Logan phantom."""
    sl = phantoms.shepp_logan(C1["phantom_scale"])
    clean = O.project_ellipsoids(g, proj, sl)
    noisy = phantoms.poisson_noise(clean, C1["i0"], C1["mu_ref"], SEED + 0)
    return noisy.astype(np.float32).astype(np.float64), sl


def c2_ellipsoids():
    """C2's phantom: 20 ellipsoids, semi-axes 5-80 mm, centres in a 200 mm
    sphere, densities 0.1-1.0 (seed + 1)."""
    return phantoms.random_ellipsoids(20, SEED + 1, axis_range=(5.0, 80.0), centre_radius=100.0)


def c3_ellipsoids():
    """C3's phantom: 20 ellipsoids (semi-axes 5-60 mm, centres within 60 mm)
    with attenuations 0.002-0.02 / mm, so that the 256 mm field holds them."""
    ell = phantoms.random_ellipsoids(20, SEED + 2, centre_radius=60.0, axis_range=(5.0, 60.0))
    ell[:, 15] *= 0.02
    return ell


def c3_noise(clean):
    """C3's pre-log Poisson noise on analytic line integrals (attenuation
    units): counts Poisson(I0 exp(-p)) at I0 = 5e4 clamped to >= 1,
    p' = -log(counts / I0), as float32."""
    rng = np.random.default_rng(SEED + 3)
    counts = np.maximum(rng.poisson(C3["i0"] * np.exp(-np.asarray(clean, dtype=np.float64))), 1)
    return (-np.log(counts / C3["i0"])).astype(np.float32)


def c3_projections(O, g, proj):
    """C3's noisy projections (float32 values in an FP64 array) from the
    oracle's analytic projection of c3_ellipsoids, rounded to float32 before
    the noise (as the GPU's analytic projector stores it, so both give the
    same noisy stack)."""
    return c3_noise(O.project_ellipsoids(g, proj, c3_ellipsoids()).astype(np.float32)).astype(np.float64)


def c3_oracle_problem(O):
    """C3 for the oracle: geometry, volume and stack descriptions, noisy
    projections."""
    c = C3
    g = O.Geometry()
    for p in circular_params(c["n"], c["sid"], c["sdd"]):
        g.add_projection(*p)
    vol = O.image(c["vol"], (c["vox"],) * 3)
    proj = O.image((*c["det"], c["n"]), (c["pix"], c["pix"], 1.0))
    return g, vol, proj, c3_projections(O, g, proj)
