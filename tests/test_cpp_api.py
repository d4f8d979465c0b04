"""The header-only C++ layer (include/rtkb200.hpp): a C++17 program that uses
it compiles against the C ABI and links librtkb200; host-side behaviour only
(geometry, geometry files, and the exceptions that argument checks raise
before any device work), so it runs without a GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r'''
#include "rtkb200.hpp"
#include <cstdio>
#include <string>

static int expect_throw(const char * what, void (*fn)(), const char * needle)
{
  try { fn(); }
  catch (const rtkb::Exception & e)
  {
    const bool ok = std::string(e.what()).find(needle) != std::string::npos;
    std::printf("%s: %s\n", what, ok ? "threw" : e.what());
    return ok ? 0 : 1;
  }
  std::printf("%s: no exception\n", what);
  return 1;
}

int main(int, char ** argv)
{
  rtkb::ThreeDCircularProjectionGeometry g;
  for (int i = 0; i < 4; i++)
    g.AddProjection(1000., 1500., 90. * i, 3., -2., 0., 0., 1., 0.5);
  std::printf("n %d\n", g.GetNumberOfProjections());
  const std::vector<double> m = g.GetMatrix(1);
  std::printf("m");
  for (double v : m)
    std::printf(" %.17g", v);
  std::printf("\n");
  g.Write(argv[1]);
  rtkb::ThreeDCircularProjectionGeometry r = rtkb::ThreeDCircularProjectionGeometry::Read(argv[1]);
  std::printf("read %d\n", r.GetNumberOfProjections());
  int bad = 0;
  bad += expect_throw("fdk without geometry", [] {
    const int sz[3] = { 8, 8, 8 }, ps[3] = { 8, 8, 4 };
    const double sp[3] = { 1., 1., 1. }, o[3] = { 0., 0., 0. };
    rtkb::FDKBackProjectionImageFilter f;
    f.SetVolume(rtkb::MakeImageDescription(sz, sp, o), nullptr, nullptr);
    f.SetProjections(rtkb::MakeImageDescription(ps, sp, o), nullptr);
    f.Update();
  }, "Geometry has not been set");
  bad += expect_throw("osem without buffers", [] {
    rtkb::ThreeDCircularProjectionGeometry h;
    h.AddProjection(1000., 1500., 0.);
    const int sz[3] = { 8, 8, 8 }, ps[3] = { 8, 8, 1 };
    const double sp[3] = { 1., 1., 1. }, o[3] = { 0., 0., 0. };
    rtkb::OSEMConeBeamReconstructionFilter f;
    f.SetGeometry(h);
    f.SetVolume(rtkb::MakeImageDescription(sz, sp, o), nullptr, nullptr);
    f.SetProjections(rtkb::MakeImageDescription(ps, sp, o), nullptr);
    f.Update();
  }, "null argument");
  bad += expect_throw("iterative fdk without buffers", [] {
    rtkb::ThreeDCircularProjectionGeometry h;
    h.AddProjection(1000., 1500., 0.);
    const int sz[3] = { 8, 8, 8 }, ps[3] = { 8, 8, 1 };
    const double sp[3] = { 1., 1., 1. }, o[3] = { 0., 0., 0. };
    rtkb::IterativeFDKConeBeamReconstructionFilter f;
    f.SetGeometry(h);
    f.SetHannCutFrequency(0.5);
    f.SetVolume(rtkb::MakeImageDescription(sz, sp, o), nullptr, nullptr);
    f.SetProjections(rtkb::MakeImageDescription(ps, sp, o), nullptr);
    f.Update();
  }, "null argument");
  bad += expect_throw("water precorrection without buffers", [] {
    const int sz[3] = { 4, 4, 2 };
    const double sp[3] = { 1., 1., 1. }, o[3] = { 0., 0., 0. };
    rtkb::WaterPrecorrectionImageFilter f;
    f.SetInput(rtkb::MakeImageDescription(sz, sp, o), nullptr);
    f.SetCoefficients({ 0.05, 0.3, 2.0 });
    f.Update();
  }, "null argument");
  bad += expect_throw("TV with no iterations", [] {
    const int sz[3] = { 4, 4, 2 };
    const double sp[3] = { 1., 1., 1. }, o[3] = { 0., 0., 0. };
    static float dummy[1];
    rtkb::TotalVariationDenoisingBPDQImageFilter f;
    f.SetInput(rtkb::MakeImageDescription(sz, sp, o), dummy);
    f.SetOutput(dummy);
    f.SetNumberOfIterations(0);
    f.Update();
  }, "niter >= 1");
  bad += expect_throw("I0 estimation with a bad bit shift", [] {
    const int sz[3] = { 4, 4, 1 };
    const double sp[3] = { 1., 1., 1. }, o[3] = { 0., 0., 0. };
    static unsigned short dummy[1];
    rtkb::I0EstimationProjectionFilter f;
    f.SetInput(rtkb::MakeImageDescription(sz, sp, o), dummy);
    f.SetBitShift(12);
    f.Update();
  }, "bit shift");
  bad += expect_throw("raw conversion with a non-finite I0", [] {
    const int sz[3] = { 4, 4, 1 };
    const double sp[3] = { 1., 1., 1. }, o[3] = { 0., 0., 0. };
    static unsigned short dummy[1];
    static float out[1];
    rtkb::LUTbasedVariableI0RawToAttenuationImageFilter f;
    f.SetInput(rtkb::MakeImageDescription(sz, sp, o), dummy);
    f.SetOutput(out);
    f.SetI0(1.0 / 0.0);
    f.Update();
  }, "finite");
  bad += expect_throw("mixed geometry", [] {
    rtkb::ThreeDCircularProjectionGeometry h;
    h.AddProjection(1000., 1500., 0.);
    h.AddProjection(1000., 0., 10.);
  }, "parallel");
  bad += expect_throw("missing file", [] { rtkb::ThreeDCircularProjectionGeometry::Read("/nonexistent/g.xml"); },
                      "ReadGeometry");
  std::printf("bad %d\n", bad);
  return bad;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_cpp_layer_compiles_and_behaves(tmp_path):
    import rtk_b200
    from rtk_b200 import build

    lib = build.build()
    src = tmp_path / "use_rtkb.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "use_rtkb"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
           lib, "-Wl,-rpath," + os.path.dirname(lib)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr
    run = subprocess.run([str(exe), str(tmp_path / "g.xml")], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stdout + run.stderr
    out = dict(line.split(" ", 1) for line in run.stdout.strip().splitlines() if " " in line)
    assert out["n"] == "4" and out["read"] == "4" and out["bad"] == "0"
    # the matrices are the C ABI's, as the Python binding reads them
    g = rtk_b200.ThreeDCircularProjectionGeometry()
    for i in range(4):
        g.AddProjection(1000.0, 1500.0, 90.0 * i, 3.0, -2.0, 0.0, 0.0, 1.0, 0.5)
    got = np.array([float(v) for v in out["m"].split()])
    np.testing.assert_array_equal(got, np.asarray(g.GetMatrix(1)).ravel())
