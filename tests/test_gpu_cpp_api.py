"""The header-only C++ layer (include/rtkb200.hpp) on a GPU: a C++ program
runs JosephForwardProjectionImageFilter, ConjugateGradientConeBeamReconstructionFilter,
FDKConeBeamReconstructionFilter and the FDKWeightProjectionFilter ->
FFTRampImageFilter chain (with the 2-D kernel of SetHannCutFrequencyY) on
device buffers it allocates itself; the results
equal those of the same entry points called through the Python binding."""
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

from tests.gpu_util import rel_l2, to_gpu, to_np

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")

PROGRAM = r'''
#include "rtkb200.hpp"
#include <cuda_runtime.h>
#include <cstdio>
#include <vector>

int main(int, char ** argv)
{
  const int nv = 24 * 20 * 22, np = 40 * 32 * 16;
  std::vector<float> vol(nv), proj(np), out(np), x(nv, 0.f);
  std::FILE * f = std::fopen(argv[1], "rb");
  if (!f || std::fread(vol.data(), 4, nv, f) != (size_t)nv || std::fread(proj.data(), 4, np, f) != (size_t)np)
    return 2;
  std::fclose(f);
  rtkb::ThreeDCircularProjectionGeometry g;
  for (int i = 0; i < 16; i++)
    g.AddProjection(600., 900., i * 22.5, 10., 0.);
  const int    vs[3] = { 24, 20, 22 }, ps[3] = { 40, 32, 16 };
  const double vsp[3] = { 6., 6., 6. }, psp[3] = { 4., 4., 1. };
  const double vo[3] = { -69., -57., -63. }, po[3] = { -78., -62., -7.5 };
  const rtkb_image_desc vd = rtkb::MakeImageDescription(vs, vsp, vo), pd = rtkb::MakeImageDescription(ps, psp, po);
  float *d_vol, *d_proj, *d_out, *d_x, *d_fdk, *d_filt, *d_w;
  if (cudaMalloc(&d_vol, nv * 4) || cudaMalloc(&d_proj, np * 4) || cudaMalloc(&d_out, np * 4) || cudaMalloc(&d_x, nv * 4) ||
      cudaMalloc(&d_fdk, nv * 4) || cudaMalloc(&d_filt, np * 4) || cudaMalloc(&d_w, np * 4))
    return 3;
  cudaMemset(d_fdk, 0, nv * 4);
  cudaMemcpy(d_vol, vol.data(), nv * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(d_proj, proj.data(), np * 4, cudaMemcpyHostToDevice);
  cudaMemset(d_out, 0, np * 4);
  cudaMemset(d_x, 0, nv * 4);
  try
  {
    rtkb::JosephForwardProjectionImageFilter fp;
    fp.SetGeometry(g);
    fp.SetVolume(vd, d_vol, nullptr);
    fp.SetProjections(pd, d_out, d_out);
    fp.Update();
    rtkb::ConjugateGradientConeBeamReconstructionFilter cg;
    cg.SetGeometry(g);
    cg.SetVolume(vd, d_x, d_x);
    cg.SetProjections(pd, d_proj);
    cg.SetNumberOfIterations(3);
    cg.SetDisableDisplacedDetectorFilter(true);
    cg.Update();
    rtkb::FDKConeBeamReconstructionFilter fdk;
    fdk.SetGeometry(g);
    fdk.SetVolume(vd, d_fdk, d_fdk);
    fdk.SetProjections(pd, d_proj);
    fdk.SetHannCutFrequency(0.8);
    fdk.SetFilteredProjectionsBuffer(d_filt);
    fdk.Update();
    rtkb::FDKWeightProjectionFilter w;
    w.SetGeometry(g);
    w.SetProjections(pd, d_proj, d_w);
    w.Update();
    rtkb::FFTRampImageFilter ramp;
    ramp.SetProjections(pd, d_w, d_w);
    ramp.SetHannCutFrequency(0.8);
    ramp.SetHannCutFrequencyY(0.5);
    ramp.Update();
  }
  catch (const rtkb::Exception & e)
  {
    std::printf("%s\n", e.what());
    return 4;
  }
  if (cudaDeviceSynchronize() != cudaSuccess)
    return 5;
  cudaMemcpy(out.data(), d_out, np * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(x.data(), d_x, nv * 4, cudaMemcpyDeviceToHost);
  std::vector<float> fdkv(nv), chain(np);
  cudaMemcpy(fdkv.data(), d_fdk, nv * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(chain.data(), d_w, np * 4, cudaMemcpyDeviceToHost);
  f = std::fopen(argv[2], "wb");
  std::fwrite(out.data(), 4, np, f);
  std::fwrite(x.data(), 4, nv, f);
  std::fwrite(fdkv.data(), 4, nv, f);
  std::fwrite(chain.data(), 4, np, f);
  std::fclose(f);
  return 0;
}
'''


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_cpp_layer_on_gpu_matches_python_binding(rtkb, tmp_path):
    from rtk_b200 import build

    lib = build.build()
    src = tmp_path / "cpp_gpu.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "cpp_gpu"
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"), str(src),
           "-o", str(exe), lib, "-Wl,-rpath," + os.path.dirname(lib), "-L", os.path.join(CUDA, "lib64"), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rng = np.random.default_rng(12)
    vol = rng.uniform(0.0, 1.0, size=(22, 20, 24)).astype(np.float32)
    proj = rng.uniform(0.0, 50.0, size=(16, 32, 40)).astype(np.float32)
    (tmp_path / "in.bin").write_bytes(vol.tobytes() + proj.tobytes())
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.join(CUDA, "lib64") + ":" + os.environ.get("LD_LIBRARY_PATH", ""))
    run = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                         text=True, timeout=120, env=env)
    assert run.returncode == 0, run.stdout + run.stderr
    data = np.frombuffer((tmp_path / "out.bin").read_bytes(), dtype=np.float32)
    fp_cpp, x_cpp = data[:proj.size].reshape(proj.shape), data[proj.size:proj.size + vol.size].reshape(vol.shape)
    fdk_cpp = data[proj.size + vol.size:proj.size + 2 * vol.size].reshape(vol.shape)
    chain_cpp = data[proj.size + 2 * vol.size:].reshape(proj.shape)

    g = rtkb.ThreeDCircularProjectionGeometry()
    for i in range(16):
        g.AddProjection(600.0, 900.0, i * 22.5, 10.0, 0.0)
    vd = rtkb.make_desc((24, 20, 22), (6.0,) * 3, origin=(-69.0, -57.0, -63.0))
    pd = rtkb.make_desc((40, 32, 16), (4.0, 4.0, 1.0), origin=(-78.0, -62.0, -7.5))
    fp = to_np(rtkb.ops.joseph_forward_project(g, vd, pd, to_gpu(vol), torch.zeros(proj.shape, device="cuda")))
    assert np.array_equal(fp_cpp, fp.astype(np.float32))
    x = torch.zeros(vol.shape, device="cuda")
    cg = rtkb.ops.ConjugateGradient(g, vd, pd, backprojector="voxel")  # the C++ filter's default, as RTK's
    cg.start(to_gpu(proj), x, displaced_detector=False)
    cg.iterate(3)
    assert rel_l2(x_cpp, to_np(x)) < 1e-5, rel_l2(x_cpp, to_np(x))
    ramp = rtkb.ops.ramp_params(hann=0.8)
    f, fd = rtkb.ops.fdk_preprocess(g, pd, to_gpu(proj), ramp)
    fdk = to_np(rtkb.ops.fdk_backproject(g, vd, fd, f, torch.zeros(vol.shape, device="cuda")))
    assert np.array_equal(fdk_cpp, fdk.astype(np.float32))
    chain = to_np(rtkb.ops.ramp_filter(pd, rtkb.ops.fdk_weight(g, pd, to_gpu(proj)),
                                       rtkb.ops.ramp_params(hann=0.8, hann_y=0.5)))
    assert np.array_equal(chain_cpp, chain.astype(np.float32))
