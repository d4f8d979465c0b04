"""Writes tests/golden/cg_c3_oracle.npz: the FP64 oracle's conjugate-gradient
reconstruction of the CG configuration (256^3 at 1 mm from 360 projections of
512 x 384 at 0.8 mm, SID 1000, SDD 1536, 20 random ellipsoids, Poisson noise
at I0 = 5e4), 3 iterations from zero with the Joseph pair, as RTK's
ConjugateGradientConeBeamReconstructionFilter computes it.

The oracle needs minutes for this size, so the GPU parity test compares with
this file instead of rerunning it.  Stored: every 8th voxel along each axis of
the iterate (32^3 values; a uniform sample for the relative L2 error), the
iterate's full FP64 norm, the squared residual norms, and two sums of the
input projections (the test regenerates the inputs and checks them first).

  python tests/golden/make_cg_c3_fixture.py [threads]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ITERATIONS = 3
STRIDE = 8


def main():
    from oracle import oracle as O

    O.build()
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else O.nthreads()
    t0 = time.time()
    from tests import workloads as W

    g, vol, proj, p = W.c3_oracle_problem(O)
    print(f"inputs: {time.time() - t0:.1f} s", flush=True)
    x, res = O.cg_joseph(g, vol, proj, p, ITERATIONS, threads=threads)
    print(f"oracle CG, {ITERATIONS} iterations: {time.time() - t0:.1f} s; residuals {res}", flush=True)
    np.savez_compressed(os.path.join(HERE, "cg_c3_oracle.npz"),
                        x_sample=x[::STRIDE, ::STRIDE, ::STRIDE].astype(np.float32),
                        x_norm=np.linalg.norm(x.ravel()), residuals=res, iterations=ITERATIONS, stride=STRIDE,
                        input_sum=p.sum(), input_sum_sq=(p * p).sum())
    print("wrote cg_c3_oracle.npz")


if __name__ == "__main__":
    main()
