"""Runs of the stage kernels on the grids and launch shapes of the
checked-index test (tests/test_gpu_debug_bounds.py): small and ragged grids,
every boundary combination, every launch shape, single grids and a mixed
batch.  Run as a script it writes the final states and status words to an
npz file; the test runs it once under the checked-index library
(GOCEAN_DEBUG_BOUNDS=1) and once under the normal one."""

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "gpu-ocean_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GRIDS = [(5, 11, (2, 2, 2, 2)), (17, 6, (1, 2, 1, 2)), (131, 45, (1, 1, 1, 1)), (257, 9, (1, 2, 1, 2)),
         (300, 170, (2, 1, 2, 1)), (600, 131, (1, 1, 1, 1))]
SHAPES = [(0, 16), (1, 16), (2, 16), (3, 16), (4, 0), (5, 3), (6, 5), (7, 24), (8, 3), (8, 0)]
STEPS = 4


def run(out_path):
    import torch
    from SWESimulators import BatchedEnsemble, CDKLM16, Common, SyntheticCases as SC

    ctx = Common.CUDAContext()
    res = {}
    for nx, ny, bc in GRIDS:
        c = SC.grf(nx, ny=ny, dx=1000.0, bc=bc, r=3.0e-3, steps=STEPS)
        for shape, rows in SHAPES:
            sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
            sim._domain.set_launch(shape, rows)
            for _ in range(STEPS):
                sim.step(c.dt)
            key = "%dx%d_%s_s%d_r%d" % (nx, ny, "".join(map(str, bc)), shape, rows)
            res[key] = np.stack(sim.download())
            res[key + "_status"] = np.array(sim.status())
    for launch in ((5, 16, 0), (8, 6, 0), (8, 24, 0)):
        sims = []
        for k, (nx, ny, bc) in enumerate(GRIDS[2:]):
            c = SC.grf(nx, ny=ny, dx=1000.0, bc=(1, 2, 1, 2), seed_bathy=43000 + k, steps=1)
            sims.append(CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs()))
        b = BatchedEnsemble.BatchedCDKLM16(sims, launch=launch)
        b.advance(STEPS)
        torch.cuda.synchronize()
        for m, s in enumerate(sims):
            key = "batch_%d_%d_m%d" % (launch[0], launch[1], m)
            res[key] = np.stack(s.download())
            res[key + "_status"] = np.array(s.status())
    np.savez(out_path, **res)


if __name__ == "__main__":
    run(sys.argv[1])
