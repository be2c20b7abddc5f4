"""Helper of tests/test_gpu_parity.py::test_staged_fp32_relax_matches_register_kernel:
run FP32 level-1 relaxation sweeps, a residual, a restriction, a
prolongation, level-2 (27-point) relaxation sweeps and a residual on a fixed
symmetric
problem, and an FP64 level-1 residual, and save the results, so the staged
and column-marching kernels and the register kernels
(BBMG_NO_STAGED) can be compared bit for bit across two processes."""
import sys

import numpy as np

from nga2_b200 import problems as P
from nga2_b200.bbmg import BBMG, FP64, MIXED, PCG_BBOX

n, out = int(sys.argv[1]), sys.argv[2]
pb = P.drops_poisson(n, seed=4, ndrops=6, rmin=2.0, rmax=5.0)  # n a power of 2: exactly symmetric
if n & (n - 1):
    # 1/n is not exact in binary: make W, S, B the E, N, T of the neighbours
    # exactly (periodic x and z wrap; the wall faces in y are zero both ways)
    o = pb.opr
    o[..., 2] = np.roll(o[..., 1], 1, axis=2)
    o[..., 4] = np.roll(o[..., 3], 1, axis=1)
    o[..., 6] = np.roll(o[..., 5], 1, axis=0)
g = BBMG(n, n, n, pb.xper, pb.yper, pb.zper, method=PCG_BBOX, precision=MIXED)
g.setup(pb.stc, pb.opr)
assert g.info["level1_stencil"] == 4
rng = np.random.default_rng(3)
shp = (n + 2, n + 2, n + 2)
g.put(1, "v", rng.standard_normal(shp), prec=1)
g.put(1, "f", rng.standard_normal(shp), prec=1)
for d in (1, -1, 1):
    g.step("relax", 1, d, prec=1)
g.step("residual", 1, 0, prec=1)
r1 = g.get(1, "r", prec=1)
g.step("restrict", 1, 0, prec=1)
f2 = g.get(2, "f", prec=1)
nx2, ny2, nz2 = g.level_dims(2)
g.put(2, "v", rng.standard_normal((nz2 + 2, ny2 + 2, nx2 + 2)), prec=1)
g.step("prolong", 1, 0, prec=1)
v1 = g.get(1, "v", prec=1)
# 27-point colours on level 2 (Galerkin operator)
g.put(2, "f", rng.standard_normal((nz2 + 2, ny2 + 2, nx2 + 2)), prec=1)
for d in (1, -1):
    g.step("relax", 2, d, prec=1)
g.step("residual", 2, 0, prec=1)
v2, r2 = g.get(2, "v", prec=1), g.get(2, "r", prec=1)
# FP64 level-1 residual (the column-marching kernel serves both precisions)
h = BBMG(n, n, n, pb.xper, pb.yper, pb.zper, method=PCG_BBOX, precision=FP64)
h.setup(pb.stc, pb.opr)
h.put(1, "v", rng.standard_normal(shp))
h.put(1, "f", rng.standard_normal(shp))
h.step("residual", 1, 0)
np.savez(out, v=v1, r=r1, f2=f2, v2=v2, r2=r2, r64=h.get(1, "r"))
