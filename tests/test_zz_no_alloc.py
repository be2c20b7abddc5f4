"""bbmg_residual_norm_noalloc: the residual check for callers that cannot call
cudaMalloc (a flow solver whose device memory comes from its own pool
allocator, or a time loop that must not allocate because allocation can
synchronise the device).  It allocates nothing -- its scratch is a static device
array -- so it is checked against the existing entry point: the residual ratio
that bbmg_solve reports for a stationary FP64 solve from a zero initial guess
(max|b - A x| / max|b|) must come out the same, on two calls in a row with
different grids sharing the one scratch array.

This file is collected last (test_zz_...) so a failure here comes after every
other test has run; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from nga2_b200 import problems as P
from nga2_b200 import bbmg as B

pytestmark = pytest.mark.gpu

RTOL = 1e-13  # the FP64 path is bit-exact; a last-digit margin only


def _lib():
    lib = B.load()
    lib.bbmg_residual_norm_noalloc.argtypes = [C.POINTER(B.Grid), C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.bbmg_residual_norm_noalloc.restype = C.c_int
    return lib


def _case(kind):
    if kind == "drops":
        pb = P.drops_poisson(24, seed=3, ndrops=4, rmin=2.0, rmax=4.0)
        return pb, 1
    stc, opr = P.random_operator(16, 12, 10, (True, False, True), seed=9, asym=1e-3)
    rng = np.random.default_rng(9)
    rhs = rng.standard_normal((10, 12, 16)); rhs -= rhs.mean()
    return P.Problem("walls", 16, 12, 10, True, False, True, stc, opr, rhs, np.ones_like(rhs), 9), 2


def _padded(a, g):
    if g == 0:
        return np.ascontiguousarray(a)
    pad = [(g, g)] * 3 + ([(0, 0)] if a.ndim == 4 else [])
    return np.pad(a, pad, constant_values=7.0)  # overlap values must be ignored


def test_noalloc_matches_solver_residual_twice():
    import torch
    lib = _lib()
    for kind in ("drops", "walls"):  # two calls in a row, different grids, one shared scratch
        pb, g = _case(kind)
        per = (pb.xper, pb.yper, pb.zper)
        dopr = torch.from_numpy(_padded(pb.opr, g)).cuda()
        drhs = torch.from_numpy(_padded(pb.rhs, g)).cuda()
        dsol = torch.zeros_like(drhs)
        h = B.BBMG(pb.nx, pb.ny, pb.nz, *per, ghost=g, method=B.BBOX, maxit=30, rcvg=1e-10)
        h.setup(pb.stc, dopr)
        _, it, rerr, st = h.solve(drhs, dsol)
        torch.cuda.synchronize()
        assert it > 0
        grid = B.Grid(pb.nx, pb.ny, pb.nz, int(pb.xper), int(pb.yper), int(pb.zper), g)
        stc = np.ascontiguousarray(pb.stc, np.int32)
        out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
        rc = lib.bbmg_residual_norm_noalloc(C.byref(grid), stc.shape[0], stc.ctypes.data_as(C.POINTER(C.c_int)),
                                            dopr.data_ptr(), drhs.data_ptr(), dsol.data_ptr(), out.data_ptr(), None)
        assert rc == 0, lib.bbmg_last_error(None)
        torch.cuda.synchronize()
        rnorm, bnorm, ratio = out.tolist()
        assert bnorm == float(np.abs(pb.rhs).max())
        assert abs(ratio - rerr) <= RTOL * rerr, (kind, ratio, rerr)
        assert abs(rnorm / bnorm - rerr) <= RTOL * rerr
        h.close()


def test_noalloc_rejects_too_many_planes():
    import torch
    lib = _lib()
    grid = B.Grid(4, 4, 8193, 1, 1, 1, 0)
    stc = np.ascontiguousarray(P.STC7, np.int32)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.bbmg_residual_norm_noalloc(C.byref(grid), 7, stc.ctypes.data_as(C.POINTER(C.c_int)), buf.data_ptr(),
                                        buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert rc == 4
    assert b"8192" in lib.bbmg_last_error(None)


def test_noalloc_zero_rhs():
    """A zero rhs and a zero solution give out = (0, 0, 0), the rerr a zero-guess
    solve reports for it; a zero rhs with a nonzero residual gives +inf."""
    import torch
    lib = _lib()
    pb, g = _case("drops")
    grid = B.Grid(pb.nx, pb.ny, pb.nz, int(pb.xper), int(pb.yper), int(pb.zper), g)
    stc = np.ascontiguousarray(pb.stc, np.int32)
    dopr = torch.from_numpy(_padded(pb.opr, g)).cuda()
    zero = torch.zeros(tuple(d + 2 * g for d in (pb.nz, pb.ny, pb.nx)), dtype=torch.float64, device="cuda")
    sol = torch.rand(zero.shape, dtype=torch.float64, device="cuda")  # not in the null space
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    for x, want in ((zero, 0.0), (sol, float("inf"))):
        rc = lib.bbmg_residual_norm_noalloc(C.byref(grid), stc.shape[0], stc.ctypes.data_as(C.POINTER(C.c_int)),
                                            dopr.data_ptr(), zero.data_ptr(), x.data_ptr(), out.data_ptr(), None)
        assert rc == 0, lib.bbmg_last_error(None)
        torch.cuda.synchronize()
        assert out[1].item() == 0.0 and out[2].item() == want, out.tolist()
