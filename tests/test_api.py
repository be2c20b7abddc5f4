"""The C ABI boundary: exported symbols, argument checking, statuses, pointer
kinds and NGA2's array layout with overlap layers."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from nga2_b200 import problems as P
from nga2_b200 import bbmg as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "bbmg_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bbmg_[a-z_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = B.load()
    names = header_functions()
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(B.EXPORTS) == sorted(names)


def test_default_params_are_the_ils_values():
    p = B.default_params()
    assert (p.method, p.precision, p.ncycle, p.relax_pre, p.relax_post, p.ncell_coarsest,
            p.use_direct_solve, p.maxit) == (B.PCG_BBOX, B.FP64, 1, 2, 2, 300, 1, 100)
    assert p.rcvg == 1e-10


def test_create_rejects_bad_arguments():
    lib = B.load()
    h = C.c_void_p()
    g = B.Grid(0, 8, 8, 1, 1, 1, 0)
    assert lib.bbmg_create(C.byref(g), None, C.byref(h)) == 4
    assert b"grid sizes" in lib.bbmg_last_error(None)
    g = B.Grid(8, 8, 8, 1, 1, 1, 0)
    p = B.default_params(); p.method = 7
    assert lib.bbmg_create(C.byref(g), C.byref(p), C.byref(h)) == 4
    assert not h.value


def test_null_handle_calls_fail_cleanly():
    lib = B.load()
    assert lib.bbmg_setup(None, 7, None, None) == 4
    assert lib.bbmg_solve(None, None, None, None, None) == 4
    assert lib.bbmg_destroy(None) == 0


def test_ils_requires_init_and_setup():
    ps = B.ILS(8, 8, 8, True, True, True)
    with pytest.raises(RuntimeError):
        ps.setup()
    with pytest.raises(RuntimeError):
        ps.solve()
    with pytest.raises(ValueError):
        ps.init(3)


# ---------------------------------------------------------------- GPU side
@pytest.mark.gpu
def test_status_codes():
    pb = P.periodic_poisson(16, seed=0)
    g = B.BBMG(16, 16, 16, 1, 1, 1)
    # solve before setup (ils_class.f90:684)
    _, _, _, st = g.solve(pb.rhs, allow=(5,))
    assert st == 5
    # stencil outside 3x3x3 (bbmg_class.f90:197)
    bad = pb.stc.copy(); bad[1] = [2, 0, 0]
    with pytest.raises(B.BBMGError) as e:
        g.setup(bad, pb.opr)
    assert e.value.code == 4
    g.setup(pb.stc, pb.opr)
    # maxit reached
    g.set_convergence(1, 1e-14)
    _, it, rerr, st = g.solve(pb.rhs, allow=(1,))
    assert st == 1 and it == 1 and rerr > 1e-14
    # NaN in the right-hand side
    g.set_convergence(100, 1e-10)
    r = pb.rhs.copy(); r[3, 4, 5] = np.nan
    _, it, rerr, st = g.solve(r, allow=(3,))
    assert st == 3
    # zero right-hand side: it = 0, rerr = 0 (bbmg_class.f90:630-633)
    _, it, rerr, st = g.solve(np.zeros_like(pb.rhs))
    assert st == 0 and it == 0 and rerr == 0.0
    # the handle still works after the failures
    x, it, rerr, st = g.solve(pb.rhs)
    assert st == 0 and rerr <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("ghost", [0, 1, 3])
def test_overlap_layers_and_device_pointers(ghost):
    """Caller arrays with NGA2's overlap layers, host and device memory give the
    same bits; the caller's overlap values of sol are left untouched."""
    import torch
    n = 16
    pb = P.drops_poisson(n, seed=2, ndrops=3, rmin=2.0, rmax=3.0)
    gsh = (n + 2 * ghost,) * 3
    opr = np.full(gsh + (7,), 7.0)
    rhs = np.full(gsh, -3.0)
    sl = (slice(ghost, ghost + n),) * 3
    opr[sl] = pb.opr
    rhs[sl] = pb.rhs
    ref = B.BBMG(n, n, n, 1, 0, 1)
    ref.setup(pb.stc, pb.opr)
    x0, it0, r0, _ = ref.solve(pb.rhs)
    g = B.BBMG(n, n, n, 1, 0, 1, ghost=ghost)
    g.setup(pb.stc, opr)
    sol = np.full(gsh, 5.0); sol[sl] = 0.0
    x, it, rerr, st = g.solve(rhs, sol)
    assert it == it0 and rerr == r0 and np.array_equal(x[sl], x0)
    mask = np.ones(gsh, bool); mask[sl] = False
    assert np.all(x[mask] == 5.0)
    # device pointers
    dopr = torch.from_numpy(opr).cuda()
    drhs = torch.from_numpy(rhs).cuda()
    dsol = torch.from_numpy(np.where(mask, 5.0, 0.0)).cuda()
    g.setup(pb.stc, dopr)
    _, it2, r2, _ = g.solve(drhs, dsol)
    torch.cuda.synchronize()
    xs = dsol.cpu().numpy()
    assert it2 == it0 and r2 == r0 and np.array_equal(xs[sl], x0)
    assert np.all(xs[mask] == 5.0)


@pytest.mark.gpu
def test_ils_interface_round_trip():
    n = 16
    pb = P.periodic_poisson(n, seed=9)
    ps = B.ILS(n, n, n, True, True, True, ghost=1, maxit=50, rcvg=1e-10)
    ps.stc[:] = pb.stc
    ps.opr[1:-1, 1:-1, 1:-1] = pb.opr
    ps.init(B.PCG_BBOX)
    ps.setup()
    ps.rhs[1:-1, 1:-1, 1:-1] = pb.rhs
    ps.sol[...] = 0.0
    ps.solve()
    assert 0 < ps.it < 20 and ps.rerr <= 1e-10
    ps.destroy()
