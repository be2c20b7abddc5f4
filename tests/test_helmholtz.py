"""The compressible two-phase pressure Helmholtz system (mast,
src/two_phase/mast_class.f90:3900-3960) through the same solver: a 7-point
operator with a positive diagonal shift 1/RHOSS2, hence nonsingular (no mean
removal, no pinned pivot in the coarsest LU), solved with pcg_bbox as mast's
``psolv`` is (ils_class.f90:184-198).

CPU tests check the generator and the oracle; the GPU tests hold the CUDA
solver to the oracle: bbox bit for bit, pcg_bbox and the mixed-precision
solver to 1e-10 residual and the oracle's solution.
"""
import numpy as np
import pytest

from nga2_b200 import problems as P
from nga2_b200.bbmg import BBOX, FP64, MIXED, PCG_BBOX
from oracle.oracle import OracleBBMG


def matvec(pb, x):
    o = pb.opr
    Ax = o[..., 0] * x
    Ax += o[..., 1] * np.roll(x, -1, 2) + o[..., 2] * np.roll(x, 1, 2)
    Ax += o[..., 3] * np.roll(x, -1, 1) + o[..., 4] * np.roll(x, 1, 1)
    Ax += o[..., 5] * np.roll(x, -1, 0) + o[..., 6] * np.roll(x, 1, 0)
    return Ax


CASES = [(24, (True, False, True), 3), (20, (False, False, False), 5), (16, (True, True, True), 7)]
IDS = [f"{n}-" + "".join("p" if p else "w" for p in per) for n, per, _ in CASES]


def small(n, per, seed):
    return P.helmholtz_mast(n, seed=seed, ndrops=4, rmin=2.0, rmax=4.0, per=per)


def test_generator_properties():
    """Row sums equal the diagonal shift 1/RHOSS2 (the Laplacian part sums to
    zero), which lies between the pure-phase values; off-diagonals are <= 0 and
    the operator is symmetric to round-off."""
    pb = small(24, (True, False, True), 3)
    o = pb.opr
    shift = o.sum(axis=-1)
    lo, hi = 1.0 / (1000.0 * 1500.0 ** 2), 1.0 / (1.0 * 340.0 ** 2)
    assert shift.min() > 0.9 * lo and shift.max() < 1.1 * hi
    assert (o[..., 1:] <= 0.0).all()
    assert np.abs(o[:, :, :-1, 1] - o[:, :, 1:, 2]).max() <= 1e-12 * np.abs(o[..., 1:]).max()
    assert np.abs(o[:, :-1, :, 3] - o[:, 1:, :, 4]).max() <= 1e-12 * np.abs(o[..., 1:]).max()
    # walls: no coupling through the y faces of the domain
    assert (o[:, 0, :, 4] == 0.0).all() and (o[:, -1, :, 3] == 0.0).all()
    assert pb.info["acoustic_cfl"][0] > 100.0


@pytest.mark.parametrize("n,per,seed", CASES, ids=IDS)
def test_oracle_solves_helmholtz(n, per, seed):
    """The oracle's pcg_bbox reaches 1e-10 and its solution satisfies A x = b
    by an independent numpy product; no coarse pivot is pinned (nonsingular)."""
    pb = small(n, per, seed)
    o = OracleBBMG(n, n, n, *per, method=PCG_BBOX, rcvg=1e-10, maxit=50)
    o.setup(pb.stc, pb.opr)
    x, it, rerr = o.solve(pb.rhs)
    assert rerr <= 1e-10 and it <= 15
    r = np.abs(pb.rhs - matvec(pb, x)).max() / np.abs(pb.rhs).max()
    assert r <= 2e-10, r
    assert o.npinned == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n,per,seed", CASES, ids=IDS)
def test_helmholtz_bbox_bitexact_gpu(n, per, seed):
    from nga2_b200.bbmg import BBMG
    pb = small(n, per, seed)
    o = OracleBBMG(n, n, n, *per, method=BBOX, rcvg=1e-10, maxit=60)
    o.setup(pb.stc, pb.opr)
    xo, ito, ro = o.solve(pb.rhs)
    g = BBMG(n, n, n, *per, method=BBOX, rcvg=1e-10, maxit=60)
    g.setup(pb.stc, pb.opr)
    xg, itg, rg, st = g.solve(pb.rhs)
    assert st == 0 and itg == ito and rg == ro and np.array_equal(xg, xo)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("n,per,seed", CASES, ids=IDS)
def test_helmholtz_pcg_gpu(n, per, seed, precision):
    from nga2_b200.bbmg import BBMG
    pb = small(n, per, seed)
    o = OracleBBMG(n, n, n, *per, method=PCG_BBOX, rcvg=1e-10, maxit=50)
    o.setup(pb.stc, pb.opr)
    xo, ito, ro = o.solve(pb.rhs)
    g = BBMG(n, n, n, *per, method=PCG_BBOX, precision=precision, rcvg=1e-10, maxit=50)
    g.setup(pb.stc, pb.opr)
    xg, itg, rg, st = g.solve(pb.rhs)
    assert st == 0 and rg <= 1e-10
    assert abs(itg - ito) <= (1 if precision == FP64 else 2)
    # nonsingular: the solution itself (no mean to remove) matches
    d = np.abs(xg - xo).max() / np.abs(xo).max()
    assert d < 1e-8, d
    r = np.abs(pb.rhs - matvec(pb, xg)).max() / np.abs(pb.rhs).max()
    assert r <= 2e-10, r
    g.close()
