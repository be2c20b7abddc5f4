"""Pins the CPU oracle (oracle/bbmg_oracle.c) before the GPU solver is checked against it.

The reference ships no tests or golden vectors for bbmg and cannot be compiled
here (Fortran 2008 + MPI + LAPACK), so the restatement is pinned by:
  * the exact discrete solution of the periodic constant-coefficient problem
    (FFT diagonalisation, the method of src/solver/fourier3d_class.f90);
  * the Galerkin identities R = P^T and A_c = P^T A P (bbmg_class.f90:1201-1303);
  * scipy's LAPACK dgesv on the dense coarsest matrix (bbmg_class.f90:913);
  * the level-count and coarsening rules of bbmg_class.f90:231-341, 584-589;
  * committed golden fixtures (tests/golden/, made by make_golden.py).
"""
import os

import numpy as np
import pytest
import scipy.linalg.lapack as lapack
import scipy.sparse as sp

from nga2_b200 import problems as P
from oracle.oracle import BBOX, PCG_BBOX, OracleBBMG, fft_solve_periodic

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _oracle_for(nx, ny, nz, per, method=PCG_BBOX, **kw):
    return OracleBBMG(nx, ny, nz, *per, method=method, **kw)


def _amat(o, n, per):
    """Sparse interior operator of level n (periodic wrap; non-periodic ghost
    couplings dropped: the overlap holds zeros)."""
    nx, ny, nz = o.level_dims(n)
    opr = o.get(n, "opr")
    rows, cols, vals = [], [], []
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                for q in range(27):
                    w = opr[k, j, i, q]
                    if w == 0.0:
                        continue
                    li, lj, lk = q % 3 - 1, (q // 3) % 3 - 1, q // 9 - 1
                    i2, j2, k2 = i + li, j + lj, k + lk
                    ok = True
                    for a, (v, nn, pp) in enumerate(((i2, nx, per[0]), (j2, ny, per[1]), (k2, nz, per[2]))):
                        if v < 1 or v > nn:
                            ok = ok and pp
                    if not ok:
                        continue
                    i2 = (i2 - 1) % nx; j2 = (j2 - 1) % ny; k2 = (k2 - 1) % nz
                    rows.append(((k - 1) * ny + j - 1) * nx + i - 1)
                    cols.append((k2 * ny + j2) * nx + i2)
                    vals.append(w)
    N = nx * ny * nz
    return sp.csr_matrix((vals, (rows, cols)), shape=(N, N))


def _pmat(o, n, per):
    """Sparse prolongation level n+1 -> n from the c2f weights (bbmg_class.f90:779-801)."""
    nxf, nyf, nzf = o.level_dims(n)
    nxc, nyc, nzc = o.level_dims(n + 1)
    c2f = o.get(n, "c2f")
    rows, cols, vals = [], [], []
    for fk in range(1, nzf + 1):
        for fj in range(1, nyf + 1):
            for fi in range(1, nxf + 1):
                ci, cj, ck = (fi + 1) // 2, (fj + 1) // 2, (fk + 1) // 2
                for s in range(8):
                    w = c2f[fk, fj, fi, s]
                    if w == 0.0:
                        continue
                    c = [ci + (s & 1), cj + ((s >> 1) & 1), ck + ((s >> 2) & 1)]
                    ok = True
                    for a, nn in enumerate((nxc, nyc, nzc)):
                        if c[a] < 1 or c[a] > nn:
                            ok = ok and per[a]
                    if not ok:
                        continue
                    c = [(c[0] - 1) % nxc, (c[1] - 1) % nyc, (c[2] - 1) % nzc]
                    rows.append(((fk - 1) * nyf + fj - 1) * nxf + fi - 1)
                    cols.append((c[2] * nyc + c[1]) * nxc + c[0])
                    vals.append(w)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nxf * nyf * nzf, nxc * nyc * nzc))


def _ref_levels(nx, ny, nz, ncell_coarsest=300):
    """bbmg_class.f90:231-341 and initialize (584-589), restated in Python."""
    def nl(n):
        k = 1
        while n > 2 ** (k - 1):
            k += 1
        return k
    lx, ly, lz = nl(nx), nl(ny), nl(nz)
    big = 10 ** 9
    n = min(lx if lx > 1 else big, ly if ly > 1 else big, lz if lz > 1 else big)
    if lx == ly == lz == 1:
        n = 1
    dims = [(nx, ny, nz)]
    for _ in range(1, n):
        a, b, c = dims[-1]
        dims.append((a // 2 + a % 2, b // 2 + b % 2, c // 2 + c % 2))
    for i, d in enumerate(dims):
        if d[0] * d[1] * d[2] <= ncell_coarsest:
            return dims[:i + 1]
    return dims


@pytest.mark.parametrize("dims", [(64, 64, 64), (256, 256, 256), (512, 512, 512), (17, 17, 17), (64, 64, 1),
                                  (256, 64, 64), (6, 7, 7), (1, 1, 1), (3, 40, 5)])
def test_level_hierarchy(dims):
    o = _oracle_for(*dims, (True, True, True)) if np.prod(dims) <= 64 ** 3 else None
    ref = _ref_levels(*dims)
    if o is not None:
        got = [o.level_dims(n) for n in range(1, o.nlvl + 1)]
        assert got == ref
    if dims == (256, 256, 256):
        assert ref[-1] == (4, 4, 4) and len(ref) == 7


@pytest.mark.parametrize("n,method,maxit_expect", [(32, BBOX, 20), (32, PCG_BBOX, 12)])
def test_periodic_known_answer(n, method, maxit_expect):
    pb = P.periodic_poisson(n, seed=3)
    exact = fft_solve_periodic(pb.opr, pb.rhs)
    o = _oracle_for(n, n, n, (True, True, True), method=method, rcvg=1e-12)
    o.setup(pb.stc, pb.opr)
    x, it, rerr = o.solve(pb.rhs)
    assert rerr <= 1e-12 and 0 < it <= maxit_expect
    err = np.abs(P.remove_mean(x) - exact).max() / np.abs(exact).max()
    assert err < 1e-10, err


def test_periodic_known_answer_64():
    """Config 1 (64^3) to 1e-10 with both methods, against the exact solution."""
    pb = P.periodic_poisson(64, seed=1)
    exact = fft_solve_periodic(pb.opr, pb.rhs)
    for method in (BBOX, PCG_BBOX):
        o = _oracle_for(64, 64, 64, (True, True, True), method=method, rcvg=1e-10)
        o.setup(pb.stc, pb.opr)
        x, it, rerr = o.solve(pb.rhs)
        assert rerr <= 1e-10
        err = np.abs(P.remove_mean(x) - exact).max() / np.abs(exact).max()
        assert err < 1e-9, (method, err)


CASES = [((8, 8, 8), (True, True, True)), ((12, 10, 9), (True, False, True)), ((9, 7, 5), (False, False, False)),
         ((16, 16, 1), (True, True, False)), ((10, 6, 12), (False, True, False))]


@pytest.mark.parametrize("dims,per", CASES)
def test_galerkin_identities(dims, per):
    stc, opr = P.random_operator(*dims, per, seed=7)
    o = _oracle_for(*dims, per, ncell_coarsest=0)
    o.setup(stc, opr)
    for n in range(1, o.nlvl):
        A = _amat(o, n, per)
        Pm = _pmat(o, n, per)
        Ac = _amat(o, n + 1, per)
        rap = (Pm.T @ A @ Pm).tocsr()
        scale = abs(A).max()
        assert abs(rap - Ac).max() <= 1e-12 * scale, n
        # R = P^T: f2c(r, c) = c2f((1-r)/2, 2c-1+r)
        f2c = o.get(n + 1, "f2c")
        c2f = o.get(n, "c2f")
        nxc, nyc, nzc = o.level_dims(n + 1)
        for ck in range(1, nzc + 1):
            for cj in range(1, nyc + 1):
                for ci in range(1, nxc + 1):
                    for q in range(27):
                        w = f2c[ck, cj, ci, q]
                        if w == 0.0:
                            continue
                        ri, rj, rk = q % 3 - 1, (q // 3) % 3 - 1, q // 9 - 1
                        pi, pj, pk = (1 - ri) // 2, (1 - rj) // 2, (1 - rk) // 2
                        assert w == c2f[2 * ck - 1 + rk, 2 * cj - 1 + rj, 2 * ci - 1 + ri, pi + 2 * pj + 4 * pk]


@pytest.mark.parametrize("dims,per", CASES[:3])
def test_coarse_operators_symmetric_zero_rowsum(dims, per):
    """A symmetric zero-row-sum fine operator stays so on every level."""
    stc, opr = P.random_operator(*dims, per, seed=11)
    o = _oracle_for(*dims, per, ncell_coarsest=0)
    o.setup(stc, opr)
    for n in range(1, o.nlvl + 1):
        A = _amat(o, n, per)
        s = np.abs(o.get(n, "opr")).sum(axis=-1).max()  # stencil magnitude of the level
        assert abs(A - A.T).max() <= 1e-13 * s
        if all(per) or n == 1:
            assert np.abs(np.asarray(A.sum(axis=1))).max() <= 1e-13 * s


def test_direct_solve_vs_lapack():
    """The coarsest LU solve agrees with LAPACK dgesv (nonsingular Helmholtz case)."""
    stc, opr = P.random_operator(16, 16, 16, (True, False, True), seed=5, diag_boost=0.05)
    o = _oracle_for(16, 16, 16, (True, False, True))
    o.setup(stc, opr)
    OP, LU, piv, info = o.direct()
    assert info == 0 and o.npinned == 0
    rng = np.random.default_rng(0)
    b = rng.standard_normal(OP.shape[0])
    x = o.direct_apply(b)
    _, _, xl, infol = lapack.dgesv(OP, b.copy())
    assert infol == 0
    assert np.abs(x - xl).max() <= 1e-12 * np.abs(xl).max()
    assert np.abs(OP @ x - b).max() <= 1e-12 * np.abs(b).max()


def test_singular_coarse_matrix_pinned():
    """Periodic problem: the coarsest matrix is singular; one pivot is pinned and the
    pinned solve still satisfies the consistent equations."""
    pb = P.periodic_poisson(16, seed=2)
    o = _oracle_for(16, 16, 16, (True, True, True))
    o.setup(pb.stc, pb.opr)
    OP, LU, piv, info = o.direct()
    assert o.npinned == 1
    rng = np.random.default_rng(1)
    b = rng.standard_normal(OP.shape[0]); b -= b.mean()
    x = o.direct_apply(b)
    assert np.abs(OP @ x - b).max() <= 1e-10 * np.abs(b).max()


def test_dgesv_semantics_option():
    """pin_singular=False keeps DGESV's behaviour: division by the round-off pivot."""
    pb = P.periodic_poisson(16, seed=2)
    o = _oracle_for(16, 16, 16, (True, True, True), method=PCG_BBOX, pin_singular=False, maxit=200)
    o.setup(pb.stc, pb.opr)
    assert o.npinned == 0
    x, it, rerr = o.solve(pb.rhs)
    assert it >= 1


@pytest.mark.parametrize("name", ["periodic16", "walls16", "drops24"])
def test_golden_fixtures(name):
    """The oracle reproduces the committed fixtures bit for bit."""
    from tests.golden.make_golden import make_case
    ref = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    pb, method = make_case(name)
    assert P_hash(pb) == str(ref["problem_sha"])
    o = _oracle_for(pb.nx, pb.ny, pb.nz, (pb.xper, pb.yper, pb.zper), method=method, rcvg=1e-10)
    o.setup(pb.stc, pb.opr)
    x, it, rerr = o.solve(pb.rhs)
    assert it == int(ref["it"]) and rerr == float(ref["rerr"])
    assert np.array_equal(x, ref["sol"])


def P_hash(pb):
    from tests.golden.make_golden import problem_sha
    return problem_sha(pb)


def test_pivots_of_high_contrast_singular_coarse_matrix():
    """The first step of the two-phase drop sequence at 128^3 (triply periodic,
    density ratio 1000): the 4^3 coarsest matrix is singular; its round-off
    pivot (~2e-14 of the largest) must be pinned, and it must be the only one
    (the genuine pivots stay above 1e-3 of the largest)."""
    import torch
    from nga2_b200 import sequence as SQ
    seq = SQ.DropSequence(128, seed=5, noise=1e-3)
    oprs = []
    seq.step(lambda opr, rhs: (oprs.append(opr.numpy().copy()), torch.zeros_like(rhs))[1])
    o = OracleBBMG(128, 128, 128, True, True, True, method=PCG_BBOX, release=True)
    o.setup(P.STC7, oprs[0])
    _, LU, _, _ = o.direct()
    d = np.sort(np.abs(np.diag(LU)))
    assert o.npinned == 1
    assert d[0] / d[-1] < 1e-12 and d[1] / d[-1] > 1e-3
