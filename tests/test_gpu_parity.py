"""GPU parity: every stage of the CUDA solver against the CPU oracle.

FP64 stages are compared bit for bit (np.array_equal; the kernels keep the
reference's term order and use no FMA contraction).  The PCG's dot products are
parallel reductions on the GPU and sequential sums in the oracle, so pcg_bbox is
compared by iteration count and solution difference; the mixed-precision solver
by residual (<= 1e-10) and solution difference against the FP64 oracle.
"""
import os

import numpy as np
import pytest

from nga2_b200 import problems as P
from nga2_b200.bbmg import BBMG, BBOX, FP64, MIXED, PCG_BBOX
from oracle.oracle import OracleBBMG, fft_solve_periodic

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

CASES = [((8, 8, 8), (True, True, True)), ((12, 10, 9), (True, False, True)), ((9, 7, 5), (False, False, False)),
         ((17, 17, 17), (True, True, True)), ((32, 32, 1), (True, True, False)), ((10, 6, 12), (False, True, False)),
         ((13, 8, 11), (True, True, True)),
         # sizes whose coarse levels run as one fused cooperative launch
         ((16, 16, 16), (True, True, True)), ((24, 16, 24), (True, False, True)), ((20, 20, 20), (False, False, False))]
IDS = ["x".join(map(str, d)) + "-" + "".join("p" if p else "w" for p in per) for d, per in CASES]


def sync_np(a, per):
    """The reference's overlap copy (vsync on one rank) on a padded numpy array."""
    a = a.copy()
    if per[0]:
        a[:, :, -1] = a[:, :, 1]; a[:, :, 0] = a[:, :, -2]
    if per[1]:
        a[:, -1, :] = a[:, 1, :]; a[:, 0, :] = a[:, -2, :]
    if per[2]:
        a[-1, :, :] = a[1, :, :]; a[0, :, :] = a[-2, :, :]
    return a


def rand_vec(shape, per, rng):
    a = np.zeros(shape)
    a[1:-1, 1:-1, 1:-1] = rng.standard_normal((shape[0] - 2, shape[1] - 2, shape[2] - 2))
    return sync_np(a, per)


def make_pair(dims, per, method=BBOX, seed=7, full27=False, precision=FP64, **kw):
    stc, opr = P.random_operator(*dims, per, seed=seed, full27=full27)
    o = OracleBBMG(*dims, *per, method=method, **kw)
    o.setup(stc, opr)
    g = BBMG(*dims, *per, method=method, precision=precision, **kw)
    g.setup(stc, opr)
    return o, g


@pytest.mark.parametrize("full27", [False, True])
@pytest.mark.parametrize("dims,per", CASES, ids=IDS)
def test_setup_bitexact(dims, per, full27):
    """update(): operators, prolongation, restriction, A*P on every level and the
    dense coarsest matrix with its LU equal the oracle's bit for bit."""
    o, g = make_pair(dims, per, full27=full27, ncell_coarsest=0 if dims[0] < 12 else 300)
    assert g.nlvl == o.nlvl
    for n in range(1, o.nlvl + 1):
        assert g.level_dims(n) == o.level_dims(n)
        names = ["opr"] + (["c2f", "oprc2f"] if n < o.nlvl else []) + (["f2c"] if n > 1 else [])
        for w in names:
            a, b = g.get(n, w), o.get(n, w)
            assert np.array_equal(a, b), (n, w, np.abs(a - b).max())
    op, lu, piv = g.direct()
    OP, LU, PIV, info = o.direct()
    assert np.array_equal(op, OP) and np.array_equal(lu, LU) and np.array_equal(piv, PIV)


@pytest.mark.parametrize("dims,per", CASES, ids=IDS)
def test_solve_steps_bitexact(dims, per):
    """relax(+1/-1), get_residual, f2c, c2f+correction, direct_solve and a full
    cycle(1) from the same state equal the oracle bit for bit."""
    o, g = make_pair(dims, per, full27=(dims[2] == 11))
    rng = np.random.default_rng(1)
    nl = o.nlvl
    for n in range(1, nl + 1):
        nx, ny, nz = o.level_dims(n)
        shp = (nz + 2, ny + 2, nx + 2)
        v, f = rand_vec(shp, per, rng), rand_vec(shp, per, rng)
        for obj in (o, g):
            obj.put(n, "v", v); obj.put(n, "f", f)
        for d in (1, -1):
            o.relax(n, d); g.step("relax", n, d)
            assert np.array_equal(g.get(n, "v"), o.get(n, "v")), ("relax", n, d)
        o.residual(n); g.step("residual", n)
        assert np.array_equal(g.get(n, "r"), o.get(n, "r")), ("residual", n)
        if n < nl:
            o.restrict(n); g.step("restrict", n)
            assert np.array_equal(g.get(n + 1, "f"), o.get(n + 1, "f")), ("restrict", n)
            nxc, nyc, nzc = o.level_dims(n + 1)
            vc = rand_vec((nzc + 2, nyc + 2, nxc + 2), per, rng)
            o.put(n + 1, "v", vc); g.put(n + 1, "v", vc)
            o.prolong(n + 1)
            # the reference prolongs into r and then adds r to v (bbmg_class.f90:768-770)
            vo = o.get(n, "v") + o.get(n, "r")
            g.step("prolong", n)
            assert np.array_equal(g.get(n, "v"), vo), ("prolong", n)
    # coarsest direct solve
    nx, ny, nz = o.level_dims(nl)
    f = rand_vec((nz + 2, ny + 2, nx + 2), per, rng)
    o.put(nl, "f", f); g.put(nl, "f", f)
    o.direct_solve(); g.step("direct", nl)
    assert np.array_equal(g.get(nl, "v"), o.get(nl, "v"))
    # a whole V-cycle from level 1
    nx, ny, nz = o.level_dims(1)
    v, f = rand_vec((nz + 2, ny + 2, nx + 2), per, rng), rand_vec((nz + 2, ny + 2, nx + 2), per, rng)
    for obj in (o, g):
        obj.put(1, "v", v); obj.put(1, "f", f)
    o.cycle(1); g.step("cycle", 1)
    assert np.array_equal(g.get(1, "v"), o.get(1, "v"))


@pytest.mark.parametrize("dims,per", CASES, ids=IDS)
def test_bbox_solve_bitexact(dims, per):
    """Stationary V-cycles (mgsolve): same it, rerr and solution bits."""
    stc, opr = P.random_operator(*dims, per, seed=3)
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal(dims[::-1])
    rhs -= rhs.mean()
    o = OracleBBMG(*dims, *per, method=BBOX, maxit=30, rcvg=1e-10)
    o.setup(stc, opr)
    xo, ito, ro = o.solve(rhs)
    g = BBMG(*dims, *per, method=BBOX, maxit=30, rcvg=1e-10)
    g.setup(stc, opr)
    xg, itg, rg, st = g.solve(rhs)
    assert itg == ito and rg == ro
    assert np.array_equal(xg, xo)


@pytest.mark.parametrize("kind", ["asym7", "channel"])
def test_bbox_solve_bitexact_level1_layouts(kind):
    """The 7-plane (non-symmetric) level-1 layout; the symmetric 4-plane layout is
    what the uniform-grid cases above use."""
    if kind == "asym7":
        dims, per = (12, 10, 8), (True, False, True)
        stc, opr = P.random_operator(*dims, per, seed=5, asym=1e-3)
        rng = np.random.default_rng(5)
        rhs = rng.standard_normal(dims[::-1]); rhs -= rhs.mean()
    else:
        pb = P.channel_poisson(16, 16, 12, seed=5)
        dims, per, stc, opr, rhs = (16, 16, 12), (True, False, True), pb.stc, pb.opr, pb.rhs
    o = OracleBBMG(*dims, *per, method=BBOX, maxit=40, rcvg=1e-10)
    o.setup(stc, opr)
    xo, ito, ro = o.solve(rhs)
    g = BBMG(*dims, *per, method=BBOX, maxit=40, rcvg=1e-10)
    g.setup(stc, opr)
    assert g.info["level1_stencil"] == 7
    xg, itg, rg, st = g.solve(rhs)
    assert itg == ito and rg == ro and np.array_equal(xg, xo)


def test_symmetric_layout_selected():
    stc, opr = P.random_operator(8, 8, 8, (True, True, True), seed=1)
    g = BBMG(8, 8, 8, True, True, True)
    g.setup(stc, opr)
    assert g.info["level1_stencil"] == 4
    stc27, opr27 = P.random_operator(8, 8, 8, (True, True, True), seed=1, full27=True)
    g.setup(stc27, opr27)
    assert g.info["level1_stencil"] == 27


@pytest.mark.parametrize("dims,per", CASES, ids=IDS)
def test_pcg_solve(dims, per):
    """V-cycle preconditioned CG (cgsolve): the dot products are reduced in a
    different order, so iteration counts may differ by one and the solutions by
    round-off amplified through the iteration."""
    stc, opr = P.random_operator(*dims, per, seed=4)
    rng = np.random.default_rng(4)
    rhs = rng.standard_normal(dims[::-1]); rhs -= rhs.mean()
    o = OracleBBMG(*dims, *per, method=PCG_BBOX, maxit=50, rcvg=1e-10)
    o.setup(stc, opr)
    xo, ito, ro = o.solve(rhs)
    g = BBMG(*dims, *per, method=PCG_BBOX, maxit=50, rcvg=1e-10)
    g.setup(stc, opr)
    xg, itg, rg, st = g.solve(rhs)
    assert st == 0 and rg <= 1e-10
    assert abs(itg - ito) <= 1
    d = np.abs(P.remove_mean(xg) - P.remove_mean(xo)).max() / np.abs(P.remove_mean(xo)).max()
    assert d < 1e-8, d


@pytest.mark.parametrize("name", ["periodic16", "walls16", "drops24"])
def test_golden_fixtures_gpu(name):
    """The committed fixtures: bbox reproduces the oracle bits, pcg_bbox to 1e-8."""
    from tests.golden.make_golden import make_case
    ref = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    pb, m = make_case(name)
    g = BBMG(pb.nx, pb.ny, pb.nz, pb.xper, pb.yper, pb.zper, method=m, rcvg=1e-10)
    g.setup(pb.stc, pb.opr)
    x, it, rerr, st = g.solve(pb.rhs)
    if m == BBOX:
        assert it == int(ref["it"]) and rerr == float(ref["rerr"]) and np.array_equal(x, ref["sol"])
    else:
        assert abs(it - int(ref["it"])) <= 1 and rerr <= 1e-10
        xr = ref["sol"]
        assert np.abs(P.remove_mean(x) - P.remove_mean(xr)).max() <= 1e-8 * np.abs(xr).max()


@pytest.mark.parametrize("method", [BBOX, PCG_BBOX])
def test_mixed_precision_matches_fp64(method):
    """FP32 V-cycle inside the FP64 outer iteration reaches rerr <= 1e-10; its
    solution agrees with the FP64 oracle's after mean removal."""
    pb = P.drops_poisson(32, seed=5, ndrops=6, rmin=2.0, rmax=5.0)
    o = OracleBBMG(32, 32, 32, True, False, True, method=PCG_BBOX, rcvg=1e-12)
    o.setup(pb.stc, pb.opr)
    xo, _, _ = o.solve(pb.rhs)
    g = BBMG(32, 32, 32, True, False, True, method=method, precision=MIXED, rcvg=1e-10, maxit=60)
    g.setup(pb.stc, pb.opr)
    xg, it, rerr, st = g.solve(pb.rhs)
    assert st == 0 and rerr <= 1e-10, (st, it, rerr)
    d = np.abs(P.remove_mean(xg) - P.remove_mean(xo)).max() / np.abs(P.remove_mean(xo)).max()
    assert d < 1e-7, d


@pytest.mark.parametrize("precision", [FP64, MIXED])
@pytest.mark.parametrize("method", [BBOX, PCG_BBOX])
def test_periodic_64_known_answer(method, precision):
    """64^3 triply periodic Laplacian (the CPU-runnable configuration) against its
    exact FFT solution."""
    pb = P.periodic_poisson(64, seed=1)
    exact = fft_solve_periodic(pb.opr, pb.rhs)
    g = BBMG(64, 64, 64, True, True, True, method=method, precision=precision, rcvg=1e-10)
    g.setup(pb.stc, pb.opr)
    x, it, rerr, st = g.solve(pb.rhs)
    assert st == 0 and rerr <= 1e-10
    err = np.abs(P.remove_mean(x) - exact).max() / np.abs(exact).max()
    assert err < 1e-8, err


@pytest.mark.parametrize("precision", [FP64, MIXED])
@pytest.mark.parametrize("method", [BBOX, PCG_BBOX])
def test_residual_norm_rhs(method, precision):
    """NORM_RHS: a zero-guess solve is unchanged (max|r0| = max|b|); a guess
    near the solution stops as soon as max|r| <= rcvg max|b|, where the
    reference's rerr (relative to the guess's own residual) keeps iterating."""
    from nga2_b200.bbmg import NORM_GUESS, NORM_RHS
    pb = P.drops_poisson(24, seed=2, ndrops=4, rmin=2.0, rmax=4.0)
    g = BBMG(24, 24, 24, True, False, True, method=method, precision=precision, rcvg=1e-10)
    g.setup(pb.stc, pb.opr)
    x0, it0, rerr0, st0 = g.solve(pb.rhs)
    g.set_residual_norm(NORM_RHS)
    x1, it1, rerr1, st1 = g.solve(pb.rhs)
    assert (it1, st1) == (it0, st0) and rerr1 == rerr0 and np.array_equal(x0, x1)
    # warm start: the zero-guess solution with a 1e-6 relative perturbation
    rng = np.random.default_rng(0)
    guess = x0 + 1e-6 * np.abs(x0).max() * rng.standard_normal(x0.shape)
    _, it_rhs, rerr_rhs, st_rhs = g.solve(pb.rhs, guess.copy())
    g.set_residual_norm(NORM_GUESS)
    _, it_ref, rerr_ref, st_ref = g.solve(pb.rhs, guess.copy())
    # under the reference's rerr the guess's residual must drop another 1e-10,
    # which can lie below the FP64 floor: MAXIT is then the honest outcome
    assert st_rhs == 0 and rerr_rhs <= 1e-10 and st_ref in (0, 1)
    assert it_rhs < it_ref and it_rhs < it0, (it_rhs, it_ref, it0)


@pytest.mark.parametrize("n", [32, 48, 64])
def test_staged_fp32_relax_matches_register_kernel(n, tmp_path):
    """The shared-memory-staged FP32 kernels (level-1 residual, restriction and
    prolongation, 27-point colours and residual on level 2) give the same bits as the
    register kernels they replace (run in a second process with
    BBMG_NO_STAGED=1)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    probe = os.path.join(root, "tests", "fp32_relax_probe.py")
    env = dict(os.environ, PYTHONPATH=root)
    a, b = str(tmp_path / "staged.npz"), str(tmp_path / "register.npz")
    subprocess.run([sys.executable, probe, str(n), a], check=True, env=env)
    env["BBMG_NO_STAGED"] = "1"
    subprocess.run([sys.executable, probe, str(n), b], check=True, env=env)
    za, zb = np.load(a), np.load(b)
    for key in ("v", "r", "f2", "v2", "r2", "r64"):
        assert np.array_equal(za[key], zb[key]), key


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("n", [48, 64])
def test_pcg_solve_k_marching(n, precision):
    """Two-phase drops with walls in y: the level-1 residual and the CG
    direction/A*p step run as k-column marching kernels (symmetric 7-point
    level; at 48^3 the operator is symmetrised exactly and the blocks hold a
    non-power-of-two number of rows); the solve matches the oracle's pcg_bbox
    within the PCG tolerance."""
    pb = P.drops_poisson(n, seed=6, ndrops=8, rmin=2.0, rmax=6.0)
    if n & (n - 1):
        o7 = pb.opr
        o7[..., 2] = np.roll(o7[..., 1], 1, axis=2)
        o7[..., 4] = np.roll(o7[..., 3], 1, axis=1)
        o7[..., 6] = np.roll(o7[..., 5], 1, axis=0)
        pb.rhs -= pb.rhs.mean()
    per = (pb.xper, pb.yper, pb.zper)
    o = OracleBBMG(n, n, n, *per, method=PCG_BBOX, rcvg=1e-10)
    o.setup(pb.stc, pb.opr)
    xo, ito, ro = o.solve(pb.rhs)
    g = BBMG(n, n, n, *per, method=PCG_BBOX, precision=precision, rcvg=1e-10)
    g.setup(pb.stc, pb.opr)
    assert g.info["level1_stencil"] == 4
    xg, itg, rg, st = g.solve(pb.rhs)
    assert st == 0 and rg <= 1e-10
    assert abs(itg - ito) <= (1 if precision == FP64 else 2)
    d = np.abs(P.remove_mean(xg) - P.remove_mean(xo)).max() / np.abs(P.remove_mean(xo)).max()
    assert d < (1e-8 if precision == FP64 else 1e-7), d


def test_setup_reuse_across_stencils_bitexact():
    """One handle set up with a 27-point operator, then a 7-point one, then
    another 7-point one: the level-1 storage keeps only the planes the stencil
    writes (the rest is zeroed when the stencil changes), and every setup
    array still equals a fresh oracle's bit for bit."""
    dims, per = (16, 12, 10), (True, False, True)
    stc27, opr27 = P.random_operator(*dims, per, seed=11, full27=True)
    stc7a, opr7a = P.random_operator(*dims, per, seed=12)
    stc7b, opr7b = P.random_operator(*dims, per, seed=13)
    g = BBMG(*dims, *per, method=BBOX)
    for stc, opr in ((stc27, opr27), (stc7a, opr7a), (stc7b, opr7b)):
        g.setup(stc, opr)
        o = OracleBBMG(*dims, *per, method=BBOX)
        o.setup(stc, opr)
        for n in range(1, o.nlvl + 1):
            names = ["opr"] + (["c2f", "oprc2f"] if n < o.nlvl else []) + (["f2c"] if n > 1 else [])
            for w in names:
                assert np.array_equal(g.get(n, w), o.get(n, w)), (n, w)


def test_setup_repeated_stencil_entries_bitexact():
    """A caller stencil that names a slot more than once (the ils scatter adds
    the entries of one slot in stencil order, ils_class.f90:247-256): the
    general form of the scatter; every setup array equals the oracle's."""
    dims, per = (16, 12, 10), (True, False, True)
    stc7, opr7 = P.random_operator(*dims, per, seed=21)
    rng = np.random.default_rng(5)
    # the centre split in two entries, the east coupling in two, in that order
    a = rng.uniform(0.2, 0.8, size=opr7.shape[:-1])
    stc = np.concatenate([stc7, stc7[[0, 1]]]).astype(np.int32)
    opr = np.concatenate([opr7, np.zeros(opr7.shape[:-1] + (2,))], axis=-1)
    opr[..., 7] = (1.0 - a) * opr7[..., 0]
    opr[..., 0] = a * opr7[..., 0]
    opr[..., 8] = 0.5 * opr7[..., 1]
    opr[..., 1] = opr7[..., 1] - opr[..., 8]
    g = BBMG(*dims, *per, method=BBOX)
    g.setup(stc, opr)
    o = OracleBBMG(*dims, *per, method=BBOX)
    o.setup(stc, opr)
    for n in range(1, o.nlvl + 1):
        names = ["opr"] + (["c2f", "oprc2f"] if n < o.nlvl else []) + (["f2c"] if n > 1 else [])
        for w in names:
            assert np.array_equal(g.get(n, w), o.get(n, w)), (n, w)


def test_pageable_host_arrays_match_device():
    """Arrays larger than one 32 MB staging chunk: the operator, rhs and
    solution given as pageable numpy arrays (copied through the pinned staging
    ring by several host threads) give the same bits as device tensors."""
    import torch
    n = 176  # 43 MB per vector, 0.3 GB operator
    pb = P.drops_poisson(n, seed=3, ndrops=8, rmin=3.0, rmax=8.0)
    per = (pb.xper, pb.yper, pb.zper)
    g = BBMG(n, n, n, *per, method=PCG_BBOX, precision=MIXED, rcvg=1e-10)
    g.setup(pb.stc, np.array(pb.opr))
    xh, ith, rh, sth = g.solve(np.array(pb.rhs), np.zeros(pb.rhs.shape))
    g.setup(pb.stc, torch.from_numpy(pb.opr).cuda())
    xd = torch.zeros(pb.rhs.shape, dtype=torch.float64, device="cuda")
    _, itd, rd, std = g.solve(torch.from_numpy(pb.rhs).cuda(), xd)
    assert sth == std == 0 and ith == itd and rh == rd
    assert np.array_equal(xh, xd.cpu().numpy())
    g.close()


@pytest.mark.parametrize("method", [BBOX, PCG_BBOX])
def test_true_residual_report(method):
    """bbmg_info.true_rerr / l2_rerr: the solution's residual recomputed in FP64
    after the last iteration.  For FP64 bbox it is the residual the iteration
    itself ended with (same bits); for pcg_bbox it agrees with an independent
    numpy product; a zero rhs reports zeros (it = 0)."""
    pb = P.drops_poisson(24, seed=4, ndrops=4, rmin=2.0, rmax=4.0)
    per = (pb.xper, pb.yper, pb.zper)
    g = BBMG(24, 24, 24, *per, method=method, rcvg=1e-10)
    g.setup(pb.stc, pb.opr)
    x, it, rerr, st = g.solve(pb.rhs)
    inf = g.info
    o = pb.opr
    Ax = (o[..., 0] * x + o[..., 1] * np.roll(x, -1, 2) + o[..., 2] * np.roll(x, 1, 2)
          + o[..., 3] * np.roll(x, -1, 1) + o[..., 4] * np.roll(x, 1, 1)
          + o[..., 5] * np.roll(x, -1, 0) + o[..., 6] * np.roll(x, 1, 0))
    r = pb.rhs - Ax
    ref = np.abs(r).max() / np.abs(pb.rhs).max()
    if method == BBOX:
        assert inf["true_rerr"] == rerr
    assert abs(inf["true_rerr"] - ref) <= 1e-3 * ref, (inf["true_rerr"], ref)  # sums in another order
    l2 = np.linalg.norm(r) / np.linalg.norm(pb.rhs)
    assert abs(inf["l2_rerr"] - l2) <= 1e-3 * l2, (inf["l2_rerr"], l2)
    assert abs(inf["true_res"] - np.abs(r).max()) <= 1e-3 * np.abs(r).max()
    _, it0, rerr0, st0 = g.solve(np.zeros_like(pb.rhs))
    inf0 = g.info
    assert (it0, rerr0, st0) == (0, 0.0, 0) and inf0["true_rerr"] == 0.0 and inf0["l2_rerr"] == 0.0
