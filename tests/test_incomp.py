"""The incompressible time loops on the GPU (nga2_b200/incomp.py): the kernels
of a sub-iteration (nga_proj_midpoint, nga_proj_advance, nga_proj_flow_stats,
nga_proj_mom_residual, nga_proj_apply_residual, nga_proj_bulk) against the
numpy oracle, and whole time steps of the turbulence example
(examples/hit/src/simulation.f90) and of the channel example
(examples/channel/src/simulation.f90, walls and implicit solves) against the
oracle's restatements of the same loops.

CPU: the oracle loops keep the velocity divergence-free, the linear forcing
holds the turbulence's kinetic energy and the bulk forcing the channel's bulk
velocity nearer their targets than the unforced loops; the timetracker's dt
rule.  GPU: midpoint, advance, residual and update bit for bit; the
statistics' maxima bit for bit and sums to round-off; three time steps of
each loop to the solvers' tolerance.
"""
import numpy as np
import pytest

from nga2_b200 import problems as P
from oracle import projection_oracle as PO


def oracle_solver(n, rcvg=1e-12):
    from oracle.oracle import OracleBBMG, PCG_BBOX
    o = OracleBBMG(n, n, n, True, True, True, method=PCG_BBOX, rcvg=rcvg)
    state = {"opr": None}

    def solve(opr, rhs):
        if state["opr"] is None or not np.array_equal(state["opr"], opr):
            o.setup(P.STC7, opr)
            state["opr"] = opr.copy()
        return o.solve(rhs)[0]
    return solve


def test_oracle_hit_stays_solenoidal_and_forced():
    n = 12
    h = PO.HITOracle(n, oracle_solver(n), seed=1)
    free = PO.HITOracle(n, oracle_solver(n), seed=1, forcing=False)
    G = h.G
    d0 = np.abs(G.interior(PO.divergence(G, h.U, h.V, h.W)[0])).max()
    for _ in range(4):
        h.step()
        free.step()
        div = np.abs(G.interior(PO.divergence(G, h.U, h.V, h.W)[0])).max()
        assert div < 1e-9 * 5.0 * n, div
    ke = PO.flow_stats(G, h.U, h.V, h.W, h.visc, h.rho, 1.0)[6]
    ke_free = PO.flow_stats(G, free.U, free.V, free.W, free.visc, free.rho, 1.0)[6]
    assert ke_free < ke < h.KE0, (ke_free, ke, h.KE0)
    assert d0 < 1e-9 * 5.0 * n


def test_timetracker_adjust_dt():
    from nga2_b200.incomp import TimeTracker
    t = TimeTracker(dtmax=1e-3, cflmax=0.9)
    t.cfl = 1.8
    t.adjust_dt()
    assert t.dt == 1e-3 * 0.9 / 1.8          # decreases at once
    t.cfl = 0.45
    t.adjust_dt()                            # wants 1e-3 (capped), damped by alpha = 0.7
    assert t.dt == 0.7 * 1e-3 + (1.0 - 0.7) * 5e-4
    t.increment()
    assert (t.n, t.it) == (1, 1) and t.t == t.dt


# ----------------------------------------------------------------------------- GPU
def padded_fields(G, rng, k=3):
    return [G.sync(rng.standard_normal(G.padded)) for _ in range(k)]


@pytest.mark.gpu
@pytest.mark.parametrize("dims,g", [((12, 10, 9), 1), ((8, 8, 8), 2)])
def test_midpoint_and_advance_bitexact(dims, g):
    import torch
    from nga2_b200.projection import Projection
    nx, ny, nz = dims
    xn, yn, zn = P.uniform_nodes(nx), P.uniform_nodes(ny, 2.0), P.uniform_nodes(nz, 0.5)
    G = PO.Grid(xn, yn, zn, (True, True, True), g)
    pr = Projection(xn, yn, zn, True, True, True, ghost=g, device=0)
    rng = np.random.default_rng(5)
    U, Uo, dU = padded_fields(G, rng), padded_fields(G, rng), padded_fields(G, rng)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    tU, tUo = [T(a) for a in U], [T(a) for a in Uo]
    pr.midpoint(*tU, *tUo)
    mid = [PO.midpoint(a, b) for a, b in zip(U, Uo)]
    for a, b in zip(tU, mid):
        assert np.array_equal(a.cpu().numpy(), b)
    tdU = [T(a) for a in dU]
    for rho, fa, mean in ((1.0, 0.0, None), (998.2, 2.3e-3, (0.1, -0.2, 0.3))):
        t = [x.clone() for x in tU]
        pr.advance(7e-4, rho, *t, *tUo, *tdU, force_a=fa, force_b=0.2, mean=mean)
        for c in range(3):
            ref = PO.advance(7e-4, rho, mid[c], Uo[c], dU[c], fa, 0.2, 0.0 if mean is None else mean[c])
            assert np.array_equal(t[c].cpu().numpy(), ref), (rho, c)
    pr.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,g", [((12, 10, 9), 1), ((16, 16, 16), 2)])
def test_flow_stats(dims, g):
    import torch
    from nga2_b200.projection import Projection
    nx, ny, nz = dims
    xn = P.uniform_nodes(nx)
    yn = 0.5 * (1.0 - np.cos(np.pi * np.arange(ny + 1) / ny))  # stretched
    zn = P.uniform_nodes(nz, 3.0)
    G = PO.Grid(xn, yn, zn, (True, True, True), g)
    pr = Projection(xn, yn, zn, True, True, True, ghost=g, device=0)
    rng = np.random.default_rng(6)
    U, V, W = padded_fields(G, rng)
    visc = G.sync(np.exp(rng.uniform(-6.0, -2.0, size=G.padded)))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for vis, v0, rho, dt in ((visc, 0.0, 1.0, 1e-3), (None, 2e-3, 998.2, 3e-4)):
        ref = PO.flow_stats(G, U, V, W, vis if vis is not None else np.full(G.padded, v0), rho, dt)
        s = pr.flow_stats(T(U), T(V), T(W), visc=None if vis is None else T(vis), visc0=v0, rho=rho, dt=dt)
        got = np.array(list(s.values()))
        assert np.array_equal(got[:6], ref[:6])
        assert np.abs(got[6:] - ref[6:]).max() <= 1e-13 * np.abs(ref[6:]).max()
    pr.close()


@pytest.mark.gpu
@pytest.mark.parametrize("forcing", [True, False])
def test_hit_steps_match_oracle(forcing):
    """Initial projection and three time steps (two sub-iterations each) of
    the turbulence example on the GPU against the oracle loop: the solves
    are PCG to 1e-12 on both sides (reductions in different orders), so the
    fields agree to the solver's tolerance, not bit for bit."""
    from nga2_b200.incomp import HIT
    n = 16
    ref = PO.HITOracle(n, oracle_solver(n), seed=2, forcing=forcing)
    h = HIT(n=n, seed=2, rcvg=1e-12, forcing=forcing)
    assert abs(h.KE0 - ref.KE0) <= 1e-10 * ref.KE0
    for s in range(3):
        its = h.step()
        ref.step()
        assert len(its) == 2 and all(0 < i < 100 for i in its)
        assert h.time.dt == pytest.approx(ref.dt, rel=1e-12)
        for a, b in ((h.fs.U, ref.U), (h.fs.V, ref.V), (h.fs.W, ref.W), (h.fs.P, ref.P)):
            b = np.asarray(b)
            d = np.abs(a.cpu().numpy() - b).max() / np.abs(b).max()
            assert d < 1e-9, (s, d)
    G = ref.G
    div = G.interior(h.fs.div.cpu().numpy())
    assert np.abs(div).max() < 1e-8
    h.close()


@pytest.mark.gpu
def test_incomp_sequence_records():
    """The turbulence sequence from the GPU time loop: one record per
    pressure solve, each solve's solution is the next one's p_prev, dp
    solves opr dp = rhs (up to the periodic null space), and the velocity
    stays divergence-free."""
    import torch
    from nga2_b200.sequence import IncompSequence
    n = 24
    seq = IncompSequence(n, seed=4)
    recs = [seq.step() for _ in range(6)]
    assert [r["step"] for r in recs] == list(range(6))
    assert seq.nu > 0.0 and seq.time.n == 3
    for a, b in zip(recs, recs[1:]):
        assert torch.equal(b["p_prev"], a["dp"])
    for r in recs:
        o, x, b = r["opr"].cpu().numpy(), r["dp"].cpu().numpy(), r["rhs"].cpu().numpy()
        Ax = o[..., 0] * x
        Ax += o[..., 1] * np.roll(x, -1, 2) + o[..., 2] * np.roll(x, 1, 2)
        Ax += o[..., 3] * np.roll(x, -1, 1) + o[..., 4] * np.roll(x, 1, 1)
        Ax += o[..., 5] * np.roll(x, -1, 0) + o[..., 6] * np.roll(x, 1, 0)
        res = (b - b.mean()) - Ax
        assert np.abs(res).max() <= 1e-8 * np.abs(b).max()
    div = seq.fs.interior(seq.fs.div).abs().max().item()
    assert div < 1e-8
    seq.close()


def test_oracle_channel_stays_solenoidal():
    from oracle.oracle import OracleBBMG, BBOX
    nx, ny, nz = 12, 10, 6
    ov = OracleBBMG(nx, ny, nz, True, False, True, method=BBOX, rcvg=1e-12, maxit=200)

    def solve_v(opr, rhs):
        ov.setup(P.STC7, np.ascontiguousarray(opr))
        return ov.solve(rhs)[0]
    ch = PO.ChannelOracle(nx, ny, nz, oracle_solver_walls(nx, ny, nz), solve_v, Lz=0.5, amp=0.1)
    G = ch.G
    for _ in range(2):
        ch.step()
        assert np.abs(G.interior(PO.divergence(G, ch.U, ch.V, ch.W)[0])).max() < 1e-9
    # the no-slip faces stay at rest
    assert np.abs(ch.V[:, G.g, :]).max() == 0.0 and np.abs(ch.U[:, :G.g, :]).max() == 0.0


def oracle_solver_walls(nx, ny, nz, rcvg=1e-12):
    from oracle.oracle import OracleBBMG, PCG_BBOX
    o = OracleBBMG(nx, ny, nz, True, False, True, method=PCG_BBOX, rcvg=rcvg)
    state = {"set": False}

    def solve(opr, rhs):
        if not state["set"]:
            o.setup(P.STC7, opr)
            state["set"] = True
        return o.solve(rhs)[0]
    return solve


@pytest.mark.gpu
def test_channel_steps_match_oracle():
    """Three time steps of the channel example (walls in y, stretched grid,
    perturbed bulk flow) on the GPU against the oracle loop: implicit and
    pressure solves to 1e-12 on both sides (reductions in different orders),
    so the fields agree to the solvers' tolerance."""
    from oracle.oracle import OracleBBMG, BBOX
    from nga2_b200.incomp import Channel
    nx, ny, nz = 16, 12, 8
    ov = OracleBBMG(nx, ny, nz, True, False, True, method=BBOX, rcvg=1e-12, maxit=200)

    def solve_v(opr, rhs):
        ov.setup(P.STC7, np.ascontiguousarray(opr))
        return ov.solve(rhs)[0]
    import torch
    kw = dict(Lz=0.5, amp=0.1)
    ref = PO.ChannelOracle(nx, ny, nz, oracle_solver_walls(nx, ny, nz), solve_v, **kw)
    ch = Channel(nx, ny, nz, rcvg=1e-12, implicit_rcvg=1e-12, implicit_maxit=200, **kw)
    G = ref.G
    assert np.array_equal(ch.fs.U.cpu().numpy(), ref.U) and np.array_equal(ch.fs.W.cpu().numpy(), ref.W)
    # the example's perturbation is aliased on so coarse a grid: start both from
    # the same random (non-solenoidal) field, no-slip faces at rest
    rng = np.random.default_rng(44)
    for c, (name, base) in enumerate((("U", 1.0), ("V", 0.0), ("W", 0.0))):
        a = G.sync(base + 0.3 * rng.standard_normal(G.padded))
        a = np.where(PO.face_mask(G, c), 0.0, a)
        setattr(ref, name, a)
        getattr(ch.fs, name).copy_(torch.from_numpy(a))
    for s in range(3):
        its = ch.step()
        ref.step()
        assert len(its) == 2 and all(0 < i < 100 for i in its)
        assert ch.time.dt == pytest.approx(ref.dt, rel=1e-12)
        vs = max(np.abs(ref.U).max(), np.abs(ref.V).max(), np.abs(ref.W).max())
        for a, b, scale in ((ch.fs.U, ref.U, vs), (ch.fs.V, ref.V, vs), (ch.fs.W, ref.W, vs),
                            (ch.fs.P, ref.P, np.abs(ref.P).max())):
            d = np.abs(a.cpu().numpy() - b).max() / scale
            assert d < 1e-9, (s, d)
    div = ref.G.interior(ch.fs.div.cpu().numpy())
    assert np.abs(div).max() < 1e-8
    ch.close()


@pytest.mark.gpu
def test_residual_update_and_bulk_kernels():
    """k_mom_residual and k_apply_residual equal the oracle bit for bit over
    the padded arrays (walls in y and z, forcing on U and W); the bulk sums
    agree to round-off."""
    import torch
    from nga2_b200.projection import Projection
    nx, ny, nz, g = 10, 9, 8, 2
    xn, yn, zn = P.uniform_nodes(nx, 2.0), 0.5 * (1.0 - np.cos(np.pi * np.arange(ny + 1) / ny)), P.uniform_nodes(nz)
    per = (True, False, False)
    G = PO.Grid(xn, yn, zn, per, g)
    pr = Projection(xn, yn, zn, *per, ghost=g, device=0)
    rng = np.random.default_rng(41)
    F = lambda: G.sync(rng.standard_normal(G.padded))
    U, Uo, R = [F() for _ in range(3)], [F() for _ in range(3)], [F() for _ in range(3)]
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    tU, tUo, tR = [T(a) for a in U], [T(a) for a in Uo], [T(a) for a in R]
    force = {0: (1.0, 0.93), 2: (0.2, -0.05)}
    pr.mom_residual(0.01, 1.3, *tU, *tUo, *tR, force=force)
    ref = [PO.mom_residual(G, c, 0.01, 1.3, U[c], Uo[c], R[c], force.get(c)) for c in range(3)]
    for a, b in zip(tR, ref):
        assert np.array_equal(a.cpu().numpy(), b)
    pr.apply_residual(*tU, *tUo, *tR)
    for c in range(3):
        assert np.array_equal(tU[c].cpu().numpy(), PO.apply_residual(U[c], Uo[c], ref[c]))
    got = pr.bulk(*(T(a) for a in U), *tUo)
    for c in range(3):
        s_ref, v_ref = PO.bulk(G, c, U[c], Uo[c])
        assert abs(got[c][1] - v_ref) <= 1e-13 * abs(v_ref)
        assert abs(got[c][0] - s_ref) <= 1e-12 * np.abs(2.0 * U[c] - Uo[c]).max() * v_ref
    pr.close()



def test_oracle_channel_forcing_holds_the_bulk_velocity():
    """The bulk forcing of the channel loop: from a uniform start the wall
    friction slows the flow; the forced run keeps its bulk velocity nearer
    Ubulk than the same loop without the forcing."""
    from oracle.oracle import OracleBBMG, BBOX
    nx, ny, nz = 8, 10, 4
    ov = OracleBBMG(nx, ny, nz, True, False, True, method=BBOX, rcvg=1e-12, maxit=200)

    def solve_v(opr, rhs):
        ov.setup(P.STC7, np.ascontiguousarray(opr))
        return ov.solve(rhs)[0]
    runs = [PO.ChannelOracle(nx, ny, nz, oracle_solver_walls(nx, ny, nz), solve_v, Lz=0.5, visc=0.05, forcing=f)
            for f in (True, False)]
    for _ in range(4):
        for ch in runs:
            ch.step()
    G = runs[0].G
    bulk = [PO.bulk(G, 0, ch.U, ch.U) for ch in runs]
    mean = [s / v for s, v in bulk]
    assert mean[1] < mean[0] <= 1.0 + 1e-12
    assert 1.0 - mean[0] < 0.5 * (1.0 - mean[1])
