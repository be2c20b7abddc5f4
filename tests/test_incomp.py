"""The incompressible time loop on the GPU (nga2_b200/incomp.py): the kernels
of a sub-iteration (nga_proj_midpoint, nga_proj_advance, nga_proj_flow_stats)
against the numpy oracle, and whole time steps of the turbulence example
(examples/hit/src/simulation.f90) against the oracle's restatement of the
same loop.

CPU: the oracle loop keeps the velocity divergence-free and its linear
forcing holds the kinetic energy nearer its initial value than free decay;
the timetracker's dt rule.  GPU: midpoint and advance bit for bit; the
statistics' maxima bit for bit and sums to round-off; three time steps of
the loop to the pressure solver's tolerance.
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
