"""The two-stage preconditioner of mixed pcg_bbox (bbmg_set_precond_stage):
z = S(r) + V(r - A S(r)) with the caller's first stage S, FP32 V-cycle V and
flexible direction updates, plain FP64 pcg_bbox as the fallback on
stagnation.  The reference's cgsolve (src/solver/bbmg_class.f90:643-703) is
the method without S; every solve here is checked against the oracle's
pcg_bbox solution (1e-7 relative after mean removal, the mixed-precision
tolerance) and must reach rerr <= 1e-10."""
import numpy as np
import pytest

from nga2_b200 import problems as P
from nga2_b200.bbmg import BBMG, FP64, MIXED, PCG_BBOX, BBMGError
from oracle.oracle import OracleBBMG

pytestmark = pytest.mark.gpu

N = 32


@pytest.fixture(scope="module")
def drops():
    pb = P.drops_poisson(N, seed=8, ndrops=6, rmin=2.0, rmax=5.0)
    o = OracleBBMG(N, N, N, pb.xper, pb.yper, pb.zper, method=PCG_BBOX, rcvg=1e-12)
    o.setup(pb.stc, pb.opr)
    xo, _, _ = o.solve(pb.rhs)
    return pb, xo


def _err(x, xo):
    return np.abs(P.remove_mean(x) - P.remove_mean(xo)).max() / np.abs(P.remove_mean(xo)).max()


def _mixed(pb, **kw):
    g = BBMG(N, N, N, pb.xper, pb.yper, pb.zper, method=PCG_BBOX, precision=MIXED, rcvg=1e-10, maxit=60, **kw)
    g.setup(pb.stc, pb.opr)
    return g


def _bufs():
    import torch
    return (torch.zeros((N, N, N), dtype=torch.float64, device="cuda"),
            torch.zeros((N, N, N), dtype=torch.float64, device="cuda"))


def test_zero_stage_is_the_vcycle(drops):
    """S = 0: the preconditioner is the V-cycle alone, through the stage path
    (residual r - A*0 in FP64, then the V-cycle): same iterations as plain
    mixed pcg_bbox (+-1)."""
    pb, xo = drops
    g = _mixed(pb)
    _, it0, r0, st0 = g.solve(pb.rhs)
    r, z = _bufs()
    g.set_precond_stage(lambda r_, z_, s: z_.zero_(), r, z)
    x, it, rerr, st = g.solve(pb.rhs)
    assert st == 0 and rerr <= 1e-10 and abs(it - it0) <= 1, (it, it0)
    assert g.info["stage_it"] == it and g.info["fallback_it"] == 0
    assert _err(x, xo) < 1e-7


def test_exact_stage_converges_at_once(drops):
    """S = A^-1 (an inner FP64 solve to 1e-13): the first iteration already
    gives the solution to round-off."""
    import torch
    pb, xo = drops
    inner = BBMG(N, N, N, pb.xper, pb.yper, pb.zper, method=PCG_BBOX, precision=FP64, rcvg=1e-13, maxit=60)
    inner.setup(pb.stc, pb.opr)

    def exact(r_, z_, stream):
        torch.cuda.ExternalStream(stream).synchronize()  # r_ was written on the solver's stream
        z_.zero_()
        inner.solve(r_, z_)

    g = _mixed(pb)
    r, z = _bufs()
    g.set_precond_stage(exact, r, z)
    x, it, rerr, st = g.solve(pb.rhs)
    assert st == 0 and rerr <= 1e-10 and it <= 2, (it, rerr)
    assert _err(x, xo) < 1e-7


def test_stage_only_first_iterations(drops):
    """iters = 2: the stage runs in the first two iterations only."""
    import torch
    pb, xo = drops
    g = _mixed(pb)
    r, z = _bufs()
    g.set_precond_stage(lambda r_, z_, s: z_.copy_(0.5 * r_ / float(pb.opr[..., 0].max())), r, z, iters=2)
    x, it, rerr, st = g.solve(pb.rhs)
    assert st == 0 and rerr <= 1e-10 and g.info["stage_it"] == 2
    assert _err(x, xo) < 1e-7
    del torch


def test_garbage_stage_falls_back(drops):
    """A stage that returns large noise: the residual stalls, the solve
    switches to the plain FP64 pcg_bbox (fallback_it > 0) and still converges
    to the oracle's solution."""
    import torch
    pb, xo = drops
    gen = torch.Generator(device="cuda").manual_seed(0)
    scale = float(np.abs(xo).max()) * 1e3

    def noise(r_, z_, s):
        z_.copy_(scale * torch.randn(z_.shape, generator=gen, dtype=torch.float64, device="cuda"))

    g = _mixed(pb)
    r, z = _bufs()
    g.set_precond_stage(noise, r, z)
    x, it, rerr, st = g.solve(pb.rhs)
    inf = g.info
    assert st == 0 and rerr <= 1e-10 and inf["fallback_it"] > 0, (st, it, rerr, inf["fallback_it"])
    assert inf["stage_it"] == inf["fallback_it"]
    assert _err(x, xo) < 1e-7


def test_stage_error_and_arguments(drops):
    """An exception in the stage ends the solve with BAD_ARGS; a stage on an
    FP64 handle, or r and z of the wrong shape, are refused."""
    pb, _ = drops
    g = _mixed(pb)
    r, z = _bufs()

    def boom(r_, z_, s):
        raise RuntimeError("stage failed")

    g.set_precond_stage(boom, r, z)
    with pytest.raises(BBMGError) as e:
        g.solve(pb.rhs)
    assert e.value.code == 4 and "stage" in str(e.value)
    assert isinstance(g.stage_error, RuntimeError)
    g.set_precond_stage(None)
    _, it, rerr, st = g.solve(pb.rhs)
    assert st == 0 and g.info["stage_it"] == 0
    h = BBMG(N, N, N, pb.xper, pb.yper, pb.zper, method=PCG_BBOX, precision=FP64)
    with pytest.raises(BBMGError):
        h.set_precond_stage(lambda *a: None, r, z)
    with pytest.raises(ValueError):
        g.set_precond_stage(lambda *a: None, r[:-1], z)


def test_learned_stage_drop_sequence():
    """The learned stage end to end at 32^3: a drop sequence from the plain FP64
    solver, (residual, error) samples of its iterations, the U-Net trained by
    the project's kernels, then solves of the following steps with the network
    as the first stage: every solve reaches rerr <= 1e-10 with the oracle's
    solution, and the trained stage approximates A^-1 r better than the
    untrained one."""
    import torch
    from nga2_b200 import learned as NL
    from nga2_b200 import sequence as SQ
    from nga2_b200.problems import STC7
    n = 32
    seq = SQ.DropSequence(n, seed=3, ndrops=6, device="cuda")
    gen = SQ.bbmg_solver(n)
    recs = [seq.step(gen) for _ in range(10)]
    torch.cuda.synchronize()
    h64 = gen.handle
    samples = []
    for rec in recs[2:8]:
        h64.setup(STC7, rec["opr"].contiguous())
        samples += NL.stage_samples(h64, rec, iters=(0, 1, 2))
    h64.set_convergence(200, 1e-10)
    net = NL.UNet(nf=2, seed=1)
    stage = NL.LearnedStage(net, kappa=NL.fit_stage_kappa(samples), use_rho=True)
    test = NL.stage_samples(h64, recs[9], iters=(0,))[0]
    h64.setup(STC7, recs[9]["opr"].contiguous())

    def stage_err():
        z = torch.zeros_like(test["r"])
        stage.set_density(test["rho"])
        stage(test["r"], z, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return float((z - z.mean() - test["e"]).norm() / test["e"].norm())

    e_before = stage_err()
    losses = NL.train_stage(stage, samples, steps=150, lr=2e-3, lr_final=2e-4, seed=1)
    e_after = stage_err()
    assert np.mean(losses[-10:]) < np.mean(losses[:10])
    assert e_after < e_before, (e_before, e_after)
    for rec in recs[8:]:
        opr = rec["opr"].contiguous()
        g = BBMG(n, n, n, True, True, True, method=PCG_BBOX, precision=MIXED, rcvg=1e-10, maxit=60)
        g.setup(STC7, opr)
        r, z = _bufs_n(n)
        stage.set_density(rec["rho"])
        g.set_precond_stage(stage, r, z)
        x = torch.zeros_like(rec["rhs"])
        _, it, rerr, st = g.solve(rec["rhs"].contiguous(), x)
        assert st == 0 and rerr <= 1e-10 and g.info["stage_it"] > 0
        o = OracleBBMG(n, n, n, True, True, True, method=PCG_BBOX, rcvg=1e-12)
        o.setup(STC7, opr.cpu().numpy())
        xo, _, _ = o.solve(rec["rhs"].cpu().numpy())
        assert _err(x.cpu().numpy(), xo) < 1e-7
        g.close()


def _bufs_n(n):
    import torch
    return (torch.zeros((n, n, n), dtype=torch.float64, device="cuda"),
            torch.zeros((n, n, n), dtype=torch.float64, device="cuda"))
