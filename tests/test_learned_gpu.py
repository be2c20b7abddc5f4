"""Learned initial guess on the GPU: every nn_* kernel against the float64 CPU
oracle, the whole network's forward pass and gradients against the oracle's
autograd, training by the project's own kernels, and what the trained
network gains over the zero guess NGA2's callers use.

Tolerances: BF16 has an 8-bit significand, so a kernel whose output is stored
in BF16 is compared with a relative tolerance of 2^-8 on top of its FP32
accumulation error; FP32 outputs (weight gradients, head, loss) get 1e-4 of
the magnitude of their terms.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from nga2_b200 import learned as NL
from nga2_b200 import sequence as SQ
from nga2_b200 import bbmg as B
from oracle import unet_oracle as U

pytestmark = pytest.mark.gpu

BF16_REL = 2.0 ** -8


def bf(x):
    return torch.as_tensor(x, dtype=torch.float64).to(torch.bfloat16).to(torch.float64)


def to_cl(x):
    """(n, c, d, h, w) float64 -> channels-last (V, c) BF16 on the GPU."""
    n, c = x.shape[:2]
    return x.permute(0, 2, 3, 4, 1).reshape(-1, c).to(torch.bfloat16).cuda().contiguous()


def from_cl(t, shape, c=None, off=0):
    n, d, h, w = shape
    a = t.float().cpu().double()
    cc = c if c is not None else a.shape[1] - off
    return a[:, off:off + cc].reshape(n, d, h, w, cc).permute(0, 4, 1, 2, 3)


def act(t, shape, c=None, off=0):
    n, d, h, w = shape
    ld = t.shape[-1]
    a = NL.Act(t.data_ptr() + 2 * off, n, d, h, w, ld if c is None else c, ld)
    return a


def P(t):
    return C.c_void_p(t.data_ptr())


def close_bf16(gpu, ref, extra=0.0):
    err = (gpu - ref).abs()
    tol = BF16_REL * ref.abs() + 1e-3 * float(ref.abs().max()) + extra
    assert bool((err <= tol).all()), float((err - tol).max())


@pytest.fixture(scope="module")
def L():
    return NL.lib()


def packed(L, w):
    """FP32 master [27][cin][cout] -> (wt, wd) BF16 packings on the GPU."""
    cin, cout = w.shape[1], w.shape[2]
    wm = torch.as_tensor(w, dtype=torch.float32).cuda().contiguous()
    wt = torch.empty(27 * cin * cout, dtype=torch.bfloat16, device="cuda")
    wd = torch.empty_like(wt)
    assert L.nn_pack_weights(P(wm), cin, cout, P(wt), P(wd), None) == 0
    return wt, wd


@pytest.mark.parametrize("cin,cout,relu,shape", [(16, 16, 1, (1, 6, 10, 12)), (48, 32, 0, (2, 4, 4, 8)),
                                                 (192, 64, 1, (1, 4, 6, 4)), (64, 128, 1, (1, 4, 4, 4)),
                                                 (32, 16, 0, (1, 3, 5, 7))])
def test_conv_forward(L, cin, cout, relu, shape):
    rng = np.random.default_rng(cin + cout)
    n, d, h, w = shape
    x = bf(rng.standard_normal((n, cin, d, h, w)))
    wt_ = bf(rng.standard_normal((27, cin, cout)) / np.sqrt(27 * cin))
    b = torch.as_tensor(rng.standard_normal(cout) * 0.1, dtype=torch.float32)
    xg = to_cl(x)
    yg = torch.empty((n * d * h * w, cout), dtype=torch.bfloat16, device="cuda")
    wt, _ = packed(L, wt_.numpy())
    bg = b.cuda()
    assert L.nn_conv3(C.byref(act(xg, shape)), P(wt), P(bg), C.byref(act(yg, shape)), relu, None) == 0
    ref = U.conv3(x, wt_, b.double())
    if relu:
        ref = torch.relu(ref)
    close_bf16(from_cl(yg, shape), ref)


@pytest.mark.parametrize("cin,cout,shape", [(48, 16, (1, 4, 6, 8)), (96, 32, (1, 4, 4, 4)),
                                            (192, 64, (2, 4, 4, 4)), (16, 16, (1, 5, 3, 7))])
def test_conv_data_gradient(L, cin, cout, shape):
    rng = np.random.default_rng(7 * cin + cout)
    n, d, h, w = shape
    dy = bf(rng.standard_normal((n, cout, d, h, w)))
    wf = bf(rng.standard_normal((27, cin, cout)) / np.sqrt(27 * cout))
    _, wd = packed(L, wf.numpy())
    dyg = to_cl(dy)
    dxg = torch.empty((n * d * h * w, cin), dtype=torch.bfloat16, device="cuda")
    assert L.nn_conv3_dgrad(C.byref(act(dyg, shape)), P(wd), C.byref(act(dxg, shape)), None) == 0
    close_bf16(from_cl(dxg, shape), U.conv3_dgrad(dy, wf))


@pytest.mark.parametrize("cin,cout,shape", [(48, 16, (1, 8, 8, 8)), (192, 64, (1, 8, 8, 16)),
                                            (16, 16, (2, 5, 6, 7))])
def test_conv_weight_gradient(L, cin, cout, shape):
    rng = np.random.default_rng(11 * cin + cout)
    n, d, h, w = shape
    x = bf(rng.standard_normal((n, cin, d, h, w)))
    dy = bf(rng.standard_normal((n, cout, d, h, w)))
    dw = torch.zeros(27 * cin * cout, dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    xg, dyg = to_cl(x), to_cl(dy)
    assert L.nn_conv3_wgrad(C.byref(act(xg, shape)), C.byref(act(dyg, shape)), P(dw), P(db), None) == 0
    rw, rb = U.conv3_wgrad(x, dy)
    scale = float(np.sqrt(n * d * h * w))  # typical magnitude of a sum of V unit products
    np.testing.assert_allclose(dw.cpu().double().numpy().reshape(27, cin, cout), rw.numpy(), rtol=0, atol=1e-4 * scale)
    np.testing.assert_allclose(db.cpu().double().numpy(), rb.numpy(), rtol=0, atol=1e-4 * scale)


def test_elementwise_kernels(L):
    rng = np.random.default_rng(5)
    sh2, sh1 = (2, 4, 6, 8), (2, 2, 3, 4)
    c = 32
    x = bf(rng.standard_normal((2, c, 4, 6, 8)))
    xg = to_cl(x)
    # pool
    yg = torch.empty((2 * 2 * 3 * 4, c), dtype=torch.bfloat16, device="cuda")
    assert L.nn_pool2(C.byref(act(xg, sh2)), C.byref(act(yg, sh1)), None) == 0
    close_bf16(from_cl(yg, sh1), U.pool2(x))
    # pool backward, plain and accumulating
    dy = bf(rng.standard_normal((2, c, 2, 3, 4)))
    dyg = to_cl(dy)
    dxg = to_cl(x)
    assert L.nn_pool2_bwd(C.byref(act(dyg, sh1)), C.byref(act(dxg, sh2)), 1, None) == 0
    close_bf16(from_cl(dxg, sh2), x + U.up2(dy) / 8.0)
    assert L.nn_pool2_bwd(C.byref(act(dyg, sh1)), C.byref(act(dxg, sh2)), 0, None) == 0
    close_bf16(from_cl(dxg, sh2), U.up2(dy) / 8.0)
    # upsampling into a channel slice of a wider (concatenation) buffer, and back
    cat = torch.zeros((2 * 4 * 6 * 8, c + 16), dtype=torch.bfloat16, device="cuda")
    assert L.nn_up2(C.byref(act(dyg, sh1)), C.byref(act(cat, sh2, c, 0)), None) == 0
    close_bf16(from_cl(cat, sh2, c, 0), U.up2(dy))
    assert float(cat[:, c:].abs().max()) == 0.0
    ug = torch.empty_like(dyg)
    assert L.nn_up2_bwd(C.byref(act(xg, sh2)), C.byref(act(ug, sh1)), None) == 0
    close_bf16(from_cl(ug, sh1), U.pool2(x) * 8.0)
    # relu backward
    yv = bf(rng.standard_normal((2, c, 4, 6, 8)))
    g, yg2 = to_cl(x), to_cl(yv)
    assert L.nn_relu_bwd(C.byref(act(g, sh2)), C.byref(act(yg2, sh2)), None) == 0
    close_bf16(from_cl(g, sh2), x * (yv > 0))
    # embedding of three FP64 fields
    f = [torch.from_numpy(rng.standard_normal(2 * 4 * 6 * 8)).cuda() for _ in range(3)]
    sc = [0.5, 2.0, -1.0]
    eg = torch.empty((2 * 4 * 6 * 8, 16), dtype=torch.bfloat16, device="cuda")
    fp = (C.c_void_p * 3)(*[t.data_ptr() for t in f])
    ss = (C.c_double * 3)(*sc)
    assert L.nn_embed(3, fp, ss, 1, C.byref(act(eg, sh2)), None) == 0
    close_bf16(from_cl(eg, sh2), U.embed([t.cpu().numpy() for t in f], sc, sh2))
    # ... and from fields on the grid twice as fine (2x2x2 means)
    ec = torch.empty((2 * 2 * 3 * 4, 16), dtype=torch.bfloat16, device="cuda")
    assert L.nn_embed(3, fp, ss, 2, C.byref(act(ec, sh1)), None) == 0
    close_bf16(from_cl(ec, sh1), U.pool2(U.embed([t.cpu().numpy() for t in f], sc, sh2)))


def test_head_loss_adam_apply(L):
    rng = np.random.default_rng(9)
    sh = (1, 4, 4, 8)
    V = 128
    x = bf(rng.standard_normal((1, 16, 4, 4, 8)))
    xg = to_cl(x)
    w = torch.as_tensor(rng.standard_normal(16), dtype=torch.float32)
    b = torch.tensor([0.25], dtype=torch.float32)
    out = torch.empty(V, dtype=torch.float32, device="cuda")
    wg, bg = w.cuda(), b.cuda()  # kept alive: kernels run after the call returns
    assert L.nn_head(C.byref(act(xg, sh)), P(wg), P(bg), P(out), None) == 0
    ref = torch.einsum("ncdhw,c->ndhw", x, w.double()).reshape(-1) + 0.25
    np.testing.assert_allclose(out.cpu().double().numpy(), ref.numpy(), rtol=1e-5, atol=1e-5)
    # loss and its gradient
    tgt = torch.from_numpy(rng.standard_normal(V)).cuda()
    grad = torch.empty(V, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.nn_mse(P(out), P(tgt), 0.5, V, P(grad), P(loss), None) == 0
    d = out.double() - 0.5 * tgt
    np.testing.assert_allclose(float(loss), float((d * d).sum()), rtol=1e-6)
    np.testing.assert_allclose(grad.cpu().numpy(), (2 * d / V).float().cpu().numpy(), rtol=1e-6, atol=1e-9)
    # head backward
    dx = torch.empty_like(xg)
    dw = torch.zeros(16, dtype=torch.float32, device="cuda")
    db = torch.zeros(1, dtype=torch.float32, device="cuda")
    assert L.nn_head_bwd(C.byref(act(xg, sh)), P(wg), P(grad), C.byref(act(dx, sh)), P(dw), P(db), None) == 0
    g64 = grad.cpu().double().reshape(1, 4, 4, 8)
    close_bf16(from_cl(dx, sh), g64[:, None] * w.double()[None, :, None, None, None])
    np.testing.assert_allclose(dw.cpu().double().numpy(), torch.einsum("ncdhw,ndhw->c", x, g64).numpy(),
                               rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(float(db), float(g64.sum()), rtol=1e-4, atol=1e-7)
    # Adam, two steps against the textbook update
    p0 = rng.standard_normal(1000).astype(np.float32)
    gs = [rng.standard_normal(1000).astype(np.float32) for _ in range(2)]
    pg, mg, vg = torch.from_numpy(p0).cuda(), torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    pr, mr, vr = p0.astype(np.float64), np.zeros(1000), np.zeros(1000)
    for t, gg in enumerate(gs, 1):
        ggd = torch.from_numpy(gg).cuda()
        assert L.nn_adam(P(pg), P(ggd), P(mg), P(vg), 1000, 1e-2, 0.9, 0.999, 1e-8, t,
                         None) == 0
        mr = 0.9 * mr + 0.1 * gg
        vr = 0.999 * vr + 0.001 * gg.astype(np.float64) ** 2
        pr = pr - 1e-2 * (mr / (1 - 0.9 ** t)) / (np.sqrt(vr / (1 - 0.999 ** t)) + 1e-8)
    np.testing.assert_allclose(pg.cpu().double().numpy(), pr, rtol=1e-5, atol=1e-6)
    # apply: same grid and 2x trilinear
    pred = torch.from_numpy(rng.standard_normal(2 * 4 * 4 * 8).astype(np.float32)).cuda()
    base = torch.from_numpy(rng.standard_normal(2 * 8 * 8 * 16)).cuda()
    o1 = torch.empty(2 * 4 * 4 * 8, dtype=torch.float64, device="cuda")
    assert L.nn_apply(None, P(pred), 3.0, 2, 4, 4, 8, 1, P(o1), None) == 0
    np.testing.assert_allclose(o1.cpu().numpy(), 3.0 * pred.cpu().double().numpy(), rtol=1e-15)
    o2 = torch.empty(2 * 8 * 8 * 16, dtype=torch.float64, device="cuda")
    assert L.nn_apply(P(base), P(pred), -2.0, 2, 4, 4, 8, 2, P(o2), None) == 0
    ref = base.cpu() - 2.0 * U.apply_up2(pred.cpu().double().numpy(), 4, 4, 8).reshape(-1)
    np.testing.assert_allclose(o2.cpu().numpy(), ref.numpy(), rtol=1e-6, atol=1e-6)


def test_bad_arguments_are_rejected(L):
    t = torch.zeros((64, 24), dtype=torch.bfloat16, device="cuda")
    bad_c = act(t, (1, 4, 4, 4), 24)   # 24 channels: not a multiple of 16
    wt = torch.zeros(27 * 24 * 16, dtype=torch.bfloat16, device="cuda")
    assert L.nn_conv3(C.byref(bad_c), P(wt), None, C.byref(act(t, (1, 4, 4, 4), 16)), 0, None) == 4
    odd = NL.Act(t.data_ptr(), 1, 4, 4, 4, 16, 17)     # odd leading dimension
    assert L.nn_pool2(C.byref(odd), C.byref(act(t, (1, 2, 2, 2), 16)), None) == 4
    assert L.nn_apply(None, P(t), 1.0, 1, 2, 2, 2, 3, P(t), None) == 4


# ---------------------------------------------------------------- network
def _sample(nf, shape, seed):
    rng = np.random.default_rng(seed)
    V = int(np.prod(shape))
    fields = [torch.from_numpy(rng.standard_normal(V)).cuda() for _ in range(nf)]
    scales = [1.0, 0.5, 0.8][:nf]
    target = torch.from_numpy(rng.standard_normal(V)).cuda()
    return fields, scales, target


def test_network_forward_and_gradients_match_oracle():
    """GPU forward vs the oracle with BF16 storage emulated; GPU gradients vs
    the oracle's float64 autograd through the same emulated rounding, layer by
    layer (BF16 activations and gradients limit the agreement to ~1e-2)."""
    shape = (1, 16, 16, 16)
    net = NL.UNet(nf=3, seed=3)
    fields, scales, target = _sample(3, shape, 4)
    b = net.buffers(shape, True)
    net.embed(b, fields, scales)
    out = net.forward(b).cpu().double()
    p = net.params.cpu().double()
    x = U.embed([f.cpu().numpy() for f in fields], scales, shape)
    ref = U.forward(p, x, round_bf16=True).reshape(-1)
    rel = float((out - ref).norm() / ref.norm())
    assert rel < 3e-2, rel
    net.loss_grad(b, target, 0.7)
    net.grads.zero_()
    net.backward(b)
    g = net.grads.cpu().double().numpy()
    q = p.clone().requires_grad_(True)
    U.loss(q, x, target.cpu().numpy(), 0.7, round_bf16=True).backward()
    gr = q.grad.numpy()
    bounds = [o for pair in net.offsets for o in pair] + [net.head_off, net.nparam]
    segs = []
    for i, (lo, hi) in enumerate(net.offsets):
        segs.append((net.spec[i][0] + ".w", lo, hi))
        segs.append((net.spec[i][0] + ".b", hi, hi + net.spec[i][2]))
    segs.append(("head", net.head_off, net.nparam))
    for name, lo, hi in segs:
        a, r = g[lo:hi], gr[lo:hi]
        if name == "enc1a.w":  # only the nf real input channels carry signal
            a = a.reshape(27, 16, 16)[:, :3].ravel()
            r = r.reshape(27, 16, 16)[:, :3].ravel()
        cos = float(a @ r / (np.linalg.norm(a) * np.linalg.norm(r) + 1e-30))
        relerr = float(np.linalg.norm(a - r) / (np.linalg.norm(r) + 1e-30))
        assert cos > 0.99 and relerr < 0.1, (name, cos, relerr)


def test_training_reduces_the_loss():
    """The project's own forward/backward/Adam kernels fit a smooth target."""
    shape = (1, 16, 16, 16)
    net = NL.UNet(nf=2, seed=1)
    rng = np.random.default_rng(2)
    z, y, x = np.meshgrid(*[np.arange(16) / 16.0] * 3, indexing="ij")
    f0 = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.1 * rng.standard_normal(x.shape)
    f1 = np.cos(2 * np.pi * z)
    tgt = 0.5 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.3 * np.cos(2 * np.pi * z)
    fields = [torch.from_numpy(f0.ravel()).cuda(), torch.from_numpy(f1.ravel()).cuda()]
    target = torch.from_numpy(tgt.ravel()).cuda()
    losses = []
    for t in range(300):
        losses.append(float(net.train_step(fields, [1.0, 1.0], target.reshape(16, 16, 16), 1.0, lr=2e-3)))
    assert np.isfinite(losses).all()
    assert min(losses[-20:]) < 0.05 * losses[0], (losses[0], losses[-20:])


def test_learned_guess_saves_iterations():
    """Train on the first steps of a drop sequence the plain GPU multigrid
    generates, then solve the following steps from the network's guess and
    from zero (NGA2's choice) to the same max|b - A x| <= 1e-10 max|b|; the
    plain warm start (the previous solve's solution) is measured beside it.
    The network predicts the change from the warm start, so its guess must be
    at least about as close to the solution as the warm start (within 5 %),
    and it must not need more iterations than the warm start."""
    torch.manual_seed(0)
    n = 32
    seq = SQ.DropSequence(n, seed=11, ndrops=10, rmin=3.0 / n, rmax=6.0 / n, device="cuda")
    solve = SQ.bbmg_solver(n)
    recs = [seq.step(solve) for _ in range(56)]
    assert all(st == 0 for _, _, st in solve.stats)
    train_recs, test_recs = recs[8:48], recs[48:]
    net = NL.UNet(nf=3, seed=0)
    guess = NL.LearnedGuess(net, kappa=NL.fit_kappa(train_recs), use_rho=True)
    losses = NL.train(guess, train_recs, steps=600, lr=2e-3, lr_final=1e-4)
    assert np.mean(losses[-50:]) < 0.5 * np.mean(losses[:20])
    h = solve.handle
    h.set_residual_norm(B.NORM_RHS)
    its0, its1, itsw, errw, errl = [], [], [], [], []
    for rec in test_recs:
        h.setup(SQ_STC(), rec["opr"].contiguous())
        b = rec["rhs"].contiguous()
        x0 = torch.zeros_like(b)
        _, it0, _, st0 = h.solve(b, x0)
        xw = rec["p_prev"].clone()
        _, itw, _, stw = h.solve(b, xw)
        x1 = torch.empty_like(b)
        guess.guess(rec, x1)
        torch.cuda.synchronize()
        dp = rec["dp"] - rec["dp"].mean()
        errw.append(float((rec["p_prev"] - rec["p_prev"].mean() - dp).norm() / dp.norm()))
        errl.append(float((x1 - x1.mean() - dp).norm() / dp.norm()))
        _, it1, rerr1, st1 = h.solve(b, x1)
        assert st0 == 0 and st1 == 0 and stw == 0
        # all stop at the same absolute residual: check it in FP64 here
        for x in (x0, x1, xw):
            r = b - apply7(rec["opr"], x)
            # the PCG stops on its recurrence residual; the true one may drift a little
            assert float(r.abs().max()) <= 1.5e-10 * float(b.abs().max())
        its0.append(it0)
        its1.append(it1)
        itsw.append(itw)
    print("iterations zero / warm / learned:", its0, itsw, its1, "errors warm / learned:", errw, errl)
    assert np.mean(its1) < np.mean(its0), (its0, its1)
    assert np.mean(its1) <= np.mean(itsw), (itsw, its1)
    assert np.mean(errl) <= 1.05 * np.mean(errw), (errw, errl)


def SQ_STC():
    from nga2_b200.problems import STC7
    return STC7


def apply7(opr, x):
    """A x for the periodic 7-point operator (k, j, i, 7) in NGA2's stencil order."""
    r = opr[..., 0] * x
    r = r + opr[..., 1] * torch.roll(x, -1, 2) + opr[..., 2] * torch.roll(x, 1, 2)
    r = r + opr[..., 3] * torch.roll(x, -1, 1) + opr[..., 4] * torch.roll(x, 1, 1)
    r = r + opr[..., 5] * torch.roll(x, -1, 0) + opr[..., 6] * torch.roll(x, 1, 0)
    return r


def test_learned_guess_on_turbulence_sequence():
    """Single-phase configuration: a decaying-turbulence sequence from the
    constant-density stepper (pressure increments solved by the plain GPU
    multigrid); the network (inputs: rhs and previous increment) trained on the
    first solves must not cost iterations against the zero guess on the next
    ones, and every solve reaches max|b - A x| <= 1e-10 max|b|."""
    torch.manual_seed(0)
    n = 32
    solve = SQ.bbmg_solver(n)
    seq = SQ.TurbulenceSequence(n, seed=3, device="cuda", solve=solve)
    recs = [seq.step() for _ in range(40)]
    assert all(st == 0 for _, _, st in solve.stats)
    train_recs, test_recs = recs[4:32], recs[32:]
    net = NL.UNet(nf=2, seed=1)
    guess = NL.LearnedGuess(net, kappa=NL.fit_kappa(train_recs), use_rho=False)
    NL.train(guess, train_recs, steps=300, lr=2e-3, lr_final=1e-4)
    h = solve.handle
    h.set_residual_norm(B.NORM_RHS)
    h.setup(SQ_STC(), recs[0]["opr"].contiguous())  # constant operator
    its0, its1 = [], []
    for rec in test_recs:
        b = rec["rhs"].contiguous()
        x0 = torch.zeros_like(b)
        _, it0, _, st0 = h.solve(b, x0)
        x1 = torch.empty_like(b)
        guess.guess(rec, x1)
        torch.cuda.synchronize()
        _, it1, _, st1 = h.solve(b, x1)
        assert st0 == 0 and st1 == 0
        r = b - apply7(rec["opr"], x1)
        assert float(r.abs().max()) <= 1.5e-10 * float(b.abs().max())
        its0.append(it0)
        its1.append(it1)
    print("turbulence iterations zero / learned:", its0, its1)
    assert np.mean(its1) <= np.mean(its0), (its0, its1)


@pytest.mark.parametrize("cin,cout,relu,dgrad,shape", [
    (16, 16, 1, False, (1, 3, 2, 128)), (48, 16, 0, False, (1, 3, 2, 128)), (16, 32, 1, False, (1, 3, 2, 128)),
    (16, 64, 0, False, (1, 3, 2, 128)), (16, 48, 0, True, (1, 3, 2, 128)),
    # tiles spanning several rows (w = 32, 16), half a row (w = 256), the U-Net's widest layers
    (96, 32, 1, False, (1, 4, 4, 32)), (192, 64, 0, False, (2, 2, 4, 16)), (64, 128, 1, False, (1, 2, 2, 256)),
    (128, 128, 0, False, (1, 4, 4, 8)), (32, 96, 0, True, (1, 4, 4, 32)), (64, 192, 0, True, (1, 4, 8, 8))])
def test_tcgen05_convolution(L, cin, cout, relu, dgrad, shape):
    """Grids of whole 128-voxel tiles take the tcgen05 path (TMEM accumulator,
    staged K ring): forward and data-gradient convolutions against the oracle,
    and no completion timeout."""
    rng = np.random.default_rng(100 + cin + cout)
    n, d, h, w = shape
    if dgrad:   # dy has cin channels, dx the forward's input channels (cout here)
        dy = bf(rng.standard_normal((n, cin, d, h, w)))
        wf = bf(rng.standard_normal((27, cout, cin)) / np.sqrt(27 * cin))
        _, wd = packed(L, wf.numpy())
        dyg = to_cl(dy)
        dxg = torch.empty((n * d * h * w, cout), dtype=torch.bfloat16, device="cuda")
        assert L.nn_conv3_dgrad(C.byref(act(dyg, shape)), P(wd), C.byref(act(dxg, shape)), None) == 0
        assert L.nn_tc_error() == 0
        close_bf16(from_cl(dxg, shape), U.conv3_dgrad(dy, wf))
        return
    x = bf(rng.standard_normal((n, cin, d, h, w)))
    wt_ = bf(rng.standard_normal((27, cin, cout)) / np.sqrt(27 * cin))
    b = torch.as_tensor(rng.standard_normal(cout) * 0.1, dtype=torch.float32)
    xg = to_cl(x)
    yg = torch.empty((n * d * h * w, cout), dtype=torch.bfloat16, device="cuda")
    wt, _ = packed(L, wt_.numpy())
    bg = b.cuda()
    assert L.nn_conv3(C.byref(act(xg, shape)), P(wt), P(bg), C.byref(act(yg, shape)), relu, None) == 0
    assert L.nn_tc_error() == 0
    ref = U.conv3(x, wt_, b.double())
    if relu:
        ref = torch.relu(ref)
    close_bf16(from_cl(yg, shape), ref)


def test_network_with_tcgen05_rows_matches_oracle():
    """A 128-voxel-wide grid (level-1 convolutions on tcgen05): the forward pass
    against the oracle with BF16 storage emulated."""
    shape = (1, 8, 8, 128)
    net = NL.UNet(nf=2, seed=5)
    fields, scales, _ = _sample(2, shape, 6)
    b = net.buffers(shape, False)
    net.embed(b, fields, scales)
    out = net.forward(b).cpu().double()
    assert NL.lib().nn_tc_error() == 0
    x = U.embed([f.cpu().numpy() for f in fields], scales, shape)
    ref = U.forward(net.params.cpu().double(), x, round_bf16=True).reshape(-1)
    rel = float((out - ref).norm() / ref.norm())
    assert rel < 3e-2, rel
