"""Learned initial guess, host side: the U-Net oracle (checked against direct
sums and finite differences), the parameter layout shared with the CUDA
kernels, the C ABI's nn_* exports, and the solve-sequence generator."""
import os
import re

import numpy as np
import pytest
import torch

from nga2_b200 import learned as NL
from nga2_b200 import sequence as SQ
from nga2_b200 import bbmg as B
from oracle import unet_oracle as U

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(name):
    txt = open(os.path.join(ROOT, "include", name)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(nn_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_learned_symbol():
    lib = B.load()
    names = header_functions("bbmg_learned.h")
    assert len(names) == 16
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(NL.NN_EXPORTS) == names
    NL.lib()  # every signature binds


def test_layer_layout_matches_oracle():
    assert NL.layer_spec() == U.layers()
    for nf in (2, 3):
        p = NL.init_params(nf)
        assert p.size == U.nparams()
        convs, (hw, hb) = U.unflatten(torch.from_numpy(p.astype(np.float64)))
        w0 = convs[0][0]
        assert float(w0[:, nf:, :].abs().max()) == 0.0   # padded input channels carry no weight
        assert hb.shape == (1,) and hw.shape == (16,)


def _direct_conv(x, w, b):
    n, cin, d, h, wd = x.shape
    y = np.zeros((n, w.shape[2], d, h, wd))
    for tap in range(27):
        dz, dy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
        xs = np.roll(x, shift=(-dz, -dy, -dx), axis=(2, 3, 4))
        y += np.einsum("ncdhw,ck->nkdhw", xs, w[tap])
    return y + b[None, :, None, None, None]


def test_oracle_conv_is_a_periodic_correlation():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 3, 4, 5, 6))
    w = rng.standard_normal((27, 3, 4))
    b = rng.standard_normal(4)
    y = U.conv3(torch.from_numpy(x), torch.from_numpy(w), torch.from_numpy(b)).numpy()
    np.testing.assert_allclose(y, _direct_conv(x, w, b), rtol=1e-12, atol=1e-12)


def test_oracle_conv_gradients_match_autograd():
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.standard_normal((1, 3, 4, 5, 6))).requires_grad_(True)
    w = torch.from_numpy(rng.standard_normal((27, 3, 5))).requires_grad_(True)
    b = torch.from_numpy(rng.standard_normal(5)).requires_grad_(True)
    dy = torch.from_numpy(rng.standard_normal((1, 5, 4, 5, 6)))
    (U.conv3(x, w, b) * dy).sum().backward()
    np.testing.assert_allclose(U.conv3_dgrad(dy, w.detach()).numpy(), x.grad.numpy(), rtol=1e-11, atol=1e-11)
    dw, db = U.conv3_wgrad(x.detach(), dy)
    np.testing.assert_allclose(dw.numpy(), w.grad.numpy(), rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(db.numpy(), b.grad.numpy(), rtol=1e-11, atol=1e-11)


def test_oracle_unet_gradient_by_finite_differences():
    """Autograd of the full float64 U-Net against central differences on a
    sample of parameters from every layer (small channels, 8^3)."""
    ch = (4, 4, 8, 8)
    rng = np.random.default_rng(2)
    p = rng.standard_normal(U.nparams(ch)) * 0.3
    x = U.embed([rng.standard_normal(512), rng.standard_normal(512)], [1.0, 0.5], (1, 8, 8, 8))
    tgt = rng.standard_normal(512)
    L0, g = U.grad(p, x, tgt, 0.7, ch)
    assert np.isfinite(L0)
    bounds = np.cumsum([0] + [27 * ci * co + co for _, ci, co in U.layers(ch)] + [ch[0] + 1])
    picks = []
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        cand = np.arange(lo, hi)
        cand = cand[np.abs(g[cand]) > 1e-6] if (np.abs(g[cand]) > 1e-6).any() else cand
        picks += list(rng.choice(cand, size=min(2, cand.size), replace=False))
    h = 1e-6
    for i in picks:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (float(U.loss(torch.from_numpy(pp), x, tgt, 0.7, ch)) - float(U.loss(torch.from_numpy(pm), x, tgt, 0.7, ch))) / (2 * h)
        assert abs(fd - g[i]) <= 2e-5 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_oracle_trilinear_prolongation_preserves_constants_and_linear_modes():
    p = np.full((1, 4, 4, 4), 2.5)
    np.testing.assert_allclose(U.apply_up2(p, 4, 4, 4).numpy(), 2.5)
    # a cosine mode is interpolated to second order
    n = 16
    x = (np.arange(n) + 0.5) / n
    xf = (np.arange(2 * n) + 0.5) / (2 * n)
    c = np.cos(2 * np.pi * x)[None, None, None, :] * np.ones((1, n, n, n))
    f = U.apply_up2(c, n, n, n).numpy()
    exact = np.cos(2 * np.pi * xf)[None, None, None, :]
    assert np.abs(f - exact).max() < 0.03


def test_drop_sequence_projection_is_divergence_free():
    """The corrector makes div(u) vanish given the exact pressure increment:
    solve the step's system with a dense direct solver at 8^3."""
    seq = SQ.DropSequence(8, seed=3, ndrops=3, rmin=0.15, rmax=0.3, ratio=50.0)

    def dense_solve(opr, rhs):
        n = rhs.shape[0]
        N = n ** 3
        A = np.zeros((N, N))
        o = opr.numpy()
        st = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
        for k in range(n):
            for j in range(n):
                for i in range(n):
                    r = (k * n + j) * n + i
                    for s, (a, b, c) in enumerate(st):
                        A[r, (((k + c) % n) * n + (j + b) % n) * n + (i + a) % n] += o[k, j, i, s]
        A[0, :] = 0.0
        A[0, 0] = 1.0
        bb = rhs.numpy().ravel().copy()
        bb[0] = 0.0
        return torch.from_numpy(np.linalg.solve(A, bb).reshape(rhs.shape))

    for _ in range(3):
        rec = seq.step(dense_solve)
        d = seq.div(seq.u)
        assert float(d.abs().max()) < 1e-8 * max(1.0, float(rec["rhs"].abs().max()) / seq.vol)
        assert float(rec["rho"].max()) <= 50.0 and float(rec["rho"].min()) >= 1.0
    # operator: symmetric, zero row sums (periodic), NGA2 stencil order
    o = rec["opr"]
    assert float((o.sum(-1)).abs().max()) < 1e-12 * float(o[..., 0].abs().max())
    np.testing.assert_allclose(o[..., 1].numpy(), torch.roll(o[..., 2], -1, dims=2).numpy(), rtol=1e-14)
    np.testing.assert_allclose(o[..., 3].numpy(), torch.roll(o[..., 4], -1, dims=1).numpy(), rtol=1e-14)
    np.testing.assert_allclose(o[..., 5].numpy(), torch.roll(o[..., 6], -1, dims=0).numpy(), rtol=1e-14)


def _fft_solve(opr, rhs):
    """Exact solve of the constant-coefficient periodic 7-point system (FFT)."""
    n = rhs.shape[0]
    c = float(opr[0, 0, 0, 1])
    k = torch.arange(n, dtype=torch.float64)
    lam = 2 - 2 * torch.cos(2 * np.pi * k / n)
    L = (-c) * (lam[:, None, None] + lam[None, :, None] + lam[None, None, :])
    L[0, 0, 0] = 1.0
    x = torch.fft.ifftn(torch.fft.fftn(rhs) / L).real
    return x - x.mean()


def test_turbulence_sequence_projection_and_decay():
    """The constant-density stepper: the initial field and every corrected
    field are discretely divergence free, u_rms starts at 1 and decays, the
    time step honours CFL 0.5, and nu gives Re_lambda = 50."""
    seq = SQ.TurbulenceSequence(16, seed=2, solve=_fft_solve)
    assert float(seq.div(seq.u).abs().max()) < 1e-12
    urms0 = (float(sum((x ** 2).mean() for x in seq.u)) / 3) ** 0.5
    assert abs(urms0 - 1.0) < 1e-12
    lam = (15.0 / (2.0 * seq._strain2())) ** 0.5
    assert abs(1.0 * lam / seq.nu - 50.0) < 1e-9
    for _ in range(4):
        umax = max(float(x.abs().max()) for x in seq.u)
        rec = seq.step()
        assert rec["dt"] <= 0.5 * seq.dx / umax + 1e-15
        assert float(seq.div(seq.u).abs().max()) < 1e-12
        assert rec["opr"].shape == (16, 16, 16, 7)
    urms = (float(sum((x ** 2).mean() for x in seq.u)) / 3) ** 0.5
    assert urms < urms0
