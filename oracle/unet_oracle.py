"""CPU oracle of the learned initial guess's U-Net (test infrastructure only).

The network has no counterpart in the reference (NGA2 starts each pressure
solve from zero), so this is the specification the CUDA kernels of
``nga2_b200/csrc/unet.cu`` are checked against: a float64 PyTorch-CPU
restatement of every operation, with gradients from autograd (themselves
checked by finite differences in the tests).  Nothing in the product imports
this file.

Conventions (shared with the CUDA kernels by specification, not by import):

* activations are (n, c, d, h, w), w fastest in memory on the GPU side, every
  direction periodic;
* a 3x3x3 convolution is y(v) = b + sum_tap sum_ci x(v + off(tap), ci) w[tap][ci][co]
  with tap = 9 (dz+1) + 3 (dy+1) + (dx+1), i.e. a cross-correlation with circular
  padding;
* pooling is the 2x2x2 mean, upsampling nearest-neighbour; the decoder input is
  the upsampled tensor's channels followed by the encoder (skip) channels;
* the 14 convolutions are ordered enc1a, enc1b, enc2a, enc2b, enc3a, enc3b,
  bota, botb, dec3a, dec3b, dec2a, dec2b, dec1a, dec1b; each has w[27][cin][cout]
  then b[cout] in the flat parameter vector, followed by the 1x1 head's w[c1], b;
* the input embedding puts scales[i]*fields[i] in channel i and zeros in the
  remaining channels up to 16;
* the loss is sum((out - scale*target)^2) / nvox.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

CH = (16, 32, 64, 128)
CIN0 = 16


def layers(ch=CH):
    c1, c2, c3, c4 = ch
    return [("enc1a", CIN0, c1), ("enc1b", c1, c1), ("enc2a", c1, c2), ("enc2b", c2, c2),
            ("enc3a", c2, c3), ("enc3b", c3, c3), ("bota", c3, c4), ("botb", c4, c4),
            ("dec3a", c4 + c3, c3), ("dec3b", c3, c3), ("dec2a", c3 + c2, c2), ("dec2b", c2, c2),
            ("dec1a", c2 + c1, c1), ("dec1b", c1, c1)]


def nparams(ch=CH):
    return sum(27 * ci * co + co for _, ci, co in layers(ch)) + ch[0] + 1


def unflatten(p, ch=CH):
    """Flat parameter tensor -> list of (w[27][cin][cout], b[cout]) and the head."""
    out, o = [], 0
    for _, ci, co in layers(ch):
        w = p[o:o + 27 * ci * co].reshape(27, ci, co); o += 27 * ci * co
        b = p[o:o + co]; o += co
        out.append((w, b))
    hw = p[o:o + ch[0]]; hb = p[o + ch[0]:o + ch[0] + 1]
    return out, (hw, hb)


def bf16(x):
    """Round to the nearest BF16 value (ties to even), kept in float64."""
    return x.to(torch.bfloat16).to(x.dtype)


def conv3(x, w, b=None):
    """Periodic 3x3x3 cross-correlation; x (n, cin, d, h, w), w [27][cin][cout]."""
    cin, cout = w.shape[1], w.shape[2]
    wt = w.reshape(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2)  # (cout, cin, kz, ky, kx)
    xp = F.pad(x, (1, 1, 1, 1, 1, 1), mode="circular")
    return F.conv3d(xp, wt, b)


def conv3_dgrad(dy, w):
    """Input gradient of conv3: the transposed (mirrored) correlation."""
    wm = torch.flip(w, dims=[0]).transpose(1, 2)  # [26 - tap][cout][cin]
    return conv3(dy, wm)


def conv3_wgrad(x, dy):
    """dw[tap][ci][co] = sum_v x(v + off(tap), ci) dy(v, co); db = sum_v dy."""
    dw = torch.empty(27, x.shape[1], dy.shape[1], dtype=x.dtype)
    for tap in range(27):
        dz, dyy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
        xs = torch.roll(x, shifts=(-dz, -dyy, -dx), dims=(2, 3, 4))
        dw[tap] = torch.einsum("ncdhw,nkdhw->ck", xs, dy)
    return dw, dy.sum(dim=(0, 2, 3, 4))


def pool2(x):
    return F.avg_pool3d(x, 2)


def up2(x):
    return x.repeat_interleave(2, dim=2).repeat_interleave(2, dim=3).repeat_interleave(2, dim=4)


def embed(fields, scales, shape):
    n, d, h, w = shape
    x = torch.zeros(n, CIN0, d, h, w, dtype=torch.float64)
    for i, (f, s) in enumerate(zip(fields, scales)):
        x[:, i] = s * torch.as_tensor(np.asarray(f, np.float64)).reshape(n, d, h, w)
    return x


def forward(p, x, ch=CH, round_bf16=False):
    """U-Net output (n, d, h, w) for the embedded input x.  round_bf16 rounds
    the weights and every stored activation to BF16 as the GPU stores them."""
    r = bf16 if round_bf16 else (lambda t: t)
    convs, (hw, hb) = unflatten(p, ch)

    def c(i, t):
        w, b = convs[i]
        return r(torch.relu(conv3(t, r(w), b)))

    x = r(x)
    e1 = c(1, c(0, x))
    e2 = c(3, c(2, r(pool2(e1))))
    e3 = c(5, c(4, r(pool2(e2))))
    u4 = c(7, c(6, r(pool2(e3))))
    u3 = c(9, c(8, torch.cat([up2(u4), e3], dim=1)))
    u2 = c(11, c(10, torch.cat([up2(u3), e2], dim=1)))
    u1 = c(13, c(12, torch.cat([up2(u2), e1], dim=1)))
    return torch.einsum("ncdhw,c->ndhw", u1, hw) + hb[0]


def loss(p, x, target, scale, ch=CH, round_bf16=False):
    out = forward(p, x, ch, round_bf16)
    t = torch.as_tensor(np.asarray(target, np.float64)).reshape(out.shape)
    return ((out - scale * t) ** 2).sum() / out.numel()


def grad(p, x, target, scale, ch=CH):
    """(loss, dloss/dparams) by autograd in float64."""
    q = torch.as_tensor(p, dtype=torch.float64).clone().requires_grad_(True)
    L = loss(q, x, target, scale, ch)
    L.backward()
    return float(L.detach()), q.grad.detach().numpy()


def apply_up2(pred, d, h, w):
    """Trilinear cell-centred 2x interpolation (weights 3/4, 1/4, periodic)."""
    p = torch.as_tensor(np.asarray(pred, np.float64)).reshape(-1, d, h, w)

    def along(t, dim):
        n = t.shape[dim]
        lo = torch.roll(t, 1, dims=dim)    # t[i-1]
        hi = torch.roll(t, -1, dims=dim)   # t[i+1]
        even = 0.75 * t + 0.25 * lo
        odd = 0.75 * t + 0.25 * hi
        out = torch.stack([even, odd], dim=dim + 1)
        shape = list(t.shape)
        shape[dim] = 2 * n
        return out.reshape(shape)

    return along(along(along(p, 1), 2), 3)
