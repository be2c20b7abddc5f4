"""Learned initial guess for the pressure solve: a small 3-D U-Net on the GPU.

NGA2 has no counterpart: its flow solvers start every pressure solve from
zero for the pressure increment (``src/two_phase/tpns_class.f90`` and
``src/constant_density/incomp_class.f90`` callers set ``psolv%sol=0`` before
``psolv%solve()``).  Here a U-Net predicts that increment from the solve's
right-hand side, the previous pressure and (for two-phase flow) the density;
the prediction is handed to ``bbmg_solve`` as the initial guess and the
multigrid, with ``rerr`` measured against max|rhs| (``NORM_RHS``), still
decides convergence, so a learned solve stops at the same max|b - A x| as the
zero-guess solve.

Every kernel is a hand-written CUDA kernel of ``csrc/unet.cu`` behind the C ABI
``include/bbmg_learned.h``: 3x3x3 periodic convolutions as implicit GEMMs on the
tensor cores (BF16 operands, FP32 accumulation), their data and weight
gradients, pooling/upsampling, the 1x1 head, the MSE loss and Adam.  This
module only owns device memory (torch tensors as allocations) and sequences
the launches on torch's current stream.

Architecture (4 levels, 16/32/64/128 channels): two ReLU convolutions per
level, 2x average pooling down, nearest-neighbour upsampling up with the
encoder output concatenated after the upsampled channels, and a 1x1 head.
Weights are FP32 master copies ``w[tap][cin][cout]`` (tap = 9 dz + 3 dy + dx)
packed to BF16 before every forward.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import bbmg as B

CH = (16, 32, 64, 128)
CIN0 = 16  # the embedded input is padded to one MMA K-step


class Act(C.Structure):
    _fields_ = [("data", C.c_void_p), ("n", C.c_int), ("d", C.c_int), ("h", C.c_int), ("w", C.c_int),
                ("c", C.c_int), ("ld", C.c_int)]


NN_EXPORTS = ["nn_conv3", "nn_conv3_dgrad", "nn_conv3_wgrad", "nn_pack_weights", "nn_relu_bwd", "nn_pool2",
              "nn_pool2_bwd", "nn_up2", "nn_up2_bwd", "nn_embed", "nn_head", "nn_head_bwd", "nn_mse", "nn_adam",
              "nn_apply", "nn_tc_error"]

_NN = None


def lib():
    """The CUDA library with the nn_* signatures declared."""
    global _NN
    if _NN is not None:
        return _NN
    L = B.load()
    P, I, D, F, LL = C.c_void_p, C.c_int, C.c_double, C.c_float, C.c_longlong
    A = C.POINTER(Act)
    sig = {
        "nn_conv3": [A, P, P, A, I, P],
        "nn_conv3_dgrad": [A, P, A, P],
        "nn_conv3_wgrad": [A, A, P, P, P],
        "nn_pack_weights": [P, I, I, P, P, P],
        "nn_relu_bwd": [A, A, P],
        "nn_pool2": [A, A, P],
        "nn_pool2_bwd": [A, A, I, P],
        "nn_up2": [A, A, P],
        "nn_up2_bwd": [A, A, P],
        "nn_embed": [I, C.POINTER(P), C.POINTER(D), I, A, P],
        "nn_head": [A, P, P, P, P],
        "nn_head_bwd": [A, P, P, A, P, P, P],
        "nn_mse": [P, P, D, LL, P, P, P],
        "nn_adam": [P, P, P, P, LL, F, F, F, F, I, P],
        "nn_apply": [P, P, D, I, I, I, I, I, P, P],
        "nn_tc_error": [],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    _NN = L
    return L


def layer_spec(ch=CH, cin0=CIN0):
    """(name, cin, cout) of the 14 convolutions, in parameter order."""
    c1, c2, c3, c4 = ch
    return [("enc1a", cin0, c1), ("enc1b", c1, c1), ("enc2a", c1, c2), ("enc2b", c2, c2),
            ("enc3a", c2, c3), ("enc3b", c3, c3), ("bota", c3, c4), ("botb", c4, c4),
            ("dec3a", c4 + c3, c3), ("dec3b", c3, c3), ("dec2a", c3 + c2, c2), ("dec2b", c2, c2),
            ("dec1a", c2 + c1, c1), ("dec1b", c1, c1)]


def init_params(nf, ch=CH, seed=0):
    """He-normal convolution weights, zero biases, a small random head: the
    flat FP32 parameter vector (per convolution w[27][cin][cout] then b[cout];
    then the head's w[c1] and b)."""
    rng = np.random.default_rng(seed)
    parts = []
    for i, (_, cin, cout) in enumerate(layer_spec(ch)):
        fan = 27 * (nf if i == 0 else cin)
        w = rng.standard_normal((27, cin, cout)) * math.sqrt(2.0 / fan)
        if i == 0:
            w[:, nf:, :] = 0.0
        parts += [w.ravel(), np.zeros(cout)]
    parts += [rng.standard_normal(ch[0]) * 0.01, np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)


def _check(st, what):
    if st != 0:
        raise B.BBMGError(st, f"{what} failed")


class UNet:
    """The network's parameters, optimiser state and activation buffers."""

    def __init__(self, nf=2, ch=CH, seed=0, device="cuda", params=None):
        import torch
        if not 1 <= nf <= 4:
            raise ValueError("nf must be 1..4")
        self.torch = torch
        self.lib = lib()
        self.nf, self.ch, self.device = nf, tuple(ch), torch.device(device)
        self.spec = layer_spec(self.ch)
        self.offsets = []
        o = 0
        for _, cin, cout in self.spec:
            self.offsets.append((o, o + 27 * cin * cout))
            o += 27 * cin * cout + cout
        self.head_off = o
        self.nparam = o + self.ch[0] + 1
        p = init_params(nf, self.ch, seed) if params is None else np.asarray(params, np.float32)
        if p.size != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters, got {p.size}")
        self.params = torch.from_numpy(p.copy()).to(self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.t = 0
        self.packed = []
        for _, cin, cout in self.spec:
            self.packed.append((torch.empty(27 * cin * cout, dtype=torch.bfloat16, device=self.device),
                                torch.empty(27 * cin * cout, dtype=torch.bfloat16, device=self.device)))
        self._bufs = {}
        self.pack()

    # ------------------------------------------------------------ plumbing
    @property
    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _ptr(self, t, elem_off=0):
        return C.c_void_p(t.data_ptr() + elem_off * t.element_size())

    def _act(self, t, shape, c=None, off=0):
        n, d, h, w = shape
        ld = t.shape[-1]
        a = Act(t.data_ptr() + 2 * off, n, d, h, w, ld if c is None else c, ld)
        return C.byref(a), a

    def w_ptr(self, i):
        return self._ptr(self.params, self.offsets[i][0])

    def b_ptr(self, i):
        return self._ptr(self.params, self.offsets[i][1])

    def gw_ptr(self, i):
        return self._ptr(self.grads, self.offsets[i][0])

    def gb_ptr(self, i):
        return self._ptr(self.grads, self.offsets[i][1])

    def pack(self):
        s = self.stream
        for i, (_, cin, cout) in enumerate(self.spec):
            wt, wd = self.packed[i]
            _check(self.lib.nn_pack_weights(self.w_ptr(i), cin, cout, self._ptr(wt), self._ptr(wd), s), "pack")

    def buffers(self, shape, train):
        """Activation (and, for training, gradient) buffers of one input shape."""
        key = (tuple(shape), bool(train))
        if key in self._bufs:
            return self._bufs[key]
        torch = self.torch
        n, d, h, w = shape
        if d % 8 or h % 8 or w % 8:
            raise ValueError("spatial sizes must be multiples of 8 (three 2x poolings)")
        c1, c2, c3, c4 = self.ch
        sh = [(n, d >> l, h >> l, w >> l) for l in range(4)]
        V = [a * b * c * e for a, b, c, e in sh]

        def bf(l, c):
            return torch.empty((V[l], c), dtype=torch.bfloat16, device=self.device)

        b = {"shape": sh, "V": V,
             "x0": bf(0, CIN0), "t1": bf(0, c1), "cat1": bf(0, c2 + c1), "p1": bf(1, c1),
             "t2": bf(1, c2), "cat2": bf(1, c3 + c2), "p2": bf(2, c2), "t3": bf(2, c3), "cat3": bf(2, c4 + c3),
             "p3": bf(3, c3), "t4": bf(3, c4), "u4": bf(3, c4), "t3b": bf(2, c3), "u3": bf(2, c3),
             "t2b": bf(1, c2), "u2": bf(1, c2), "t1b": bf(0, c1), "u1": bf(0, c1),
             "out": torch.empty(V[0], dtype=torch.float32, device=self.device)}
        if train:
            b.update({"du1": bf(0, c1), "dt1b": bf(0, c1), "dcat1": bf(0, c2 + c1), "du2": bf(1, c2),
                      "dt2b": bf(1, c2), "dcat2": bf(1, c3 + c2), "du3": bf(2, c3), "dt3b": bf(2, c3),
                      "dcat3": bf(2, c4 + c3), "du4": bf(3, c4), "dt4": bf(3, c4), "dp3": bf(3, c3),
                      "dt3": bf(2, c3), "dp2": bf(2, c2), "dt2": bf(1, c2), "dp1": bf(1, c1), "dt1": bf(0, c1),
                      "dout": torch.empty(V[0], dtype=torch.float32, device=self.device),
                      "loss": torch.zeros(1, dtype=torch.float64, device=self.device)})
        self._bufs[key] = b
        return b

    # ------------------------------------------------------------ forward
    def embed(self, b, fields, scales, pool=1):
        """Input channels from FP64 fields on the network's grid (pool = 1) or
        on the grid twice as fine (pool = 2, 2x2x2 means)."""
        if len(fields) != self.nf:
            raise ValueError(f"expected {self.nf} input fields")
        fp = (C.c_void_p * self.nf)(*[f.data_ptr() for f in fields])
        sc = (C.c_double * self.nf)(*scales)
        x0, _k = self._act(b["x0"], b["shape"][0])
        _check(self.lib.nn_embed(self.nf, fp, sc, pool, x0, self.stream), "embed")

    def forward(self, b):
        """Run the network on b["x0"]; the prediction lands in b["out"]."""
        L, s = self.lib, self.stream
        c1, c2, c3, c4 = self.ch
        sh = b["shape"]
        keep = []

        def act(name, l, c=None, off=0):
            r, a = self._act(b[name], sh[l], c, off)
            keep.append(a)
            return r

        def conv(i, x, y):
            wt, _ = self.packed[i]
            _check(L.nn_conv3(x, self._ptr(wt), self.b_ptr(i), y, 1, s), self.spec[i][0])

        conv(0, act("x0", 0), act("t1", 0))
        conv(1, act("t1", 0), act("cat1", 0, c1, c2))                  # skip 1 = cat1[:, c2:]
        _check(L.nn_pool2(act("cat1", 0, c1, c2), act("p1", 1), s), "pool1")
        conv(2, act("p1", 1), act("t2", 1))
        conv(3, act("t2", 1), act("cat2", 1, c2, c3))                  # skip 2 = cat2[:, c3:]
        _check(L.nn_pool2(act("cat2", 1, c2, c3), act("p2", 2), s), "pool2")
        conv(4, act("p2", 2), act("t3", 2))
        conv(5, act("t3", 2), act("cat3", 2, c3, c4))                  # skip 3 = cat3[:, c4:]
        _check(L.nn_pool2(act("cat3", 2, c3, c4), act("p3", 3), s), "pool3")
        conv(6, act("p3", 3), act("t4", 3))
        conv(7, act("t4", 3), act("u4", 3))
        _check(L.nn_up2(act("u4", 3), act("cat3", 2, c4, 0), s), "up3")
        conv(8, act("cat3", 2), act("t3b", 2))
        conv(9, act("t3b", 2), act("u3", 2))
        _check(L.nn_up2(act("u3", 2), act("cat2", 1, c3, 0), s), "up2")
        conv(10, act("cat2", 1), act("t2b", 1))
        conv(11, act("t2b", 1), act("u2", 1))
        _check(L.nn_up2(act("u2", 1), act("cat1", 0, c2, 0), s), "up1")
        conv(12, act("cat1", 0), act("t1b", 0))
        conv(13, act("t1b", 0), act("u1", 0))
        _check(L.nn_head(act("u1", 0), self._ptr(self.params, self.head_off),
                         self._ptr(self.params, self.head_off + c1), self._ptr(b["out"]), s), "head")
        return b["out"]

    # ------------------------------------------------------------ backward
    def backward(self, b):
        """Gradients of the loss whose d/d(out) is in b["dout"], accumulated
        into self.grads (zero it first)."""
        L, s = self.lib, self.stream
        c1, c2, c3, c4 = self.ch
        sh = b["shape"]
        keep = []

        def act(name, l, c=None, off=0):
            r, a = self._act(b[name], sh[l], c, off)
            keep.append(a)
            return r

        def conv_bwd(i, x, y, dy, dx):
            """dy holds d/dy of the ReLU output y; turn it into d/d(pre-activation),
            then weight/bias gradients and (if dx) the input gradient."""
            _check(L.nn_relu_bwd(dy, y, s), "relu_bwd")
            _check(L.nn_conv3_wgrad(x, dy, self.gw_ptr(i), self.gb_ptr(i), s), "wgrad")
            if dx is not None:
                _, wd = self.packed[i]
                _check(L.nn_conv3_dgrad(dy, self._ptr(wd), dx, s), "dgrad")

        hw = self._ptr(self.params, self.head_off)
        _check(L.nn_head_bwd(act("u1", 0), hw, self._ptr(b["dout"]), act("du1", 0),
                             self._ptr(self.grads, self.head_off), self._ptr(self.grads, self.head_off + c1), s),
               "head_bwd")
        conv_bwd(13, act("t1b", 0), act("u1", 0), act("du1", 0), act("dt1b", 0))
        conv_bwd(12, act("cat1", 0), act("t1b", 0), act("dt1b", 0), act("dcat1", 0))
        _check(L.nn_up2_bwd(act("dcat1", 0, c2, 0), act("du2", 1), s), "up1_bwd")
        conv_bwd(11, act("t2b", 1), act("u2", 1), act("du2", 1), act("dt2b", 1))
        conv_bwd(10, act("cat2", 1), act("t2b", 1), act("dt2b", 1), act("dcat2", 1))
        _check(L.nn_up2_bwd(act("dcat2", 1, c3, 0), act("du3", 2), s), "up2_bwd")
        conv_bwd(9, act("t3b", 2), act("u3", 2), act("du3", 2), act("dt3b", 2))
        conv_bwd(8, act("cat3", 2), act("t3b", 2), act("dt3b", 2), act("dcat3", 2))
        _check(L.nn_up2_bwd(act("dcat3", 2, c4, 0), act("du4", 3), s), "up3_bwd")
        conv_bwd(7, act("t4", 3), act("u4", 3), act("du4", 3), act("dt4", 3))
        conv_bwd(6, act("p3", 3), act("t4", 3), act("dt4", 3), act("dp3", 3))
        _check(L.nn_pool2_bwd(act("dp3", 3), act("dcat3", 2, c3, c4), 1, s), "pool3_bwd")
        conv_bwd(5, act("t3", 2), act("cat3", 2, c3, c4), act("dcat3", 2, c3, c4), act("dt3", 2))
        conv_bwd(4, act("p2", 2), act("t3", 2), act("dt3", 2), act("dp2", 2))
        _check(L.nn_pool2_bwd(act("dp2", 2), act("dcat2", 1, c2, c3), 1, s), "pool2_bwd")
        conv_bwd(3, act("t2", 1), act("cat2", 1, c2, c3), act("dcat2", 1, c2, c3), act("dt2", 1))
        conv_bwd(2, act("p1", 1), act("t2", 1), act("dt2", 1), act("dp1", 1))
        _check(L.nn_pool2_bwd(act("dp1", 1), act("dcat1", 0, c1, c2), 1, s), "pool1_bwd")
        conv_bwd(1, act("t1", 0), act("cat1", 0, c1, c2), act("dcat1", 0, c1, c2), act("dt1", 0))
        conv_bwd(0, act("x0", 0), act("t1", 0), act("dt1", 0), None)

    # ------------------------------------------------------------ training
    def loss_grad(self, b, target, scale):
        """MSE of out against scale*target; dL/d(out) into b["dout"]; returns
        the loss tensor (device, not synchronised)."""
        b["loss"].zero_()
        _check(self.lib.nn_mse(self._ptr(b["out"]), self._ptr(target), float(scale), b["V"][0],
                               self._ptr(b["dout"]), self._ptr(b["loss"]), self.stream), "mse")
        return b["loss"]

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        _check(self.lib.nn_adam(self._ptr(self.params), self._ptr(self.grads), self._ptr(self.m), self._ptr(self.v),
                                self.nparam, lr, b1, b2, eps, self.t, self.stream), "adam")
        self.pack()

    def train_step(self, fields, scales, target, tscale, lr=1e-3):
        """One Adam step on one sample; returns the (device) MSE sum."""
        shape = (1,) + tuple(target.shape[-3:])
        b = self.buffers(shape, True)
        self.embed(b, fields, scales)
        self.forward(b)
        loss = self.loss_grad(b, target, tscale)
        self.grads.zero_()
        self.backward(b)
        self.adam(lr)
        return loss

    # ------------------------------------------------------------ inference
    def predict(self, fields, scales, shape):
        """Network output (FP32, voxels of `shape` = (n, d, h, w))."""
        b = self.buffers(tuple(shape), False)
        self.embed(b, fields, scales)
        return self.forward(b)

    def state(self):
        return {"nf": self.nf, "ch": self.ch, "params": self.params.detach().cpu().numpy()}


class LearnedGuess:
    """A trained UNet turned into an initial guess for bbmg_solve.

    Inputs of a solve: its rhs b, the previous solve's solution p_prev (the
    previous pressure increment) and (``use_rho``) the density.  The guess is
    p_prev + kappa max|b| net(...): the network predicts the change of the
    increment from one solve to the next, scaled by max|b| (the problem is
    linear in b, so the scale is taken out of the network), and a network that
    outputs zero reproduces the plain warm start.  With ``coarse`` the network
    runs on the grid twice as coarse (inputs pooled 2x2x2, prediction
    interpolated trilinearly back), which is how a network trained at 128^3
    serves a 256^3 solve."""

    def __init__(self, net: UNet, kappa=1.0, use_rho=True, ratio=1000.0, coarse=False):
        self.net, self.kappa, self.use_rho, self.ratio, self.coarse = net, float(kappa), use_rho, ratio, coarse
        if net.nf != (3 if use_rho else 2):
            raise ValueError("network input count does not match use_rho")

    def fields(self, rec):
        b, pp = rec["rhs"], rec["p_prev"]
        bmax = float(b.abs().max())
        pmax = float(pp.abs().max())
        f = [b, pp]
        s = [1.0 / bmax if bmax > 0 else 0.0, 1.0 / pmax if pmax > 0 else 0.0]
        if self.use_rho:
            f.append(rec["rho"])
            s.append(1.0 / self.ratio)
        return f, s, bmax

    def _input(self, rec, train):
        """Embed the fields into the network's input buffer; returns the buffers."""
        net = self.net
        nz, ny, nx = rec["rhs"].shape
        f, s, bmax = self.fields(rec)
        k = 2 if self.coarse else 1
        b = net.buffers((1, nz // k, ny // k, nx // k), train)
        net.embed(b, f, s, pool=k)
        return b, bmax

    def guess(self, rec, out):
        """Write the predicted dp (FP64, rec's shape) into `out`."""
        net = self.net
        b, bmax = self._input(rec, False)
        net.forward(b)
        n, d, h, w = b["shape"][0]
        base = rec["p_prev"].contiguous()
        _check(net.lib.nn_apply(net._ptr(base), net._ptr(b["out"]), self.kappa * bmax, n, d, h, w,
                                2 if self.coarse else 1, net._ptr(out), net.stream), "apply")
        return out

    def train_step(self, rec, lr):
        net = self.net
        b, bmax = self._input(rec, True)
        net.forward(b)
        loss = net.loss_grad(b, rec["target"], 1.0 / (self.kappa * bmax))
        net.grads.zero_()
        net.backward(b)
        net.adam(lr)
        return loss


class LearnedStage:
    """A trained UNet as the first stage of the pcg_bbox preconditioner
    (``BBMG.set_precond_stage``): z1 = kappa max|r| net(r / max|r|, rho / ratio),
    an approximation of A^-1 r that the FP32 V-cycle then corrects (the solver
    forms r - A z1 in FP64 and applies the V-cycle to it).  The network is the
    guess's architecture with the residual (and the density, for two-phase
    flow) as inputs; it is trained on (residual, error) pairs of the plain
    solver's own iterations (``stage_samples``).  ``coarse``: the network runs
    on the grid twice as coarse, as the guess does."""

    def __init__(self, net: UNet, kappa=1.0, use_rho=True, ratio=1000.0, coarse=False):
        self.net, self.kappa, self.use_rho, self.ratio, self.coarse = net, float(kappa), use_rho, ratio, coarse
        if net.nf != (2 if use_rho else 1):
            raise ValueError("network input count does not match use_rho")
        self.rho = None
        self.calls = 0

    def set_density(self, rho):
        """The density field of the operator being solved (FP64, the solve's shape)."""
        self.rho = rho

    def _fields(self, r, rho, rmax):
        f, s = [r], [1.0 / rmax if rmax > 0 else 0.0]
        if self.use_rho:
            f.append(rho)
            s.append(1.0 / self.ratio)
        return f, s

    def _buffers(self, shape, train):
        nz, ny, nx = shape
        k = 2 if self.coarse else 1
        return self.net.buffers((1, nz // k, ny // k, nx // k), train)

    def __call__(self, r, z, stream):
        """The stage: z = kappa max|r| net(r) on the solver's stream."""
        torch = self.net.torch
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            net = self.net
            rmax = float(r.abs().max())
            b = self._buffers(r.shape, False)
            f, s = self._fields(r, self.rho, rmax)
            net.embed(b, f, s, pool=2 if self.coarse else 1)
            net.forward(b)
            n, d, h, w = b["shape"][0]
            _check(net.lib.nn_apply(None, net._ptr(b["out"]), self.kappa * rmax, n, d, h, w,
                                    2 if self.coarse else 1, net._ptr(z), net.stream), "apply")
        self.calls += 1

    def train_step(self, rec, lr):
        """One Adam step on a (residual "r", error "e", density "rho") sample."""
        net = self.net
        r = rec["r"]
        rmax = float(r.abs().max())
        b = self._buffers(r.shape, True)
        f, s = self._fields(r, rec.get("rho"), rmax)
        net.embed(b, f, s, pool=2 if self.coarse else 1)
        net.forward(b)
        loss = net.loss_grad(b, rec["target"], 1.0 / (self.kappa * rmax))
        net.grads.zero_()
        net.backward(b)
        net.adam(lr)
        return loss


def apply_opr7(opr, x):
    """A x for a 7-point operator opr[k, j, i, st] (NGA2's stencil order) on a
    periodic (or wall-coefficient-zero) field x[k, j, i] (torch or numpy)."""
    roll = x.roll if hasattr(x, "roll") else (lambda sh, ax: np.roll(x, sh, ax))
    return (opr[..., 0] * x + opr[..., 1] * roll(-1, 2) + opr[..., 2] * roll(1, 2)
            + opr[..., 3] * roll(-1, 1) + opr[..., 4] * roll(1, 1)
            + opr[..., 5] * roll(-1, 0) + opr[..., 6] * roll(1, 0))


def stage_samples(handle, rec, iters=(0, 1, 2)):
    """(residual, error) pairs of the plain FP64 pcg_bbox on one sequence
    record: from the zero guess (r = rhs, e = dp) and after k = 1, 2, ...
    iterations (x_k from a solve stopped at maxit = k, r_k = rhs - A x_k,
    e_k = dp - x_k with the mean removed: the periodic problem fixes the
    solution up to a constant).  `handle` is a BBMG handle set up with rec's
    operator."""
    zeros = rec["rhs"].new_zeros
    out = []
    b, dp, opr = rec["rhs"], rec["dp"], rec["opr"]
    for k in iters:
        if k == 0:
            r, e = b.clone(), dp - dp.mean()
        else:
            x = zeros(b.shape)
            handle.set_convergence(k, 1e-30)
            handle.solve(b, x, allow=(0, 1))
            r = b - apply_opr7(opr, x)
            e = dp - x
            e = e - e.mean()
        out.append({"r": r.contiguous(), "e": e.contiguous(), "rho": rec.get("rho"), "k": k})
    return out


def fit_stage_kappa(samples):
    """Median of max|e| / max|r| over the samples."""
    return float(np.median([float(s["e"].abs().max()) / float(s["r"].abs().max()) for s in samples]))


def train_stage(stage: LearnedStage, samples, steps, lr=2e-3, lr_final=2e-4, seed=0):
    """Adam on randomly drawn (residual, error) samples, cosine learning-rate
    decay; returns the per-step losses (normalised MSE)."""
    torch = stage.net.torch
    rng = np.random.default_rng(seed)
    for smp in samples:
        if "target" not in smp:
            t = smp["e"]
            if stage.coarse:
                t = torch.nn.functional.avg_pool3d(t[None, None], 2)[0, 0]
            smp["target"] = t.contiguous()
    losses = []
    for t in range(steps):
        lr_t = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * t / max(1, steps)))
        smp = samples[int(rng.integers(len(samples)))]
        nvox = smp["r"].numel() // (8 if stage.coarse else 1)
        losses.append(float(stage.train_step(smp, lr_t)) / nvox)
    return losses


def fit_kappa(records):
    """Median of max|dp - p_prev| / max|rhs| over the training records."""
    r = [float((rec["dp"] - rec["p_prev"]).abs().max()) / float(rec["rhs"].abs().max()) for rec in records]
    return float(np.median(r))


def _with_target(rec, coarse):
    """The record with the network's target: the change from the warm start, on its grid."""
    if "target" not in rec:
        torch = __import__("torch")
        t = rec["dp"] - rec["p_prev"]
        if coarse:
            t = torch.nn.functional.avg_pool3d(t[None, None], 2)[0, 0]
        rec["target"] = t.contiguous()
    return rec


def train(guess: LearnedGuess, records, steps, lr=2e-3, lr_final=2e-4, seed=0, log=None, fetch=None):
    """Adam on randomly drawn training records with a cosine learning-rate
    decay; returns the per-step losses (normalised MSE).  ``fetch`` (optional)
    turns a stored record into the FP64 record a step trains on (for training
    sets kept in a compact form); without it the targets are cached on the
    records."""
    rng = np.random.default_rng(seed)
    if fetch is None:
        for rec in records:
            _with_target(rec, guess.coarse)
    losses = []
    for t in range(steps):
        lr_t = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * t / max(1, steps)))
        rec = records[int(rng.integers(len(records)))]
        if fetch is not None:
            rec = _with_target(fetch(rec), guess.coarse)
        nvox = rec["rhs"].numel() // (8 if guess.coarse else 1)
        losses.append(float(guess.train_step(rec, lr_t)) / nvox)
        if log and (t % 50 == 0 or t == steps - 1):
            log(t, losses[-1])
    return losses


def _time_forward(n, reps=5):
    """Average device milliseconds and TFLOP/s of one forward pass of the
    3-input U-Net on an n^3 grid (random inputs; for profiling)."""
    import torch
    net = UNet(nf=3, seed=0)
    rng = np.random.default_rng(0)
    V = n ** 3
    fields = [torch.from_numpy(rng.standard_normal(V)).cuda() for _ in range(3)]
    b = net.buffers((1, n, n, n), False)
    for _ in range(3):
        net.embed(b, fields, [1.0, 1.0, 1.0])
        net.forward(b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.embed(b, fields, [1.0, 1.0, 1.0])
        net.forward(b)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    depth = {"1": 0, "2": 1, "3": 2, "t": 3}
    flops = sum(2 * 27 * ci * co * (V >> (3 * depth[name[3] if name[:3] in ("enc", "dec") else "t"]))
                for name, ci, co in layer_spec())
    return {"n": n, "forward_ms": ms, "gflop": flops / 1e9, "tflops": flops / ms / 1e9}


if __name__ == "__main__":
    import sys
    print(_time_forward(int(sys.argv[1]) if len(sys.argv) > 1 else 128))
