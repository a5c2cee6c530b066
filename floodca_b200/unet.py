"""The flood-depth surrogate: a 4-level U-Net on 256 x 256 grids.

Input channels: elevation relief, Manning n, rain intensity, rain duration
(4 channels, stored in 16). Output: peak depth in a transformed scale.
Encoder levels at 256/128/64/32 with 32/64/128/256 channels (two 3x3
convolutions + ReLU each, 2x2 max pooling between); the decoder upsamples
(nearest 2x) and concatenates the skip connection in one pass, then applies two 3x3
convolutions + ReLU; a 1x1 head gives one channel. Dropout (MC dropout at
inference) follows the bottleneck and the two deeper decoder levels.

Weights are FP32 masters updated by Adam; every step uses their BF16 copies
(forward [Cout][9][Cin] and the flipped, transposed data-gradient weights).
Activations are BF16 matrices of NHWC images with a one-pixel zero border
(floodca_b200/csrc/unet_tc.cu). Every layer runs a kernel of the core
library (tcgen05 tensor cores for the 3x3 convolutions); torch only
allocates device memory.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from .lib import FcabError, check, core, last_error

CIN_PAD = 16
CHANNELS = (32, 64, 128, 256)


def _p(t):
    return C.c_void_p(t.data_ptr())


def bordered(N, H, W, Cc, device="cuda"):
    import torch
    return torch.zeros((N * (H + 2) * (W + 2), Cc), dtype=torch.bfloat16, device=device)


def interior_view(m, N, H, W):
    """[N*(H+2)*(W+2), C] -> [N, H, W, C] view of the interior pixels."""
    return m.view(N, H + 2, W + 2, -1)[:, 1:H + 1, 1:W + 1, :]


class Conv3:
    """3x3 convolution, FP32 master weights and Adam state."""

    def __init__(self, cin, cout, rng, cin_real=None, device="cuda"):
        import torch
        self.cin, self.cout = cin, cout
        fan = 9 * (cin_real or cin)
        w = rng.standard_normal((cout, 9, cin)).astype(np.float32) * math.sqrt(2.0 / fan)
        if cin_real is not None:
            w[:, :, cin_real:] = 0.0
        self.w = torch.tensor(w, device=device)
        self.b = torch.zeros(cout, device=device)
        self.wb = torch.empty((cout, 9, cin), dtype=torch.bfloat16, device=device)
        self.wt = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device=device)
        self.dw = torch.zeros_like(self.w)
        self.db = torch.zeros_like(self.b)
        self.state = [torch.zeros_like(self.w), torch.zeros_like(self.w),
                      torch.zeros_like(self.b), torch.zeros_like(self.b)]

    def params(self):
        return [(self.w, self.dw, self.state[0], self.state[1]),
                (self.b, self.db, self.state[2], self.state[3])]

    def prep(self, L, st):
        check(L.fcab_unet_prep_weights(_p(self.w), _p(self.wb), _p(self.wt), self.cout, self.cin,
                                       st), "prep_weights")


class UNet:
    def __init__(self, seed=0, p_drop=0.1, device="cuda"):
        self.L = core()
        self.device = device
        rng = np.random.default_rng(seed)
        c0, c1, c2, c3 = CHANNELS
        self.p_drop = p_drop
        self.enc = [
            (Conv3(CIN_PAD, c0, rng, cin_real=4, device=device), Conv3(c0, c0, rng, device=device)),
            (Conv3(c0, c1, rng, device=device), Conv3(c1, c1, rng, device=device)),
            (Conv3(c1, c2, rng, device=device), Conv3(c2, c2, rng, device=device)),
            (Conv3(c2, c3, rng, device=device), Conv3(c3, c3, rng, device=device)),
        ]
        self.dec = [   # deepest first: level 2, 1, 0
            (Conv3(c3 + c2, c2, rng, device=device), Conv3(c2, c2, rng, device=device)),
            (Conv3(c2 + c1, c1, rng, device=device), Conv3(c1, c1, rng, device=device)),
            (Conv3(c1 + c0, c0, rng, device=device), Conv3(c0, c0, rng, device=device)),
        ]
        import torch
        self.hw = torch.tensor(rng.standard_normal(c0).astype(np.float32) * math.sqrt(1.0 / c0),
                               device=device)
        self.hb = torch.zeros(1, device=device)
        self.dhw = torch.zeros_like(self.hw)
        self.dhb = torch.zeros_like(self.hb)
        self.hstate = [torch.zeros_like(self.hw), torch.zeros_like(self.hw),
                       torch.zeros_like(self.hb), torch.zeros_like(self.hb)]
        self.step_t = 0
        self._bufs = {}

    def convs(self):
        for pair in self.enc + self.dec:
            yield from pair

    def prep(self, st=None):
        for c in self.convs():
            c.prep(self.L, st)

    # -- buffers -------------------------------------------------------------
    def _buf(self, key, N, H, W, Cc):
        k = (key, N, H, W, Cc)
        b = self._bufs.get(k)
        if b is None:
            b = bordered(N, H, W, Cc, self.device)
            self._bufs[k] = b
        return b

    def _idx(self, key, N, H, W, Cc):
        import torch
        k = (key, N, H, W, Cc, "idx")
        b = self._bufs.get(k)
        if b is None:
            b = torch.empty((N, H // 2, W // 2, Cc), dtype=torch.uint8, device=self.device)
            self._bufs[k] = b
        return b

    # -- forward ---------------------------------------------------------------
    def _conv(self, conv, x, N, H, W, key, st):
        y = self._buf(key, N, H, W, conv.cout)
        check(self.L.fcab_unet_conv_fwd(_p(x), N, H, W, conv.cin, _p(conv.wb), conv.cout,
                                        _p(conv.b), 1, _p(y), st), "conv_fwd")
        return y

    def _drop(self, y, seed, st):
        check(self.L.fcab_unet_dropout(_p(y), y.numel(), self.p_drop, seed & 0xFFFFFFFF, st),
              "dropout")

    def forward(self, inp, dropout_seed=None, st=None):
        """inp: fp32 [N, H, W, 4] (device). Returns the fp32 head output
        [N, H, W]; keeps what backward needs. dropout_seed: None disables
        dropout (deterministic prediction)."""
        import torch
        L = self.L
        N, H, W, cs = inp.shape
        self.N, self.H, self.W = N, H, W
        self.seed = dropout_seed
        x = self._buf("in", N, H, W, CIN_PAD)
        check(L.fcab_unet_pack_input(_p(inp), cs, _p(x), CIN_PAD, N, H, W, st), "pack_input")
        acts = {"x0": x}
        skips = []
        h, w = H, W
        cur = x
        for lvl, (ca, cb) in enumerate(self.enc):
            a = self._conv(ca, cur, N, h, w, f"e{lvl}a", st)
            b = self._conv(cb, a, N, h, w, f"e{lvl}b", st)
            acts[f"e{lvl}a"], acts[f"e{lvl}b"] = a, b
            if lvl == 3:
                if dropout_seed is not None:
                    self._drop(b, dropout_seed * 16 + 1, st)
                cur = b
                break
            skips.append((b, h, w, cb.cout))
            pooled = self._buf(f"p{lvl}", N, h // 2, w // 2, cb.cout)
            idx = self._idx(f"p{lvl}", N, h, w, cb.cout)
            check(L.fcab_unet_maxpool2(_p(b), _p(pooled), _p(idx), N, h, w, cb.cout, st), "maxpool")
            acts[f"p{lvl}"] = pooled
            cur, h, w = pooled, h // 2, w // 2
        cch = self.enc[3][1].cout
        for j, (ca, cb) in enumerate(self.dec):
            lvl = 2 - j
            skip, hs, ws, cs_ = skips[lvl]
            cat = self._buf(f"c{lvl}", N, hs, ws, cch + cs_)
            check(L.fcab_unet_upcat(_p(cur), cch, _p(skip), cs_, _p(cat), N, hs, ws, st), "upcat")
            a = self._conv(ca, cat, N, hs, ws, f"d{lvl}a", st)
            b = self._conv(cb, a, N, hs, ws, f"d{lvl}b", st)
            acts[f"c{lvl}"], acts[f"d{lvl}a"], acts[f"d{lvl}b"] = cat, a, b
            if dropout_seed is not None and lvl > 0:
                self._drop(b, dropout_seed * 16 + 2 + lvl, st)
            cur, h, w, cch = b, hs, ws, cb.cout
        out = self._bufs.get(("out", N, H, W))
        if out is None:
            out = torch.empty((N, H, W), dtype=torch.float32, device=self.device)
            self._bufs[("out", N, H, W)] = out
        check(L.fcab_unet_head_fwd(_p(cur), _p(self.hw), _p(self.hb), _p(out), N, H, W, cch, st),
              "head_fwd")
        self.acts = acts
        self.out = out
        return out

    # -- backward --------------------------------------------------------------
    def _conv_bwd(self, conv, g, x, y, N, H, W, key, need_dx, st, drop_seed=None):
        """g: gradient at the conv's (post-ReLU, post-dropout) output y."""
        L = self.L
        if drop_seed is not None:
            self._drop(g, drop_seed, st)
        check(L.fcab_unet_relu_bwd(_p(g), _p(y), g.numel(), st), "relu_bwd")
        check(L.fcab_unet_bias_grad(_p(g), g.shape[0], conv.cout, _p(conv.db), st), "bias_grad")
        check(L.fcab_unet_conv_wgrad(_p(g), _p(x), N, H, W, conv.cin, conv.cout, _p(conv.dw), st),
              "wgrad")
        if not need_dx:
            return None
        dx = self._buf(key, N, H, W, conv.cin)
        check(L.fcab_unet_conv_dgrad(_p(g), N, H, W, conv.cout, _p(conv.wt), conv.cin, _p(dx), st),
              "dgrad")
        return dx

    def backward(self, target, st=None) -> None:
        """Gradients of the mean squared error between the head output and
        target (fp32 [N, H, W]) into every dw/db; the loss sum goes to
        self.loss_sum (device)."""
        import torch
        L = self.L
        N, H, W = self.N, self.H, self.W
        A = self.acts
        seed = self.seed
        for t in (self.dhw, self.dhb):
            t.zero_()
        for c in self.convs():
            c.dw.zero_()
            c.db.zero_()
        self.loss_sum = torch.zeros(1, device=self.device)
        c0 = self.dec[2][1].cout
        g = self._buf("g_head", N, H, W, c0)
        check(L.fcab_unet_head_bwd(_p(A["d0b"]), _p(self.hw), _p(self.out), _p(target), _p(g),
                                   _p(self.dhw), _p(self.dhb), _p(self.loss_sum), N, H, W, c0, st),
              "head_bwd")
        # decoder, level 0 up to 2
        sizes = [(H >> l, W >> l) for l in range(4)]
        skip_grads = {}
        for j in (2, 1, 0):
            lvl = 2 - j
            ca, cb = self.dec[j]
            h, w = sizes[lvl]
            ds = None if (seed is None or lvl == 0) else seed * 16 + 2 + lvl
            ga = self._conv_bwd(cb, g, A[f"d{lvl}a"], A[f"d{lvl}b"], N, h, w, f"gd{lvl}a", True, st,
                                drop_seed=ds)
            gc = self._conv_bwd(ca, ga, A[f"c{lvl}"], A[f"d{lvl}a"], N, h, w, f"gc{lvl}", True, st)
            cup = ca.cin - self.enc[lvl][1].cout
            cs_ = self.enc[lvl][1].cout
            # the skip's share stays in gc until the pooling's backward adds it
            skip_grads[lvl] = (gc, ca.cin, cup)
            hd, wd = sizes[lvl + 1]
            g = self._buf(f"gdn{lvl}", N, hd, wd, cup)
            check(L.fcab_unet_upcat_bwd(_p(gc), cup, cs_, _p(g), N, h, w, st), "upcat_bwd")
        # encoder, bottleneck down to level 0
        for lvl in (3, 2, 1, 0):
            ca, cb = self.enc[lvl]
            h, w = sizes[lvl]
            if lvl < 3:
                # gradient at e{lvl}b: through the pooling plus the skip
                gb = self._buf(f"ge{lvl}b", N, h, w, cb.cout)
                idx = self._idx(f"p{lvl}", N, h, w, cb.cout)
                gc, ctot, off = skip_grads[lvl]
                check(L.fcab_unet_maxpool2_bwd_add(_p(g), _p(idx), _p(gc), ctot, off, _p(gb), N, h,
                                                   w, cb.cout, st), "maxpool_bwd")
                g = gb
            ds = (seed * 16 + 1) if (seed is not None and lvl == 3) else None
            xin = A["x0"] if lvl == 0 else A[f"p{lvl - 1}"]
            ga = self._conv_bwd(cb, g, A[f"e{lvl}a"], A[f"e{lvl}b"], N, h, w, f"ge{lvl}a", True, st,
                                drop_seed=ds)
            g = self._conv_bwd(ca, ga, xin, A[f"e{lvl}a"], N, h, w, f"gx{lvl}", lvl > 0, st)

    # -- optimiser -------------------------------------------------------------
    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0, st=None):
        self.step_t += 1
        L = self.L
        groups = [p for c in self.convs() for p in c.params()]
        groups += [(self.hw, self.dhw, self.hstate[0], self.hstate[1]),
                   (self.hb, self.dhb, self.hstate[2], self.hstate[3])]
        for w, g, m, v in groups:
            check(L.fcab_unet_adam(_p(w), _p(g), _p(m), _p(v), w.numel(), lr, b1, b2, eps,
                                   self.step_t, wd, st), "adam")
        self.prep(st)

    def device_error(self) -> int:
        return int(self.L.fcab_unet_device_error())

    def flops_forward(self, N, H, W) -> float:
        """Multiply-adds x 2 of the 3x3 convolutions (with real input
        channels), per forward pass of N images."""
        f = 0.0
        for lvl, (ca, cb) in enumerate(self.enc):
            px = N * (H >> lvl) * (W >> lvl)
            cin = 4 if lvl == 0 else ca.cin
            f += 2.0 * px * 9 * (cin * ca.cout + cb.cin * cb.cout)
        for j, (ca, cb) in enumerate(self.dec):
            lvl = 2 - j
            px = N * (H >> lvl) * (W >> lvl)
            f += 2.0 * px * 9 * (ca.cin * ca.cout + cb.cin * cb.cout)
        return f

    def state_dict(self) -> dict:
        d = {}
        for i, c in enumerate(self.convs()):
            d[f"w{i}"] = c.w.detach().cpu().numpy()
            d[f"b{i}"] = c.b.detach().cpu().numpy()
        d["hw"] = self.hw.cpu().numpy()
        d["hb"] = self.hb.cpu().numpy()
        return d

    def load_state_dict(self, d: dict) -> None:
        import torch
        for i, c in enumerate(self.convs()):
            c.w.copy_(torch.as_tensor(d[f"w{i}"]))
            c.b.copy_(torch.as_tensor(d[f"b{i}"]))
        self.hw.copy_(torch.as_tensor(d["hw"]))
        self.hb.copy_(torch.as_tensor(d["hb"]))
        self.prep()
