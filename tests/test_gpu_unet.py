"""The surrogate's layers on the GPU.

The tcgen05 convolutions (forward, data gradient, weight gradient) are
checked against the C reference loops (oracle/conv_ref.c, double
accumulation) on bf16-representable inputs; the tolerance covers the bf16
rounding of the kernels' outputs (2^-8 relative) and FP32 accumulation.
The other layers are checked against numpy, and the whole U-Net's output and
weight gradients against torch-CPU autograd of the same network."""
import numpy as np
import pytest
import torch

from floodca_b200.lib import core
from oracle import pyconv

pytestmark = pytest.mark.gpu


def _bf(a):
    """Round to bf16-representable float32."""
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).float().numpy()


def _to_b(x):
    """[N, H, W, C] float -> bordered bf16 matrix on the GPU."""
    N, H, W, C = x.shape
    m = torch.zeros((N, H + 2, W + 2, C), dtype=torch.bfloat16)
    m[:, 1:H + 1, 1:W + 1, :] = torch.tensor(x)
    return m.view(-1, C).cuda()


def _from_b(m, N, H, W):
    return m.view(N, H + 2, W + 2, -1).float().cpu().numpy()


def _border_zero(m, N, H, W):
    a = m.view(N, H + 2, W + 2, -1).float().cpu()
    return (a[:, 0].abs().max() == 0 and a[:, -1].abs().max() == 0 and a[:, :, 0].abs().max() == 0
            and a[:, :, -1].abs().max() == 0)


def _p(t):
    import ctypes as C
    return C.c_void_p(t.data_ptr())


def _close(got, ref, rel):
    scale = float(np.sqrt(np.mean(ref.astype(np.float64) ** 2))) + 1e-30
    err = np.abs(got.astype(np.float64) - ref)
    return float((err / (np.abs(ref) * rel + rel * scale)).max())


CASES = [  # N, H, W, Cin, Cout
    (2, 16, 16, 16, 32), (2, 16, 16, 32, 32), (1, 16, 16, 96, 32), (1, 8, 8, 64, 128),
    (1, 8, 8, 384, 128), (1, 4, 4, 256, 256), (2, 12, 20, 192, 64), (3, 7, 9, 32, 64),
]


@pytest.mark.parametrize("N,H,W,Cin,Cout", CASES)
def test_conv_fwd_dgrad_wgrad(N, H, W, Cin, Cout):
    L = core()
    rng = np.random.default_rng(Cin * 7 + Cout)
    x = _bf(rng.standard_normal((N, H, W, Cin)))
    w = _bf(rng.standard_normal((Cout, 9, Cin)) / np.sqrt(9 * Cin))
    b = rng.standard_normal(Cout).astype(np.float32)
    dy = _bf(rng.standard_normal((N, H, W, Cout)))
    xb, dyb = _to_b(x), _to_b(dy)
    wf = torch.tensor(w).cuda()
    wb = torch.empty((Cout, 9, Cin), dtype=torch.bfloat16, device="cuda")
    wt = torch.empty((Cin, 9, Cout), dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_prep_weights(_p(wf), _p(wb), _p(wt), Cout, Cin, None) == 0
    bias = torch.tensor(b).cuda()
    y = torch.zeros((xb.shape[0], Cout), dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_conv_fwd(_p(xb), N, H, W, Cin, _p(wb), Cout, _p(bias), 1, _p(y), None) == 0
    dx = torch.zeros((xb.shape[0], Cin), dtype=torch.bfloat16, device="cuda")
    has_dx = Cin % 32 == 0     # the 16-channel input layer needs no data gradient
    if has_dx:
        assert L.fcab_unet_conv_dgrad(_p(dyb), N, H, W, Cout, _p(wt), Cin, _p(dx), None) == 0
    else:
        assert L.fcab_unet_conv_dgrad(_p(dyb), N, H, W, Cout, _p(wt), Cin, _p(dx), None) != 0
    dw = torch.zeros((Cout, 9, Cin), dtype=torch.float32, device="cuda")
    assert L.fcab_unet_conv_wgrad(_p(dyb), _p(xb), N, H, W, Cin, Cout, _p(dw), None) == 0
    torch.cuda.synchronize()
    assert L.fcab_unet_device_error() == 0
    assert _border_zero(y, N, H, W) and _border_zero(dx, N, H, W)
    yr = pyconv.fwd(x, w, b, relu=True)
    assert _close(_from_b(y, N, H, W)[:, 1:H + 1, 1:W + 1], yr, 8e-3) <= 1.0
    if has_dx:
        dxr = pyconv.dgrad(dy, w)
        assert _close(_from_b(dx, N, H, W)[:, 1:H + 1, 1:W + 1], dxr, 8e-3) <= 1.0
    dwr = pyconv.wgrad(dy, x)
    assert _close(dw.cpu().numpy(), dwr, 1e-4) <= 1.0


def test_conv_larger_than_one_wave():
    """Many CTAs (several per SM and more than one wave), 256x256 images."""
    L = core()
    N, H, W, Cin, Cout = 4, 256, 256, 32, 64
    rng = np.random.default_rng(3)
    x = _bf(rng.standard_normal((N, H, W, Cin)))
    w = _bf(rng.standard_normal((Cout, 9, Cin)) / np.sqrt(9 * Cin))
    xb = _to_b(x)
    wf = torch.tensor(w).cuda()
    wb = torch.empty((Cout, 9, Cin), dtype=torch.bfloat16, device="cuda")
    wt = torch.empty((Cin, 9, Cout), dtype=torch.bfloat16, device="cuda")
    L.fcab_unet_prep_weights(_p(wf), _p(wb), _p(wt), Cout, Cin, None)
    y = torch.zeros((xb.shape[0], Cout), dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_conv_fwd(_p(xb), N, H, W, Cin, _p(wb), Cout, None, 0, _p(y), None) == 0
    dw = torch.zeros((Cout, 9, Cin), dtype=torch.float32, device="cuda")
    dyb = _to_b(_bf(rng.standard_normal((N, H, W, Cout))))
    assert L.fcab_unet_conv_wgrad(_p(dyb), _p(xb), N, H, W, Cin, Cout, _p(dw), None) == 0
    torch.cuda.synchronize()
    assert L.fcab_unet_device_error() == 0
    # torch-CPU convolution as the second reference
    xt = torch.tensor(x).permute(0, 3, 1, 2)
    wt4 = torch.tensor(w).view(Cout, 3, 3, Cin).permute(0, 3, 1, 2)
    yr = torch.nn.functional.conv2d(xt, wt4, padding=1).permute(0, 2, 3, 1).numpy()
    assert _close(_from_b(y, N, H, W)[:, 1:H + 1, 1:W + 1], yr, 8e-3) <= 1.0
    dy = _from_b(dyb, N, H, W)[:, 1:H + 1, 1:W + 1]
    gw = torch.nn.grad.conv2d_weight(xt, wt4.shape, torch.tensor(dy).permute(0, 3, 1, 2), padding=1)
    gw = gw.permute(0, 2, 3, 1).reshape(Cout, 9, Cin).numpy()
    assert _close(dw.cpu().numpy(), gw, 1e-3) <= 1.0


def test_pool_upsample_concat_add_relu():
    L = core()
    rng = np.random.default_rng(1)
    N, H, W, C = 2, 8, 6, 32
    x = _bf(rng.standard_normal((N, H, W, C)))
    xb = _to_b(x)
    y = torch.zeros(((N) * (H // 2 + 2) * (W // 2 + 2), C), dtype=torch.bfloat16, device="cuda")
    idx = torch.empty((N, H // 2, W // 2, C), dtype=torch.uint8, device="cuda")
    assert L.fcab_unet_maxpool2(_p(xb), _p(y), _p(idx), N, H, W, C, None) == 0
    xr = x.reshape(N, H // 2, 2, W // 2, 2, C)
    ref = xr.max(axis=(2, 4))
    assert np.array_equal(_from_b(y, N, H // 2, W // 2)[:, 1:-1, 1:-1], ref)
    g = _bf(rng.standard_normal((N, H // 2, W // 2, C)))
    gb = _to_b(g)
    dx = torch.zeros_like(xb)
    assert L.fcab_unet_maxpool2_bwd(_p(gb), _p(idx), _p(dx), N, H, W, C, None) == 0
    dxr = np.zeros_like(x)
    am = xr.transpose(0, 1, 3, 5, 2, 4).reshape(N, H // 2, W // 2, C, 4).argmax(-1)
    for k in range(4):
        dxr[:, (k >> 1)::2, (k & 1)::2, :] = np.where(am == k, g, 0)
    assert np.array_equal(_from_b(dx, N, H, W)[:, 1:-1, 1:-1], dxr)
    # upsample and its gradient
    up = torch.zeros(((N) * (2 * H + 2) * (2 * W + 2), C), dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_upsample2(_p(xb), _p(up), N, H, W, C, None) == 0
    assert np.array_equal(_from_b(up, N, 2 * H, 2 * W)[:, 1:-1, 1:-1],
                          x.repeat(2, axis=1).repeat(2, axis=2))
    gu = _bf(rng.standard_normal((N, 2 * H, 2 * W, C)))
    gub = _to_b(gu)
    gd = torch.zeros_like(xb)
    assert L.fcab_unet_upsample2_bwd(_p(gub), _p(gd), N, H, W, C, None) == 0
    s = gu.reshape(N, H, 2, W, 2, C).sum(axis=(2, 4))
    assert np.allclose(_from_b(gd, N, H, W)[:, 1:-1, 1:-1], s, rtol=8e-3, atol=1e-2)
    # concat and split
    b2 = _bf(rng.standard_normal((N, H, W, 16)))
    bb = _to_b(b2)
    cat = torch.zeros((xb.shape[0], C + 16), dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_concat(_p(xb), C, _p(bb), 16, _p(cat), N, H, W, 0, None) == 0
    assert np.array_equal(_from_b(cat, N, H, W)[:, 1:-1, 1:-1], np.concatenate([x, b2], -1))
    ga, gb2 = torch.zeros_like(xb), torch.zeros_like(bb)
    assert L.fcab_unet_concat(_p(ga), C, _p(gb2), 16, _p(cat), N, H, W, 1, None) == 0
    assert torch.equal(ga, xb) and torch.equal(gb2, bb)
    # add, relu backward
    s2 = xb.clone()
    assert L.fcab_unet_add(_p(s2), _p(xb), s2.numel(), None) == 0
    assert torch.equal(s2, (xb.float() * 2).to(torch.bfloat16))
    gg = torch.ones_like(xb)
    assert L.fcab_unet_relu_bwd(_p(gg), _p(xb), gg.numel(), None) == 0
    assert torch.equal(gg, (xb.float() > 0).to(torch.bfloat16))
    torch.cuda.synchronize()


def test_dropout_bias_head_adam():
    L = core()
    rng = np.random.default_rng(2)
    n = 1 << 20
    x = torch.ones(n, dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_dropout(_p(x), n, 0.25, 7, None) == 0
    xf = x.float().cpu().numpy()
    kept = xf != 0
    assert abs(kept.mean() - 0.75) < 0.005
    assert np.allclose(xf[kept], 1 / 0.75, rtol=4e-3)
    x2 = torch.ones(n, dtype=torch.bfloat16, device="cuda")
    L.fcab_unet_dropout(_p(x2), n, 0.25, 7, None)
    assert torch.equal(x, x2)                      # same seed, same mask
    # bias gradient
    g = torch.tensor(_bf(rng.standard_normal((5000, 64)))).to(torch.bfloat16).cuda()
    db = torch.zeros(64, device="cuda")
    assert L.fcab_unet_bias_grad(_p(g), 5000, 64, _p(db), None) == 0
    assert np.allclose(db.cpu().numpy(), g.float().sum(0).cpu().numpy(), rtol=1e-4, atol=1e-3)
    # head forward / backward
    N, H, W, C = 2, 6, 5, 32
    a = _bf(rng.standard_normal((N, H, W, C)))
    ab = _to_b(a)
    hw = torch.tensor(rng.standard_normal(C).astype(np.float32)).cuda()
    hb = torch.tensor([0.3], device="cuda")
    out = torch.empty((N, H, W), device="cuda")
    assert L.fcab_unet_head_fwd(_p(ab), _p(hw), _p(hb), _p(out), N, H, W, C, None) == 0
    ref = a @ hw.cpu().numpy() + 0.3
    assert np.allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=1e-5)
    tgt = torch.tensor(rng.standard_normal((N, H, W)).astype(np.float32)).cuda()
    dx = torch.zeros_like(ab)
    dw = torch.zeros(C, device="cuda")
    dbh = torch.zeros(1, device="cuda")
    loss = torch.zeros(1, device="cuda")
    assert L.fcab_unet_head_bwd(_p(ab), _p(hw), _p(out), _p(tgt), _p(dx), _p(dw), _p(dbh),
                                _p(loss), N, H, W, C, None) == 0
    e = out.cpu().numpy() - tgt.cpu().numpy()
    d = 2 * e / e.size
    assert np.isclose(loss.item(), (e ** 2).sum(), rtol=1e-5)
    assert np.allclose(dbh.item(), d.sum(), rtol=1e-4, atol=1e-7)
    assert np.allclose(dw.cpu().numpy(), np.einsum("nhw,nhwc->c", d, a), rtol=1e-4, atol=1e-7)
    assert np.allclose(_from_b(dx, N, H, W)[:, 1:-1, 1:-1], d[..., None] * hw.cpu().numpy(),
                       rtol=8e-3, atol=1e-9)
    # Adam
    w = torch.tensor(rng.standard_normal(1000).astype(np.float32)).cuda()
    gr = torch.tensor(rng.standard_normal(1000).astype(np.float32)).cuda()
    m, v = torch.zeros_like(w), torch.zeros_like(w)
    w0 = w.cpu().numpy().copy()
    for t in (1, 2):
        assert L.fcab_unet_adam(_p(w), _p(gr), _p(m), _p(v), 1000, 1e-2, 0.9, 0.999, 1e-8, t,
                                0.0, None) == 0
    gn = gr.cpu().numpy()
    mm, vv, ww = np.zeros(1000), np.zeros(1000), w0.astype(np.float64)
    for t in (1, 2):
        mm = 0.9 * mm + 0.1 * gn
        vv = 0.999 * vv + 0.001 * gn * gn
        ww -= 1e-2 * (mm / (1 - 0.9 ** t)) / (np.sqrt(vv / (1 - 0.999 ** t)) + 1e-8)
    assert np.allclose(w.cpu().numpy(), ww, rtol=1e-5, atol=1e-6)


def _bf16_round(t):
    """Rounds to bf16 in the forward pass with an identity gradient, where the
    kernels store bf16 activations (so ReLU masks and pooling arg maxes see
    the same values)."""
    return t + (t.to(torch.bfloat16).float() - t).detach()


def _torch_unet(model, inp, target):
    """The same network in torch (fp32 on the CPU) with the model's bf16
    weights and bf16-rounded activations; returns the output and the
    gradients of the mean squared error."""
    import torch.nn.functional as F
    convs = list(model.convs())
    ws, bs = [], []
    for c in convs:
        w = c.wb.float().cpu().view(c.cout, 3, 3, c.cin).permute(0, 3, 1, 2).contiguous()
        ws.append(w.requires_grad_())
        bs.append(c.b.cpu().clone().requires_grad_())
    hw = model.hw.cpu().clone().requires_grad_()
    hb = model.hb.cpu().clone().requires_grad_()
    x = _bf16_round(torch.tensor(inp).permute(0, 3, 1, 2))
    x = F.pad(x, (0, 0, 0, 0, 0, 16 - x.shape[1]))
    k = 0

    def conv(t):
        nonlocal k
        y = _bf16_round(F.relu(F.conv2d(t, ws[k], bs[k], padding=1)))
        k += 1
        return y
    skips = []
    for lvl in range(4):
        x = conv(conv(x))
        if lvl < 3:
            skips.append(x)
            x = F.max_pool2d(x, 2)
    for lvl in (2, 1, 0):
        x = F.interpolate(x, scale_factor=2, mode="nearest")
        x = torch.cat([x, skips[lvl]], 1)
        x = conv(conv(x))
    out = torch.einsum("nchw,c->nhw", x, hw) + hb
    loss = ((out - torch.tensor(target)) ** 2).mean()
    loss.backward()
    return out.detach().numpy(), ws, bs, hw, hb


def test_unet_forward_backward_matches_torch():
    from floodca_b200.unet import UNet
    N, H, W = 2, 32, 32
    rng = np.random.default_rng(4)
    inp = rng.standard_normal((N, H, W, 4)).astype(np.float32)
    target = rng.standard_normal((N, H, W)).astype(np.float32)
    model = UNet(seed=1)
    model.prep()
    out = model.forward(torch.tensor(inp).cuda()).cpu().numpy()
    model.backward(torch.tensor(target).cuda())
    torch.cuda.synchronize()
    assert model.device_error() == 0
    ref, ws, bs, hw, hb = _torch_unet(model, inp, target)
    rel = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert rel < 3e-2, rel
    for c, w, b in zip(model.convs(), ws, bs):
        gw = w.grad.permute(0, 2, 3, 1).reshape(c.cout, 9, c.cin).numpy()
        got = c.dw.cpu().numpy()
        if c.cin == 16:
            gw, got = gw[:, :, :4], got[:, :, :4]
        cos = float((gw * got).sum() / (np.linalg.norm(gw) * np.linalg.norm(got) + 1e-30))
        nrel = float(np.linalg.norm(gw - got) / (np.linalg.norm(gw) + 1e-30))
        assert cos > 0.995 and nrel < 0.1, (c.cin, c.cout, cos, nrel)
        gb = b.grad.numpy()
        assert np.linalg.norm(gb - c.db.cpu().numpy()) <= 0.1 * np.linalg.norm(gb) + 1e-6
    assert np.allclose(model.dhw.cpu().numpy(), hw.grad.numpy(), rtol=0.05, atol=1e-4)


def test_fused_upcat_and_pool_backward_add():
    """upcat = concat(upsample2(coarse), skip); upcat_bwd = upsample2_bwd of
    the first channels; maxpool2_bwd_add = maxpool2_bwd + a channel slice."""
    L = core()
    rng = np.random.default_rng(5)
    N, H, W, C1, C2 = 2, 8, 12, 64, 32
    co = _bf(rng.standard_normal((N, H // 2, W // 2, C1)))
    sk = _bf(rng.standard_normal((N, H, W, C2)))
    cob, skb = _to_b(co), _to_b(sk)
    cat = torch.zeros((skb.shape[0], C1 + C2), dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_upcat(_p(cob), C1, _p(skb), C2, _p(cat), N, H, W, None) == 0
    ref = np.concatenate([co.repeat(2, axis=1).repeat(2, axis=2), sk], -1)
    assert np.array_equal(_from_b(cat, N, H, W)[:, 1:-1, 1:-1], ref)
    g = _bf(rng.standard_normal((N, H, W, C1 + C2)))
    gb = _to_b(g)
    gco = torch.zeros_like(cob)
    assert L.fcab_unet_upcat_bwd(_p(gb), C1, C2, _p(gco), N, H, W, None) == 0
    s = g[..., :C1].reshape(N, H // 2, 2, W // 2, 2, C1).sum(axis=(2, 4))
    assert np.allclose(_from_b(gco, N, H // 2, W // 2)[:, 1:-1, 1:-1], s, rtol=8e-3, atol=1e-2)
    # pooling of the skip tensor and its gradient plus the concat slice
    pooled = torch.zeros_like(cob[:, :C2].contiguous())
    idx = torch.empty((N, H // 2, W // 2, C2), dtype=torch.uint8, device="cuda")
    assert L.fcab_unet_maxpool2(_p(skb), _p(pooled), _p(idx), N, H, W, C2, None) == 0
    dyp = _to_b(_bf(rng.standard_normal((N, H // 2, W // 2, C2))))
    plain = torch.zeros_like(skb)
    assert L.fcab_unet_maxpool2_bwd(_p(dyp), _p(idx), _p(plain), N, H, W, C2, None) == 0
    fused = torch.zeros_like(skb)
    assert L.fcab_unet_maxpool2_bwd_add(_p(dyp), _p(idx), _p(gb), C1 + C2, C1, _p(fused), N, H, W,
                                        C2, None) == 0
    want = _from_b(plain, N, H, W)[:, 1:-1, 1:-1] + g[..., C1:]
    assert np.allclose(_from_b(fused, N, H, W)[:, 1:-1, 1:-1], want, rtol=8e-3, atol=1e-2)
    assert _border_zero(fused, N, H, W) and _border_zero(cat, N, H, W)


def test_bounded_wait_gives_up_and_reports():
    """The conv kernels' mbarrier wait on a phase that never completes (no
    arrival ever comes) gives up after its limit, records error 10 and
    returns; the context stays usable and a following convolution is
    correct with no error recorded."""
    L = core()
    assert L.fcab_unet_device_error() == 0
    assert L.fcab_unet_wait_probe(0, None) != 0                 # limit out of range
    assert L.fcab_unet_wait_probe(1 << 20, None) == 0           # about half a millisecond
    torch.cuda.synchronize()
    assert L.fcab_unet_device_error() == 10
    assert L.fcab_unet_device_error() == 0                      # read clears it
    N, H, W, Cin, Cout = 1, 8, 8, 16, 32
    rng = np.random.default_rng(4)
    x = _bf(rng.standard_normal((N, H, W, Cin)))
    w = _bf(rng.standard_normal((Cout, 9, Cin)) / 12.0)
    xb = _to_b(x)
    wf = torch.tensor(w).cuda()
    wb = torch.empty((Cout, 9, Cin), dtype=torch.bfloat16, device="cuda")
    wt = torch.empty((Cin, 9, Cout), dtype=torch.bfloat16, device="cuda")
    L.fcab_unet_prep_weights(_p(wf), _p(wb), _p(wt), Cout, Cin, None)
    y = torch.zeros((xb.shape[0], Cout), dtype=torch.bfloat16, device="cuda")
    assert L.fcab_unet_conv_fwd(_p(xb), N, H, W, Cin, _p(wb), Cout, None, 0, _p(y), None) == 0
    torch.cuda.synchronize()
    assert L.fcab_unet_device_error() == 0
    xt = torch.tensor(x).permute(0, 3, 1, 2)
    wt4 = torch.tensor(w).view(Cout, 3, 3, Cin).permute(0, 3, 1, 2)
    yr = torch.nn.functional.conv2d(xt, wt4, padding=1).permute(0, 2, 3, 1).numpy()
    assert _close(_from_b(y, N, H, W)[:, 1:H + 1, 1:W + 1], yr, 8e-3) <= 1.0
