"""The CPU reference of the surrogate's 3x3 convolutions (oracle/conv_ref.c)
against torch's CPU convolution and its autograd gradients."""
import numpy as np
import torch

from oracle import pyconv


def _torch_w(w):
    co, _, ci = w.shape
    return torch.tensor(w).view(co, 3, 3, ci).permute(0, 3, 1, 2).contiguous()


def test_conv_ref_matches_torch():
    rng = np.random.default_rng(0)
    for N, H, W, ci, co in [(2, 6, 5, 3, 4), (1, 9, 7, 16, 32), (2, 4, 4, 8, 8)]:
        x = rng.standard_normal((N, H, W, ci)).astype(np.float32)
        w = rng.standard_normal((co, 9, ci)).astype(np.float32)
        b = rng.standard_normal(co).astype(np.float32)
        dy = rng.standard_normal((N, H, W, co)).astype(np.float32)
        xt = torch.tensor(x).permute(0, 3, 1, 2).requires_grad_()
        wt = _torch_w(w).requires_grad_()
        out = torch.nn.functional.conv2d(xt, wt, torch.tensor(b), padding=1)
        out.backward(torch.tensor(dy).permute(0, 3, 1, 2))
        y = out.detach().permute(0, 2, 3, 1).numpy()
        assert np.allclose(pyconv.fwd(x, w, b), y, atol=1e-4)
        assert np.allclose(pyconv.fwd(x, w, b, relu=True), np.maximum(y, 0), atol=1e-4)
        assert np.allclose(pyconv.dgrad(dy, w), xt.grad.permute(0, 2, 3, 1).numpy(), atol=1e-4)
        gw = wt.grad.permute(0, 2, 3, 1).reshape(co, 9, ci).numpy()
        assert np.allclose(pyconv.wgrad(dy, x), gw, atol=1e-3)
