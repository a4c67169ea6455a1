"""CPU oracle of the learned-initial-guess network (test infrastructure only).

A plain PyTorch FP32 restatement, evaluated on the CPU with autograd, of the
periodic U-Net whose BF16 tensor-core kernels live in the library
(forward, data and weight gradients, pooling and upsampling adjoints).  The
reference has no such network -- its GMG solver only offers the hook
(utils/EBE_GMG.py:648-757 ``_prepare_init_levels``) -- so this oracle pins
the kernels against torch's own conv3d / avg_pool3d / nearest upsampling with
circular padding, not against reference outputs.

Layouts follow the library: activations channels-last (B, r^3, C) with voxel
id x*r*r + y*r + z; weights [taps][cin][cout] with tap = 9(dx+1) + 3(dy+1) +
(dz+1) for 3x3x3 kernels, meaning out[v] += in[v + (dx, dy, dz)] @ W[tap].
"""
from __future__ import annotations

import torch
import torch.nn.functional as F


def _to_ncdhw(x, r):
    B, N, C = x.shape
    return x.reshape(B, r, r, r, C).permute(0, 4, 1, 2, 3)


def _to_nvc(x):
    B, C = x.shape[:2]
    return x.permute(0, 2, 3, 4, 1).reshape(B, -1, C)


def _bf16(x, on):
    """BF16 storage rounding with a straight-through gradient."""
    if not on:
        return x
    return x + (x.to(torch.bfloat16).to(x.dtype) - x).detach()


def conv3d_periodic(x, W, b=None):
    """x (B, C, n, n, n), W [taps][cin][cout] -> (B, cout, n, n, n)."""
    taps, cin, cout = W.shape
    if taps == 1:
        w = W.reshape(cin, cout).t().reshape(cout, cin, 1, 1, 1)
        return F.conv3d(x, w, b)
    w = W.reshape(3, 3, 3, cin, cout).permute(4, 3, 0, 1, 2)
    return F.conv3d(F.pad(x, (1, 1, 1, 1, 1, 1), mode="circular"), w, b)


def unet_forward(params, x, r, widths, round_bf16=False, acts=None):
    """params: name -> (W [taps][cin][cout], b [cout]) FP32 tensors (names as
    the library: enc{l}a/b, mid_a/b, up{l}, dec{l}a/b, head).  x: (B, r^3, C)
    input features.  Returns (B, r^3, 21) FP32.  If `acts` is a dict, every
    stored activation is kept there (NCDHW) under the library's buffer name
    (enc{l}a/b, pool{l}, mid_a/b, up{l}, skip{l}, dec{l}a/b)."""
    L = len(widths)
    h = _to_ncdhw(x, r)
    keep = acts if acts is not None else {}

    def conv(name, inp, relu):
        W, b = params[name]
        y = conv3d_periodic(inp, W, b)
        return F.relu(y) if relu else y

    def store(name, t):
        t = _bf16(t, round_bf16)
        if acts is not None:
            t.retain_grad() if t.requires_grad else None
        keep[name] = t
        return t

    skips = []
    for lv in range(L - 1):
        a = store(f"enc{lv}a", conv(f"enc{lv}a", h, True))
        bb = store(f"enc{lv}b", conv(f"enc{lv}b", a, True))
        skips.append(bb)
        h = store(f"pool{lv + 1}", F.avg_pool3d(bb, 2))
    h = store("mid_a", conv("mid_a", h, True))
    h = store("mid_b", conv("mid_b", h, True))
    for lv in reversed(range(L - 1)):
        c = store(f"up{lv}", conv(f"up{lv}", h, False))
        d = store(f"skip{lv}", F.interpolate(c, scale_factor=2, mode="nearest") + skips[lv])
        a = store(f"dec{lv}a", conv(f"dec{lv}a", d, True))
        h = store(f"dec{lv}b", conv(f"dec{lv}b", a, True))
    out = conv("head", h, False)
    return _to_nvc(out)


def features(rho, C=8):
    """Network input (B, N, C): channel 0 = rho^(1/3), channel 1 = rho."""
    rho = torch.as_tensor(rho)
    B, N = rho.shape
    x = torch.zeros(B, N, C, dtype=torch.float32)
    x[..., 0] = rho.clamp_min(0).pow(1.0 / 3.0).float()
    x[..., 1] = rho.float()
    return x


def mse_and_grads(params, x, target, r, widths, round_bf16=False, acts=None):
    """Loss mean((out - target)^2), the output, and the gradients w.r.t.
    every parameter (and, with `acts`, w.r.t. every stored activation in
    acts[name].grad)."""
    leaves = {k: (W.clone().requires_grad_(True), b.clone().requires_grad_(True)) for k, (W, b) in params.items()}
    out = unet_forward(leaves, x, r, widths, round_bf16, acts)
    loss = (out - target).pow(2).mean()
    loss.backward()
    return float(loss.detach()), out.detach(), {k: (W.grad, b.grad) for k, (W, b) in leaves.items()}
