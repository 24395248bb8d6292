"""CPU oracle of the warm-start U-Net: the same network in torch CPU autograd (FP32 or FP64).

Test infrastructure only -- the product runs the network on its own CUDA kernels
(solver-cfd_b200/unet).  The warm start has no counterpart in the reference, so this oracle
restates the network itself: 3x3 "same" convolutions (cross-correlation, zero padding), 2x2
average pooling, nearest 2x upsampling, skip concatenation [upsampled, skip], ReLU, a head
without activation and the masked mean-square error sum(w (y - t)^2) * inv_norm.  It reads the
product's flat parameter layout (per layer W^T [kp][cout] with row (ky*3+kx)*cin + c, then the
bias), so parameters and gradients compare entry by entry.

`bf16_acts=True` rounds the input, the weights and every stored activation to BF16 in the
forward pass, as the product does (straight-through: the gradient itself is not rounded).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as Fn


def _round_bf16(x):
    return x + (x.to(torch.bfloat16).to(x.dtype) - x).detach()


def _conv_weight(flat, L, dtype):
    wt = flat[L.off_w: L.off_w + L.kp * L.cout].view(L.kp, L.cout)[: 9 * L.cin]
    w = wt.reshape(3, 3, L.cin, L.cout).permute(3, 2, 0, 1)
    b = flat[L.off_b: L.off_b + L.cout]
    return w.to(dtype), b.to(dtype)


def forward_loss(convs, levels, params: np.ndarray, X: np.ndarray, T: np.ndarray, Wt: np.ndarray,
                 inv_norm: float, dtype=torch.float32, bf16_acts=True):
    """X: [B, H, W, cin] (NHWC), T/Wt: [B, H, W, 8].  Returns (loss, y [B,H,W,8], grads flat)."""
    by = {L.name: L for L in convs}
    flat = torch.tensor(params, dtype=torch.float32)
    if bf16_acts:
        flat_used = flat.to(torch.bfloat16).to(torch.float32)
        # biases enter the product's epilogue in FP32 (not rounded)
        for L in convs:
            flat_used[L.off_b: L.off_b + L.cout] = flat[L.off_b: L.off_b + L.cout]
    else:
        flat_used = flat.clone()
    flat_used = flat_used.to(dtype).requires_grad_(True)
    rnd = _round_bf16 if bf16_acts else (lambda t: t)
    x = torch.tensor(X, dtype=dtype).permute(0, 3, 1, 2)
    x = rnd(x)

    def conv(name, t):
        L = by[name]
        w, b = _conv_weight(flat_used, L, dtype)
        y = Fn.conv2d(t, w, b, padding=1)
        return rnd(torch.relu(y)) if L.relu else y

    skips = []
    t = x
    for l in range(levels):
        t = conv(f"enc{l}b", conv(f"enc{l}a", t))
        if l + 1 < levels:
            skips.append(t)
            t = rnd(Fn.avg_pool2d(t, 2))
    for l in range(levels - 2, -1, -1):
        up = Fn.interpolate(t, scale_factor=2, mode="nearest")
        t = torch.cat([up, skips[l]], dim=1)
        t = conv(f"dec{l}b", conv(f"dec{l}a", t))
    y = conv("head", t).permute(0, 2, 3, 1)
    tt = torch.tensor(T, dtype=dtype)
    ww = torch.tensor(Wt, dtype=dtype)
    loss = (ww * (y - tt) ** 2).sum() * inv_norm
    loss.backward()
    g = flat_used.grad.detach().to(torch.float64).numpy()
    return float(loss.detach()), y.detach().numpy(), g
