"""Test oracle for the learned warm start's U-Net: the same network restated
with torch on the CPU in float64 (no counterpart in the reference, which has
no learned component).

Used only by tests/ to check the CUDA network's forward pass and gradients.
With ``emulate_bf16`` the oracle rounds to bfloat16 exactly where the CUDA
network stores BF16: the weights, the packed input and every stored activation
on the forward pass, and on the backward pass every layer's output gradient
after the ReLU mask (the operand the weight, bias and input gradients are
computed from, k_dz in the CUDA network), so that the comparison isolates the
FP32-versus-FP64 accumulation; without it the oracle is the exact float64
network.

Parameter layout (flat float32, as imp_unet_get_params): for every layer the
weights [cout][ky][kx][cin] then the bias [cout].
"""
from __future__ import annotations

import numpy as np

# cin, cout, kernel size, ReLU -- the layer table of the CUDA network
CFG = [(16, 32, 3, 1), (32, 32, 3, 1), (32, 64, 3, 1), (64, 64, 3, 1), (64, 128, 3, 1),
       (128, 128, 3, 1), (128, 256, 3, 1), (256, 256, 3, 1), (256, 128, 1, 0),
       (256, 128, 3, 1), (128, 128, 3, 1), (128, 64, 1, 0), (128, 64, 3, 1), (64, 64, 3, 1),
       (64, 32, 1, 0), (64, 32, 3, 1), (32, 32, 3, 1), (32, 16, 1, 0)]


def n_params() -> int:
    return sum(co * k * k * ci + co for ci, co, k, _ in CFG)


def unpack(params, torch):
    """flat parameters -> list of (weight [cout][cin][k][k], bias) float64 tensors"""
    p = torch.as_tensor(np.asarray(params, np.float64))
    out, off = [], 0
    for ci, co, k, _ in CFG:
        n = co * k * k * ci
        w = p[off:off + n].reshape(co, k, k, ci).permute(0, 3, 1, 2).contiguous()
        off += n
        b = p[off:off + co]
        off += co
        out.append((w, b))
    return out


def pack(grads_per_layer, torch) -> np.ndarray:
    """list of (dW [cout][cin][k][k], db) -> flat layout"""
    parts = []
    for (dw, db) in grads_per_layer:
        parts.append(dw.permute(0, 2, 3, 1).reshape(-1))
        parts.append(db.reshape(-1))
    return torch.cat(parts).numpy()


def forward(params, x, H: int, W: int, emulate_bf16: bool = True, torch=None,
            requires_grad: bool = False):
    """x [B][2][H*W] -> (output [B][2][H*W], leaf parameter tensors)."""
    if torch is None:
        import torch  # noqa: F811
    import torch.nn.functional as F
    layers = unpack(params, torch)

    def bf(t):
        return t.to(torch.bfloat16).to(torch.float64) if emulate_bf16 else t

    # The network computes with BF16 copies of its FP32 weights and returns the
    # gradient with respect to those copies in FP32: the rounded weights are
    # the leaves, so that autograd does not round their gradients back through
    # the dtype cast.
    leaves = []
    for w, b in layers:
        w = bf(w).detach()
        w.requires_grad_(requires_grad)
        b.requires_grad_(requires_grad)
        leaves.append((w, b))

    class GradBF16(torch.autograd.Function):
        """Identity whose backward rounds the incoming gradient to BF16."""

        @staticmethod
        def forward(ctx, t):
            return t.view_as(t)

        @staticmethod
        def backward(ctx, g):
            return g.to(torch.bfloat16).to(torch.float64)

    gbf = GradBF16.apply if emulate_bf16 else (lambda t: t)

    B = x.shape[0]
    x = torch.as_tensor(np.asarray(x, np.float64)).reshape(B, 2, H, W)
    h0 = torch.zeros(B, 16, H, W, dtype=torch.float64)
    h0[:, :2] = x
    h0 = bf(h0)

    def conv(i, h, last=False):
        w, b = leaves[i]
        ci, co, k, relu = CFG[i]
        y = gbf(F.conv2d(h, w, b, padding=k // 2))
        if relu:
            y = F.relu(y)
        return y if last else bf(y)

    pool = lambda h: F.max_pool2d(h, 2)
    up = lambda h: F.interpolate(h, scale_factor=2, mode="nearest")
    e1 = conv(0, h0)
    s1 = conv(1, e1)
    e2 = conv(2, pool(s1))
    s2 = conv(3, e2)
    e3 = conv(4, pool(s2))
    s3 = conv(5, e3)
    m1 = conv(6, pool(s3))
    m2 = conv(7, m1)
    d3 = torch.cat([s3, up(conv(8, m2))], 1)
    f3 = conv(10, conv(9, d3))
    d2 = torch.cat([s2, up(conv(11, f3))], 1)
    f2 = conv(13, conv(12, d2))
    d1 = torch.cat([s1, up(conv(14, f2))], 1)
    f1 = conv(16, conv(15, d1))
    out = conv(17, f1, last=True)[:, :2]
    return out.reshape(B, 2, H * W), leaves


def loss_and_grads(params, x, target, H: int, W: int, emulate_bf16: bool = True):
    """Mean squared error and its parameter gradients (flat layout)."""
    import torch
    out, leaves = forward(params, x, H, W, emulate_bf16, torch, requires_grad=True)
    t = torch.as_tensor(np.asarray(target, np.float64)).reshape(out.shape)
    loss = ((out - t) ** 2).mean()
    loss.backward()
    grads = pack([(w.grad, b.grad) for w, b in leaves], torch)
    return float(loss.detach()), grads


def layer_slices():
    """(start, stop) of each layer's weights in the flat layout"""
    out, off = [], 0
    for ci, co, k, _ in CFG:
        n = co * k * k * ci
        out.append((off, off + n))
        off += n + co
    return out
