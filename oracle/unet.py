"""TEST INFRASTRUCTURE ONLY: an f64 CPU restatement of the learned preconditioner's network (no reference counterpart:
the reference has no learned part), used to check the CUDA forward pass and its hand-written gradients.

The network maps the Jacobi-scaled, rms-normalised residual and three operator features to the scaled error:
    input (4 ch): r̂/s, d̂x = dx / sqrt(d_i d_{i+1}), d̂y = dy / sqrt(d_i d_{i+w}), m = c / d   (d the diagonal)
    level 0: conv 4→8, conv 8→8           (e0)    pool
    level 1: conv 8→16, conv 16→16        (e1)    pool
    level 2: conv 16→32, conv 32→32       (e2)    pool
    level 3: conv 32→64, conv 64→64       (e3)
    up to 2: conv 64→32 on up(e3) (u2); conv 32→32 on u2 + e2 (d2)
    up to 1: conv 32→16 on up(d2) (u1); conv 16→16 on u1 + e1 (d1)
    up to 0: conv 16→8 on up(d1) (u0);  conv 8→8 on u0 + e0 (d0)
    head:    conv 8→1 on d0 (no ReLU)
Every other conv is 3x3, zero-padded, followed by ReLU; pool averages each 2x2 block (over the cells that exist);
up repeats each cell over its 2x2 block. Parameters, in order: per layer W[cout][3][3][cin] then b[cout].
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

# (cin, cout, input mode, relu): input mode "in" the features, "prev" the previous output, "pool" it pooled, "up" it
# upsampled, "skip" it plus an encoder output
LAYERS = [
    (4, 8, "in", True), (8, 8, "prev", True),
    (8, 16, "pool", True), (16, 16, "prev", True),
    (16, 32, "pool", True), (32, 32, "prev", True),
    (32, 64, "pool", True), (64, 64, "prev", True),
    (64, 32, "up", True), (32, 32, "skip", True),
    (32, 16, "up", True), (16, 16, "skip", True),
    (16, 8, "up", True), (8, 8, "skip", True),
    (8, 1, "prev", False),
]
SKIP_OF = {9: 5, 11: 3, 13: 1}  # layer -> the encoder layer whose output it adds


def param_count() -> int:
    return sum(co * 9 * ci + co for ci, co, _, _ in LAYERS)


def unpack(theta: torch.Tensor):
    out, k = [], 0
    for ci, co, _, _ in LAYERS:
        w = theta[k:k + co * 9 * ci].reshape(co, 3, 3, ci).permute(0, 3, 1, 2)  # -> (co, ci, ky, kx)
        k += co * 9 * ci
        b = theta[k:k + co]
        k += co
        out.append((w, b))
    return out


def pool(x):
    """(N, C, H, W) -> (N, C, ceil(H/2), ceil(W/2)), the mean over the cells of each block that exist."""
    n, c, h, w = x.shape
    ph, pw = (h + 1) // 2 * 2, (w + 1) // 2 * 2
    xs = F.pad(x, (0, pw - w, 0, ph - h))
    ones = F.pad(torch.ones((1, 1, h, w), dtype=x.dtype), (0, pw - w, 0, ph - h))
    return F.avg_pool2d(xs, 2) / F.avg_pool2d(ones, 2)


def up(x, h, w):
    return x.repeat_interleave(2, dim=2).repeat_interleave(2, dim=3)[:, :, :h, :w]


def _bf16(x: torch.Tensor) -> torch.Tensor:
    """Round to FP32, then to BF16 (round to nearest even), back to f64: what the tensor-core kernels feed the MMA."""
    return x.to(torch.float32).to(torch.bfloat16).to(torch.float64)


class _ConvBF16(torch.autograd.Function):
    """A 3x3 convolution as the CUDA kernels compute it: forward and data gradient on BF16-rounded operands (the
    tensor-core implicit GEMMs), the weight and bias gradients from the unrounded values (the CUDA-core kernels)."""

    @staticmethod
    def forward(ctx, x, w, b):
        ctx.save_for_backward(x, w)
        return F.conv2d(_bf16(x), _bf16(w), b, padding=1)

    @staticmethod
    def backward(ctx, g):
        x, w = ctx.saved_tensors
        gx = torch.nn.grad.conv2d_input(x.shape, _bf16(w), _bf16(g), padding=1)
        gw = torch.nn.grad.conv2d_weight(x, w.shape, g, padding=1)
        return gx, gw, g.sum((0, 2, 3))


def forward(theta: torch.Tensor, feats: torch.Tensor, bf16: bool = False) -> torch.Tensor:
    """feats (N, 4, H, W) -> (N, 1, H, W); `bf16` rounds every convolution's operands as the GPU kernels do."""
    params = unpack(theta)
    outs = []
    x = feats
    for li, ((ci, co, mode, relu), (w, b)) in enumerate(zip(LAYERS, params)):
        if mode == "pool":
            x = pool(outs[-1])
        elif mode == "up":
            lvl_h, lvl_w = outs[SKIP_OF[li + 1]].shape[2:]
            x = up(outs[-1], lvl_h, lvl_w)
        elif mode == "skip":
            x = outs[-1] + outs[SKIP_OF[li]]
        elif mode == "prev":
            x = outs[-1]
        y = _ConvBF16.apply(x, w, b) if bf16 else F.conv2d(x, w, b, padding=1)
        if relu:
            y = F.relu(y)
        outs.append(y)
    return outs[-1]


def init_params(seed: int) -> np.ndarray:
    """He-style initialisation with a random head and zero biases (tests pass these weights to the GPU)."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co, _, relu in LAYERS:
        std = np.sqrt(2.0 / (9 * ci)) if relu else np.sqrt(1.0 / (9 * ci))
        parts.append(rng.normal(0.0, std, co * 9 * ci))
        parts.append(np.zeros(co))
    return np.concatenate(parts)


def scaled_operator(feats: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """Â v over each crop: unit diagonal, -d̂x (feature 1) to the +x neighbour and -d̂y (feature 2) to the +y one,
    symmetric, the couplings that leave the crop dropped. v (N, H, W)."""
    dx = feats[:, 1, :, :-1]
    dy = feats[:, 2, :-1, :]
    out = v.clone()
    out[:, :, :-1] -= dx * v[:, :, 1:]
    out[:, :, 1:] -= dx * v[:, :, :-1]
    out[:, :-1, :] -= dy * v[:, 1:, :]
    out[:, 1:, :] -= dy * v[:, :-1, :]
    return out


def loss_and_grad(theta: np.ndarray, feats: np.ndarray, target: np.ndarray, bf16: bool = False):
    """The loss (1/B) Σ_b δ_bᵀÂδ_b / (E_b + ε), δ = target − output (N, H, W), E_b = t_bᵀÂt_b, ε = 10⁻³ mean E_b, and
    its gradient, in f64 (with `bf16`, the convolutions' operands rounded as the GPU kernels round them)."""
    t = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    f = torch.tensor(feats, dtype=torch.float64)
    y = forward(t, f, bf16)[:, 0]
    tg = torch.tensor(target, dtype=torch.float64)
    energy = (tg * scaled_operator(f, tg)).sum((1, 2))
    eps = 1e-3 * energy.mean()
    d = tg - y
    loss = ((d * scaled_operator(f, d)).sum((1, 2)) / (energy + eps)).mean()
    loss.backward()
    return float(loss.item()), t.grad.numpy().copy(), y.detach().numpy()
