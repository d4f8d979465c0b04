"""FP64 oracle of the learned preconditioner's network -- test infrastructure only.

A torch-CPU float64 restatement (with autograd for the gradients) of the 3D
U-Net in rtk_b200/csrc/unet.cu.  It has no counterpart in RTK: RTK's
conjugate gradient is unpreconditioned
(include/rtkConjugateGradientImageFilter.hxx:108-258), so this oracle is
pinned by construction only -- it is the textbook network written with
torch.nn.functional (conv3d, avg_pool3d, nearest interpolation, concatenation),
against which the hand-written kernels are compared.

With ``bf16=True`` it rounds to bfloat16 exactly where the GPU stores BF16:
the weights of the ten tensor-core layers and every stored activation (the
first and last layers keep FP32 weights, the output is FP32); arithmetic stays
float64.  Parameter layout: per 3x3x3 layer W[tap][c_in][c_out] with
tap = (kz*3+ky)*3+kx, then the 16 output weights.
"""
from __future__ import annotations

import numpy as np

LAYERS = [(1, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16)]


def split(flat):
    out, o = [], 0
    for ci, co in LAYERS:
        k = 27 * ci * co
        out.append(np.asarray(flat[o:o + k], dtype=np.float64).reshape(27, ci, co))
        o += k
    out.append(np.asarray(flat[o:o + 16], dtype=np.float64))
    return out


def to_torch_weights(layers, requires_grad=False):
    """[(27, ci, co)] + [(16,)] -> list of float64 tensors: conv weights
    (co, ci, kz, ky, kx) and the output vector."""
    import torch

    ws = []
    for w in layers[:10]:
        ci, co = w.shape[1], w.shape[2]
        t = torch.tensor(np.ascontiguousarray(w.reshape(3, 3, 3, ci, co).transpose(4, 3, 0, 1, 2)),
                         dtype=torch.float64, requires_grad=requires_grad)
        ws.append(t)
    ws.append(torch.tensor(layers[10], dtype=torch.float64, requires_grad=requires_grad))
    return ws


def grads_to_layout(ws):
    """Gradients of to_torch_weights tensors -> flat vector in the C layout."""
    parts = []
    for t in ws[:10]:
        g = t.grad.detach().numpy()  # (co, ci, kz, ky, kx)
        co, ci = g.shape[0], g.shape[1]
        parts.append(g.transpose(2, 3, 4, 1, 0).reshape(27 * ci * co))
    parts.append(ws[10].grad.detach().numpy().reshape(16))
    return np.concatenate(parts)


def forward(x, ws, bf16=True, normalize=False):
    """x: float64 tensor (batch, z, y, x); ws from to_torch_weights.
    Returns the float64 output (batch, z, y, x)."""
    import torch
    import torch.nn.functional as F

    def r(t):
        return t.to(torch.bfloat16).to(torch.float64) if bf16 else t

    def conv(t, w, relu=True):
        y = F.conv3d(t, w, padding=1)
        return r(F.relu(y) if relu else y)

    def up(t):
        return F.interpolate(t, scale_factor=2, mode="nearest")

    x5 = x[:, None]
    s = x.pow(2).mean().sqrt() if normalize else None
    if normalize:
        x5 = x5 / s
    e1a = r(F.relu(F.conv3d(x5, ws[0], padding=1)))
    e1 = conv(e1a, r(ws[1]))
    p1 = r(F.avg_pool3d(e1, 2))
    e2a = conv(p1, r(ws[2]))
    e2 = conv(e2a, r(ws[3]))
    p2 = r(F.avg_pool3d(e2, 2))
    b1 = conv(p2, r(ws[4]))
    b2 = conv(b1, r(ws[5]))
    d2a = conv(torch.cat([up(b2), e2], 1), r(ws[6]))
    d2 = conv(d2a, r(ws[7]))
    d1a = conv(torch.cat([up(d2), e1], 1), r(ws[8]))
    d1 = conv(d1a, r(ws[9]))
    out = torch.einsum("bczyx,c->bzyx", d1, ws[10])
    return out * s if normalize else out


def loss_and_gradients(x, target, flat_params, bf16=True, margin=0):
    """Mean squared error of forward(x) against target over the voxels at
    least `margin` inside every face, and its gradients (flat, C layout), in
    float64 with autograd."""
    import torch

    ws = to_torch_weights(split(flat_params), requires_grad=True)
    out = forward(torch.as_tensor(x, dtype=torch.float64), ws, bf16=bf16)
    d = out - torch.as_tensor(target, dtype=torch.float64)
    if margin:
        m = margin
        d = d[:, m:d.shape[1] - m, m:d.shape[2] - m, m:d.shape[3] - m]
    loss = d.pow(2).mean()
    loss.backward()
    return float(loss.detach()), grads_to_layout(ws), out.detach().numpy()
