"""TEST INFRASTRUCTURE ONLY - float32 PyTorch-CPU restatement of the learned proposal network.

The network of shotsweep_b200/proposal.py (layer table LAYERS, flat parameter
layout) as ordinary PyTorch operations on the CPU, differentiated by autograd.
It rounds to BF16 exactly where the CUDA path stores BF16: the weights' BF16
copy, every activation after its leaky ReLU, every pre-activation gradient and
every column gradient (the input-gradient GEMM's output, before col2im sums it
onto the input); everything else is float32.  Used only by tests/ to check the GPU forward pass
and every parameter gradient; nothing in the product imports it.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

from shotsweep_b200.proposal import HEAD_C, HEAD_OFF, LAYERS, OUT, SLOPE, param_layout, plan_shapes


class RoundBF16(torch.autograd.Function):
    """Forward: round to BF16; backward: identity (a stored activation or weight copy)."""
    @staticmethod
    def forward(ctx, x):
        return x.to(torch.bfloat16).float()

    @staticmethod
    def backward(ctx, g):
        return g


class GradRoundBF16(torch.autograd.Function):
    """Forward: identity; backward: round the gradient to BF16 (a stored pre-activation gradient)."""
    @staticmethod
    def forward(ctx, x):
        return x

    @staticmethod
    def backward(ctx, g):
        return g.to(torch.bfloat16).float()


def loss_and_grads(params, x0, target):
    """(pred [B,70,70], loss, flat parameter gradient) for inputs x0 [B,1000,70,5] (BF16 values) and targets."""
    lay, total = param_layout()
    P = torch.tensor(np.asarray(params, np.float32), requires_grad=True)
    x = torch.as_tensor(x0, dtype=torch.float32)
    for L, shape in zip(LAYERS, plan_shapes()):
        K, Kc, N = shape[4:]
        o, n = lay[L.name + '.w']
        W = RoundBF16.apply(P[o:o + n].view(N, Kc)[:, :K])
        ob, nb = lay[L.name + '.b']
        pre = GradRoundBF16.apply(_pre(L, shape, W, P[ob:ob + nb], x))
        x = RoundBF16.apply(F.leaky_relu(pre, SLOPE))
    o, n = lay['head.w']
    wh = P[o:o + n].view(3, 3, HEAD_C).permute(2, 0, 1)[None]
    bh = P[lay['head.b'][0]:lay['head.b'][0] + 1]
    xc = x[:, HEAD_OFF:HEAD_OFF + OUT, HEAD_OFF:HEAD_OFF + OUT, :].permute(0, 3, 1, 2)
    pred = torch.tanh(F.conv2d(xc, wh, bh, padding=1)[:, 0])
    loss = (pred - torch.as_tensor(target, dtype=torch.float32)).abs().mean()
    loss.backward()
    return pred.detach().numpy(), float(loss.detach()), P.grad.numpy()


def adamw_step(p, g, m, v, step, lr, wd=1e-4, b1=0.9, b2=0.999, eps=1e-8):
    """One AdamW step (torch.optim.AdamW's update), float32."""
    p = p * (1 - lr * wd)
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mhat = m / (1 - b1 ** step)
    vhat = v / (1 - b2 ** step)
    return (p - lr * mhat / (np.sqrt(vhat) + eps)).astype(np.float32), m.astype(np.float32), v.astype(np.float32)


def _pre(L, shape, W, b, x):
    """Pre-activation [B, ho, wo, N] as columns x weights^T + bias; the columns' gradient is rounded to BF16."""
    hi, wi, ho, wo, K, Kc, N = shape
    B = x.shape[0]
    if L.kind == 'conv':
        xin = x.permute(0, 3, 1, 2)
        if L.up > 1:
            xin = F.interpolate(xin, scale_factor=L.up, mode='nearest')
        u = F.unfold(xin, (L.kh, L.kw), padding=(L.ph, L.pw), stride=(L.sh, L.sw))     # [B, (c, kh, kw), pixels]
        cols = u.view(B, L.cin, L.kh * L.kw, -1).permute(0, 3, 2, 1).reshape(B, -1, K)  # [B, pixels, (kh, kw, c)]
        return F.linear(GradRoundBF16.apply(cols), W, b).view(B, ho, wo, N)
    cols = GradRoundBF16.apply(x.reshape(B, -1))
    if L.kind == 'window':
        return F.linear(cols, W, b).view(B, 1, 1, N)
    return F.linear(cols, W, b).view(B, L.out_hw, L.out_hw, L.cout)


def layer_weights(params, i):
    lay, _ = param_layout()
    L, (hi, wi, ho, wo, K, Kc, N) = LAYERS[i], plan_shapes()[i]
    o, n = lay[L.name + '.w']
    ob, nb = lay[L.name + '.b']
    P = torch.as_tensor(np.asarray(params, np.float32))
    return P[o:o + n].view(N, Kc)[:, :K].to(torch.bfloat16).float(), P[ob:ob + nb].clone()


def layer_forward(params, i, x):
    """Layer i's BF16 output from its input x [B, H, W, C] (BF16 values)."""
    W, b = layer_weights(params, i)
    return F.leaky_relu(_pre(LAYERS[i], plan_shapes()[i], W, b, torch.as_tensor(x)), SLOPE).to(torch.bfloat16).float()


def layer_backward(params, i, x, dpre):
    """(dW [N][K], db [N], dpre of the layer below or None) from layer i's input x and pre-activation gradient dpre."""
    W, b = layer_weights(params, i)
    W.requires_grad_(True)
    b.requires_grad_(True)
    xt = torch.as_tensor(x).clone().requires_grad_(i > 0)
    pre = _pre(LAYERS[i], plan_shapes()[i], W, b, xt)
    pre.backward(torch.as_tensor(dpre).view(pre.shape))
    below = None
    if i > 0:
        below = torch.where(xt.detach() > 0, xt.grad, SLOPE * xt.grad).to(torch.bfloat16).float()
    return W.grad.numpy(), b.grad.numpy(), None if below is None else below.numpy()


def head_forward(params, x):
    lay, _ = param_layout()
    P = torch.as_tensor(np.asarray(params, np.float32))
    o, n = lay['head.w']
    wh = P[o:o + n].view(3, 3, HEAD_C).permute(2, 0, 1)[None]
    bh = P[lay['head.b'][0]:lay['head.b'][0] + 1]
    xc = torch.as_tensor(x)[:, HEAD_OFF:HEAD_OFF + OUT, HEAD_OFF:HEAD_OFF + OUT, :].permute(0, 3, 1, 2)
    return torch.tanh(F.conv2d(xc, wh, bh, padding=1)[:, 0]).numpy()


def head_backward(params, x, dpre_head):
    """(dw [9*C], db, dpre of d5 [B,H,W,C]) from the d5 output x and the head's pre-tanh gradient."""
    lay, _ = param_layout()
    P = torch.as_tensor(np.asarray(params, np.float32))
    o, n = lay['head.w']
    wh = P[o:o + n].view(3, 3, HEAD_C).clone().requires_grad_(True)
    bh = P[lay['head.b'][0]:lay['head.b'][0] + 1].clone().requires_grad_(True)
    xt = torch.as_tensor(x).clone().requires_grad_(True)
    xc = xt[:, HEAD_OFF:HEAD_OFF + OUT, HEAD_OFF:HEAD_OFF + OUT, :].permute(0, 3, 1, 2)
    pre = F.conv2d(xc, wh.permute(2, 0, 1)[None], bh, padding=1)[:, 0]
    pre.backward(torch.as_tensor(dpre_head))
    below = torch.where(xt.detach() > 0, xt.grad, SLOPE * xt.grad).to(torch.bfloat16).float()
    return wh.grad.reshape(-1).numpy(), float(bh.grad[0]), below.numpy()


def l1_tanh_grad(pred, target):
    """d mean|pred - target| / d(pre-tanh), with pred = tanh(pre)."""
    d = np.asarray(pred, np.float32) - np.asarray(target, np.float32)
    return (np.sign(d) / d.size * (1 - np.asarray(pred, np.float32) ** 2)).astype(np.float32)
