"""Differentiable forward modelling: gathers(v) as a torch.autograd.Function.

Forward: the B200 forward kernel, keeping only the wavefield pairs
(p[t-1], p[t]) every K steps (K = ceil(sqrt(nt)) by default, 32 for nt=1000).
Backward: the exact discrete adjoint of the same discretisation, rebuilt
segment by segment from those checkpoints (each segment recomputes K steps on
the GPU, keeps their Laplacians in an L2-sized history and runs the adjoint
over them), as in the reference's checkpointed Sim._gradient
(openfwi/physics/gpu.py:152-188) but with the adjoint source taken from the
incoming gradient, so any differentiable loss of the gathers works.

    v = torch.tensor(models, device='cuda', requires_grad=True)
    sim = simulate(v)                       # [B, 5, nt, nx]
    loss = 0.5 * ((sim - obs) ** 2).sum()
    loss.backward()                         # v.grad: d loss / d v, summed over shots

The gradient includes the velocity-dependent source strength and the
edge-padded absorbing layer, like the reference's.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import engine as E
from .constants import DT, DX, NT, NX, NZ, SRC_X

_ENGINES = {}


def default_engine(device=None, pad=40, R=1e-5):
    dev = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
    key = (str(dev), pad, R)
    if key not in _ENGINES:
        cols = [int(round(x / DX)) for x in SRC_X]
        _ENGINES[key] = E.Engine(E.geometry(NZ, NX, NT, pad, cols, 1, DX, DT, R), dev)
    return _ENGINES[key]


def default_interval(nt):
    return max(1, math.ceil(math.sqrt(nt)))


class Gathers(torch.autograd.Function):
    """gathers = F(v) for velocities v [B, nz, nx] (float32, CUDA)."""

    @staticmethod
    def forward(ctx, vel, eng, wavelet, interval):
        vel = vel.detach().contiguous()
        out, ck = eng.forward(vel, wavelet, ckpt_interval=interval)
        ctx.eng, ctx.interval = eng, interval
        ctx.save_for_backward(vel, wavelet, ck)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        vel, wavelet, ck = ctx.saved_tensors
        grad, _ = ctx.eng.adjoint_from_checkpoints(vel, wavelet, ck, ctx.interval, grad_out.contiguous().float())
        return grad.sum(1), None, None, None


def simulate(vel, eng=None, wavelet=None, interval=None):
    """Differentiable gathers [B, S, nt, nx] of velocities [B, nz, nx]."""
    eng = default_engine(vel.device) if eng is None else eng
    if wavelet is None:
        t = np.arange(eng.g.nt) * eng.g.dt
        a = (np.pi * 15.0 * (t - 1.2 / 15.0)) ** 2
        wavelet = E.scaled_wavelet((1 - 2 * a) * np.exp(-a), eng.device)
    interval = default_interval(eng.g.nt) if interval is None else int(interval)
    return Gathers.apply(vel, eng, wavelet, interval)


def misfit_gradient(vel, obs, eng=None, wavelet=None, interval=None):
    """(J, dJ/dv) of J = 0.5 * sum (F(v) - obs)^2, the unmuted misfit of Sim.gradient."""
    v = vel.detach().clone().requires_grad_(True)
    sim = simulate(v, eng, wavelet, interval)
    J = 0.5 * ((sim - obs) ** 2).sum()
    J.backward()
    return J.detach(), v.grad
