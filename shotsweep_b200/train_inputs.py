"""The training-input transforms of openfwi/3_train.py on the GPU.

``stored_gathers``  sign(g) log1p(|g|) as float16, the form load_data keeps (3_train.py:157)
``batch_gathers``   a batch's float32 gathers, the stored form / scale (3_train.py:198)
``targets``         normalised velocities (v - 3000) / 1500 (3_train.py:158)
``vref``            the clipped normalised reference velocity v1 + trend (3_train.py:188-189)
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib


def _cuda_f32(t, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
        raise ValueError(f'{name} must be a float32 CUDA tensor')
    return t.contiguous()


def stored_gathers(g):
    g = _cuda_f32(g, 'gathers')
    out = torch.empty(g.shape, dtype=torch.float16, device=g.device)
    with torch.cuda.device(g.device):
        _lib.check(_lib.load().ss_signed_log1p_f16(_lib.ptr(g), g.numel(), _lib.ptr(out),
                                                   _lib.stream_handle(g.device)), 'ss_signed_log1p_f16')
    return out


def batch_gathers(stored, scale, out=None):
    if not math.isfinite(scale) or scale <= 0:
        raise ValueError('Gather normalization scale must be finite and positive')
    if not isinstance(stored, torch.Tensor) or not stored.is_cuda or stored.dtype != torch.float16:
        raise ValueError('stored gathers must be a float16 CUDA tensor')
    stored = stored.contiguous()
    out = torch.empty(stored.shape, dtype=torch.float32, device=stored.device) if out is None else out
    with torch.cuda.device(stored.device):
        _lib.check(_lib.load().ss_f16_scaled(_lib.ptr(stored), stored.numel(), float(scale), _lib.ptr(out),
                                             _lib.stream_handle(stored.device)), 'ss_f16_scaled')
    return out


def targets(vel):
    vel = _cuda_f32(vel, 'velocities')
    y = torch.empty_like(vel)
    with torch.cuda.device(vel.device):
        _lib.check(_lib.load().ss_velocity_targets(_lib.ptr(vel), vel.numel(), _lib.ptr(y), None, None, 0, 1, 1,
                                                   None, _lib.stream_handle(vel.device)), 'ss_velocity_targets')
    return y


def vref(v1, trend, nx=70):
    v1 = _cuda_f32(v1, 'surface velocities')
    tr = _cuda_f32(trend, 'trend')
    out = torch.empty(v1.numel(), tr.numel(), nx, dtype=torch.float32, device=v1.device)
    with torch.cuda.device(v1.device):
        _lib.check(_lib.load().ss_velocity_targets(None, 0, None, _lib.ptr(v1), _lib.ptr(tr), v1.numel(), tr.numel(),
                                                   nx, _lib.ptr(out), _lib.stream_handle(v1.device)),
                   'ss_velocity_targets')
    return out
