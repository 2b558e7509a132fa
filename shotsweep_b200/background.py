"""Surface velocity and backgrounds on the GPU (the reference's openfwi/physics/background.py).

``estimate_surface_velocity`` keeps the reference's call and return value
(background.py:19-83: a dict of seven diagnostics, or ValueError with the
reference's message); ``estimate_surface_velocity_batch`` runs the same
estimator for many models in one launch (one CTA per model: onset picks of
every trace in parallel, then the fits in float64) and returns the dicts, or
raises for the first model the reference would reject.  ``backgrounds`` builds
the slow / medium / fast laterally constant models (background.py:97-99) on
the device; ``depth_trend`` is the reference's training-set statistic
(background.py:91-94), a host reduction done once per dataset.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .constants import DT, DX, NT, NX, SRC_X

RHOS = (0.6, 1.0, 1.4)
KEYS = ('velocity', 'confidence', 'fit_rmse_ms', 'short_offset_curvature', 'shot_slope_spread',
        'far_offset_velocity', 'possible_refraction')
MESSAGES = {
    _lib.SURF_NO_ONSETS: 'surface velocity unavailable: no nonzero onset traces',
    _lib.SURF_FEW_NEAR: 'surface velocity unavailable: insufficient 10–60 m offsets',
    _lib.SURF_SLOPE: 'surface velocity unavailable: short-offset slope is outside 1400–4600 m/s',
    _lib.SURF_FEW_SHOTS: 'surface velocity unavailable: fewer than three usable shots',
}


def _device(device):
    dev = torch.device('cuda') if device is None else torch.device(device)
    _lib.require_cuda(dev)
    return torch.device('cuda', torch.cuda.current_device()) if dev.index is None else dev


def surface_estimates(gathers, frac=0.05, src_x=SRC_X, dx=DX, dt=DT, device=None):
    """Raw ss_surface_estimate records for gathers [n, n_shots, nt, nx] (array or tensor)."""
    if not 0 < frac < 1:
        raise ValueError('onset threshold frac must lie between zero and one')
    if isinstance(gathers, torch.Tensor) and gathers.is_cuda:
        dev = gathers.device
        g = gathers.to(torch.float32).contiguous()
    else:
        dev = _device(device)
        g = torch.as_tensor(np.asarray(gathers), dtype=torch.float32).to(dev).contiguous()
    if g.dim() != 4 or g.shape[1] != len(src_x):
        raise ValueError(f'observations must be finite with shape (N, {len(src_x)}, nt, nx)')
    n, ns, nt, nx = g.shape
    out = torch.empty(n * ctypes.sizeof(_lib.SurfaceEstimate), dtype=torch.uint8, device=dev)
    xs = (ctypes.c_double * ns)(*[float(x) for x in src_x])
    L = _lib.load()
    with torch.cuda.device(dev):
        _lib.check(L.ss_surface_velocity(_lib.ptr(g), n, ns, nt, nx, xs, dx, dt, frac, _lib.ptr(out),
                                         _lib.stream_handle(dev)), 'ss_surface_velocity')
    host = out.cpu().numpy()
    return (_lib.SurfaceEstimate * n).from_buffer_copy(host.tobytes())


def _as_dict(e, nt, nx, n_shots):
    if e.status == _lib.SURF_OK:
        return {'velocity': e.velocity, 'confidence': e.confidence, 'fit_rmse_ms': e.fit_rmse_ms,
                'short_offset_curvature': e.short_offset_curvature, 'shot_slope_spread': e.shot_slope_spread,
                'far_offset_velocity': e.far_offset_velocity, 'possible_refraction': bool(e.possible_refraction)}
    if e.status == _lib.SURF_NONFINITE:
        raise ValueError(f'observations must be finite with shape ({n_shots}, {nt}, {nx})')
    if e.status == _lib.SURF_UNRELIABLE:
        raise ValueError('surface velocity unreliable: curved or inconsistent short-offset arrivals '
                         f'(RMSE={e.fit_rmse_ms:.2f} ms, curvature={e.short_offset_curvature:.3f}, '
                         f'shot spread={e.shot_slope_spread:.3f})')
    raise ValueError(MESSAGES[e.status])


def estimate_surface_velocity_batch(gathers, frac=0.05, src_x=SRC_X, dx=DX, dt=DT, device=None):
    """Diagnostics of every model of gathers [n, n_shots, nt, nx]; ValueError 'model k: ...' for a rejected one."""
    est = surface_estimates(gathers, frac, src_x, dx, dt, device)
    nt, nx = gathers.shape[2], gathers.shape[3]
    out = []
    for k, e in enumerate(est):
        try:
            out.append(_as_dict(e, nt, nx, len(src_x)))
        except ValueError as error:
            raise ValueError(f'model {k}: {error}') from None
    return out


def estimate_surface_velocity(obs, frac=0.05):
    """background.py:19-83 for one model's gathers (5, 1000, 70)."""
    obs = np.asarray(obs)
    if obs.shape != (5, NT, NX):
        raise ValueError(f'observations must be finite with shape (5, {NT}, {NX})')
    if not 0 < frac < 1:
        raise ValueError('onset threshold frac must lie between zero and one')
    e = surface_estimates(obs[None], frac)[0]
    return _as_dict(e, NT, NX, 5)


def surface_velocity(obs, frac=0.05):
    """background.py:86-88."""
    return estimate_surface_velocity(obs, frac)['velocity']


def depth_trend(models):
    """background.py:91-94: mean over models of mean_x v(z) - mean_x v(0)."""
    m = np.asarray(models, np.float64)
    return (m.mean(2) - m[:, :1, :].mean(2)).mean(0)


def backgrounds(v_surface, trend, rhos=RHOS, nx=NX, device=None):
    """Backgrounds [n, len(rhos), nz, nx] float32 on the device for surface velocities [n] (or a scalar)."""
    dev = _device(device)
    v = torch.as_tensor(np.atleast_1d(np.asarray(v_surface, np.float64)), dtype=torch.float64).to(dev)
    tr = torch.as_tensor(np.asarray(trend, np.float64), dtype=torch.float64).to(dev)
    rh = torch.as_tensor(np.asarray(rhos, np.float64), dtype=torch.float64).to(dev)
    n, nz = v.numel(), tr.numel()
    out = torch.empty(n, len(rhos), nz, nx, dtype=torch.float32, device=dev)
    L = _lib.load()
    with torch.cuda.device(dev):
        _lib.check(L.ss_backgrounds(_lib.ptr(v), _lib.ptr(tr), _lib.ptr(rh), n, len(rhos), nz, nx, _lib.ptr(out),
                                    _lib.stream_handle(dev)), 'ss_backgrounds')
    return out
