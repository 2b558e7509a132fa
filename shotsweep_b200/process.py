"""2_process's per-batch work on the GPU (openfwi/2_process.py:193-213).

For a batch of models' observed gathers: surface velocity from first-arrival
onsets (``background.estimate_surface_velocity_batch``), the three backgrounds,
the RTM images of every (model, background, shot) muted at the surface
velocity, and the float16 image cache (top two rows zeroed, divided by each
model's 99th percentile of |image|, clipped to +-4).  Everything stays on the
device until the cache is complete; the reference runs the picks and the cache
in NumPy per model on the host.

    out = process_batch(sim, gathers, trend)      # gathers [n, 5, 1000, 70]
    out['images']                                  # float16 [n, 3, 5, 70, 70]
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import background as BG


def image_cache(images, zero_rows=2, q=99.0, clip=4.0):
    """(float16 cache, per-model scale) of images [n, ...images..., nz, nx] (float32, CUDA) as 2_process.py:206-210.

    Raises ValueError, as 2_process does, if a model's images are not finite or its scale is not positive.
    """
    if not isinstance(images, torch.Tensor) or not images.is_cuda or images.dtype != torch.float32:
        raise ValueError('images must be a float32 CUDA tensor')
    img = images.contiguous()
    n, nz, nx = img.shape[0], img.shape[-2], img.shape[-1]
    n_images = int(np.prod(img.shape[1:-2])) if img.dim() > 3 else 1
    out = torch.empty(img.shape, dtype=torch.float16, device=img.device)
    scale = torch.empty(n, dtype=torch.float32, device=img.device)
    status = torch.empty(n, dtype=torch.int32, device=img.device)
    L = _lib.load()
    with torch.cuda.device(img.device):
        _lib.check(L.ss_image_cache(_lib.ptr(img), n, n_images, nz, nx, zero_rows, float(q), float(clip),
                                    _lib.ptr(out), _lib.ptr(scale), _lib.ptr(status),
                                    _lib.stream_handle(img.device)), 'ss_image_cache')
    st = status.cpu().numpy()
    bad = np.flatnonzero(st != _lib.OK)
    if len(bad):
        more = f' and {len(bad) - 10} more' if len(bad) > 10 else ''
        raise ValueError(f'models {bad[:10].tolist()}{more}: nonfinite or zero-energy images')
    return out, scale


def process_batch(sim, gathers, trend, t_mute=0.12):
    """The cache entries of one batch of models: images, surface velocity and its diagnostics."""
    eng = sim.engine
    dev = eng.device
    obs = gathers if isinstance(gathers, torch.Tensor) else torch.as_tensor(np.asarray(gathers, np.float32))
    obs = obs.to(device=dev, dtype=torch.float32).contiguous()
    n = obs.shape[0]
    est = BG.estimate_surface_velocity_batch(obs)
    v1 = np.array([e['velocity'] for e in est])
    nb = len(BG.RHOS)
    bgs = BG.backgrounds(v1, trend, device=dev).reshape(n * nb, eng.g.nz, eng.g.nx)
    vm = torch.tensor(np.repeat(v1, nb), dtype=torch.float32, device=dev)
    obs_rows = obs.repeat_interleave(nb, dim=0)
    img, _ = eng.images(bgs, sim._wavelet(), obs_rows, vm, t_mute)
    eng.status()
    cache, _ = image_cache(img.reshape(n, nb, eng.g.n_shots, eng.g.nz, eng.g.nx))
    return {'images': cache, 'surface_velocity': v1.astype(np.float32),
            'surface_confidence': np.array([e['confidence'] for e in est], np.float32),
            'surface_fit_rmse_ms': np.array([e['fit_rmse_ms'] for e in est], np.float32),
            'surface_possible_refraction': np.array([e['possible_refraction'] for e in est], bool)}
