"""TEST INFRASTRUCTURE ONLY - the CPU oracle of the steps around the RTM images.

Plain NumPy restatements, used only by tests/ as the checker of the CUDA
kernels in shotsweep_b200/csrc/process.cu; nothing in the product imports it.

* ``estimate_surface_velocity``  openfwi/physics/background.py:19-83, for any
  acquisition (the reference fixes 5 shots, 1000 steps, 70 receivers)
* ``image_cache``                openfwi/2_process.py:206-210
* ``signed_log1p``, ``scaled``, ``targets``, ``vref``  openfwi/3_train.py:157-158,188-189,198

Pinned by tests/test_oracle.py against the reference's own outputs in
tests/golden/process_small.npz (tests/golden/make_golden_process.py).
"""
from __future__ import annotations

import numpy as np

DX, DT = 10.0, 1e-3
SRC_X = np.array([0, 17, 34, 52, 69]) * DX          # constants.py:5


def _line(offsets, times):
    """background.py:14-17."""
    slope, intercept = np.polyfit(offsets, times, 1)
    residual = times - (intercept + slope * offsets)
    return slope, float(np.sqrt(np.mean(residual ** 2)))


def estimate_surface_velocity(obs, frac=0.05, src_x=SRC_X, dx=DX, dt=DT):
    """background.py:20-83 with the acquisition as arguments; raises the reference's ValueErrors."""
    obs = np.asarray(obs)
    n_shots, nt, nx = obs.shape
    if len(src_x) != n_shots or not np.isfinite(obs).all():
        raise ValueError(f'observations must be finite with shape ({len(src_x)}, {nt}, {nx})')
    if not 0 < frac < 1:
        raise ValueError('onset threshold frac must lie between zero and one')
    offsets, arrivals, shots = [], [], []
    for s, gather in enumerate(obs):                                        # background.py:38-46
        amplitude = np.abs(gather)
        peaks = amplitude.max(axis=0)
        for r in range(nx):
            h = abs(r * dx - src_x[s])
            if 10 <= h <= 250 and peaks[r] > 0:
                offsets.append(h)
                arrivals.append(np.argmax(amplitude[:, r] > frac * peaks[r]) * dt)
                shots.append(s)
    offsets, arrivals, shots = map(np.asarray, (offsets, arrivals, shots))
    if len(offsets) == 0:
        raise ValueError('surface velocity unavailable: no nonzero onset traces')
    distances = np.unique(offsets)                                          # background.py:50-52
    times = np.array([np.median(arrivals[offsets == h]) for h in distances])
    near = (distances >= 10) & (distances <= 60)
    if near.sum() != 6:
        raise ValueError('surface velocity unavailable: insufficient 10–60 m offsets')
    slope, rmse = _line(distances[near], times[near])
    if slope <= 0 or not 1400 <= 1 / slope <= 4600:
        raise ValueError('surface velocity unavailable: short-offset slope is outside 1400–4600 m/s')
    first = (distances >= 10) & (distances <= 40)                           # background.py:58-62
    last = (distances >= 30) & (distances <= 60)
    early_slope, _ = _line(distances[first], times[first])
    late_slope, _ = _line(distances[last], times[last])
    curvature = abs(early_slope - late_slope) / slope
    shot_slopes = []
    for s in range(n_shots):                                                # background.py:63-67
        keep = (shots == s) & (offsets >= 10) & (offsets <= 60)
        if len(np.unique(offsets[keep])) >= 4:
            shot_slopes.append(_line(offsets[keep], arrivals[keep])[0])
    if len(shot_slopes) < 3:
        raise ValueError('surface velocity unavailable: fewer than three usable shots')
    spread = float(np.std(shot_slopes) / slope)
    if rmse > 0.002 or curvature > 0.15 or spread > 0.15:                   # background.py:71-73
        raise ValueError('surface velocity unreliable: curved or inconsistent short-offset arrivals '
                         f'(RMSE={rmse * 1000:.2f} ms, curvature={curvature:.3f}, shot spread={spread:.3f})')
    far = (distances >= 120) & (distances <= 250)                           # background.py:74-78
    far_slope = _line(distances[far], times[far])[0] if far.sum() >= 4 else slope
    far_velocity = 1 / far_slope if far_slope > 0 else float('nan')
    refraction = max(0.0, 1 - far_slope / slope)
    confidence = 1 / (1 + rmse / dt + curvature / 0.15 + spread / 0.15 + refraction)
    return {
        'velocity': float(np.clip(1 / slope, 1500.0, 4500.0)),
        'confidence': float(confidence),
        'fit_rmse_ms': rmse * 1000,
        'short_offset_curvature': float(curvature),
        'shot_slope_spread': spread,
        'far_offset_velocity': float(far_velocity),
        'possible_refraction': bool(refraction > 0.15),
    }


def image_cache(img, zero_rows=2, q=99, clip=4.0):
    """2_process.py:206-210: img [n, nb, S, nz, nx] float32 -> (float16 cache, per-model scale)."""
    img = np.array(img, dtype=np.float32, copy=True)
    n = img.shape[0]
    img[..., :zero_rows, :] = 0
    scale = np.percentile(np.abs(img).reshape(n, -1), q, axis=1)[:, None, None, None, None]
    if not np.isfinite(img).all() or np.any(scale <= 0):
        raise ValueError('nonfinite or zero-energy images')
    return np.clip(img / scale, -clip, clip).astype(np.float16), scale.reshape(n)


def signed_log1p(g):
    """3_train.py:157: the stored float16 form of the gathers."""
    g = np.asarray(g, np.float32)
    return (np.sign(g) * np.log1p(np.abs(g))).astype(np.float16)


def scaled(stored, scale):
    """3_train.py:198: a batch's float32 gathers from the stored float16 form."""
    return stored.astype(np.float32) / scale


def targets(y):
    """3_train.py:158."""
    return (np.asarray(y, np.float32) - 3000) / 1500


def vref(v1, trend):
    """3_train.py:188-189."""
    v1 = np.asarray(v1, np.float32)
    vr = np.broadcast_to(v1[:, None, None] + np.asarray(trend, np.float32)[None, :, None], (len(v1), len(trend), len(trend)))
    return np.clip((vr - 3000) / 1500, -1, 1).astype(np.float32)
