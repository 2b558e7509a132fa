"""Seeded synthetic velocity models shaped like OpenFWI's (70x70 cells of 10 m, 1500-4500 m/s).

No OpenFWI data is available offline; these generators stand in for it with the
same shapes, spacing and value range.  Families:

* ``layered``  - 3-5 flat layers, velocity increasing with depth;
* ``curved``   - the same with sinusoidally curved interfaces
  (amplitude 0-4 cells, wavelength 35-140 cells);
* ``faulted``  - layered models cut by 1-3 planar faults with 5-20-cell throw;
* ``textured`` - curved layers plus a Gaussian random field (sigma 150 m/s,
  correlation length 3-10 cells, FFT-filtered white noise).

Every model is a pure function of its seed, so fixtures and benchmarks are
reproducible.
"""
from __future__ import annotations

import numpy as np

VMIN, VMAX = 1500.0, 4500.0
FAMILIES = ('layered', 'curved', 'faulted', 'textured')


def _interfaces(rng, nz, nx, curved):
    n_layers = int(rng.integers(3, 6))
    depths = np.sort(rng.uniform(5, nz - 5, n_layers - 1))
    vels = np.sort(rng.uniform(VMIN, VMAX, n_layers))
    x = np.arange(nx)
    surfaces = []
    for d in depths:
        if curved:
            amp = rng.uniform(0, 4)
            lam = rng.uniform(35, 140)
            phase = rng.uniform(0, 2 * np.pi)
            surfaces.append(d + amp * np.sin(2 * np.pi * x / lam + phase))
        else:
            surfaces.append(np.full(nx, d))
    return surfaces, vels


def _paint(surfaces, vels, nz, nx):
    z = np.arange(nz)[:, None] + 0.5
    v = np.full((nz, nx), vels[0])
    for s, vel in zip(surfaces, vels[1:]):
        v = np.where(z >= s[None, :], vel, v)
    return v


def layered(rng, nz=70, nx=70, curved=False):
    surfaces, vels = _interfaces(rng, nz, nx, curved)
    return _paint(surfaces, vels, nz, nx)


def faulted(rng, nz=70, nx=70):
    surfaces, vels = _interfaces(rng, nz, nx, curved=bool(rng.integers(0, 2)))
    zz, xx = np.mgrid[0:nz, 0:nx].astype(np.float64)
    v = _paint(surfaces, vels, nz, nx)
    for _ in range(int(rng.integers(1, 4))):
        x0 = rng.uniform(0.2 * nx, 0.8 * nx)
        dip = rng.uniform(-1.5, 1.5)           # dx per dz of the fault plane
        throw = rng.uniform(5, 20) * rng.choice((-1, 1))
        hanging = xx > x0 + dip * zz
        shifted = _paint([s + throw for s in surfaces], vels, nz, nx)
        v = np.where(hanging, shifted, v)
    return v


def gaussian_field(rng, nz, nx, sigma, corr):
    noise = rng.standard_normal((nz, nx))
    kz = np.fft.fftfreq(nz)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    filt = np.exp(-2 * (np.pi * corr) ** 2 * (kz ** 2 + kx ** 2))
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    return field * (sigma / max(field.std(), 1e-12))


def textured(rng, nz=70, nx=70):
    v = layered(rng, nz, nx, curved=True)
    return v + gaussian_field(rng, nz, nx, 150.0, rng.uniform(3, 10))


def model(family, seed, nz=70, nx=70):
    """One float32 (nz, nx) model of ``family`` from ``seed``."""
    rng = np.random.default_rng(seed)
    if family == 'layered':
        v = layered(rng, nz, nx)
    elif family == 'curved':
        v = layered(rng, nz, nx, curved=True)
    elif family == 'faulted':
        v = faulted(rng, nz, nx)
    elif family == 'textured':
        v = textured(rng, nz, nx)
    else:
        raise ValueError(f'unknown family {family!r}')
    return np.clip(v, VMIN, VMAX).astype(np.float32)


def population(n=500, nz=70, nx=70, tag=1):
    """``n`` models, an equal mix of the four families; model i uses seed [tag, i]."""
    return np.stack([model(FAMILIES[i * len(FAMILIES) // n], [tag, i], nz, nx) for i in range(n)])


def small_model(seed=0, nz=70, nx=70):
    """The single curved 3-5-layer model of the small plain-method case."""
    return model('curved', seed, nz, nx)


RHOS = (0.6, 1.0, 1.4)   # slow / medium / fast background factors of the depth trend


def uneven_workload(n_solves=2000, seed=2, nz_range=(70, 200), nx_range=(70, 300), nt_range=(1000, 3000),
                    shots_range=(1, 9), bgs_range=(1, 3)):
    """Seeded models of uneven size for batched RTM, until `n_solves` (model, background, shot) solves.

    Per model: nz, nx, nt, shot count and background count drawn uniformly from the
    ranges (inclusive), family cycling through FAMILIES, shots at
    round(linspace(0, nx - 1, n)), backgrounds clip(v_s + rho * trend) for the
    first `n_bg` of a seeded permutation of RHOS, with v_s the model's top-row
    mean and trend its own lateral-mean depth profile minus v_s.  The last model's
    shots are cut so that the total is exactly `n_solves`.
    Returns a list of dicts: truth [nz, nx], backgrounds [n_bg, nz, nx], nt, shot_cols, v_s.
    """
    rng = np.random.default_rng([seed, 7])
    out, total, i = [], 0, 0
    while total < n_solves:
        nz = int(rng.integers(nz_range[0], nz_range[1] + 1))
        nx = int(rng.integers(nx_range[0], nx_range[1] + 1))
        nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
        ns = int(rng.integers(shots_range[0], shots_range[1] + 1))
        nb = int(rng.integers(bgs_range[0], bgs_range[1] + 1))
        rhos = [RHOS[j] for j in rng.permutation(len(RHOS))[:nb]]
        left = n_solves - total
        if ns * nb > left:                       # trim the last model
            nb = min(nb, left)
            ns = max(1, left // nb)
            nb = left // ns
            rhos = rhos[:nb]
        truth = model(FAMILIES[i % len(FAMILIES)], [seed, i], nz, nx)
        v_s = float(truth[0].astype(np.float64).mean())
        trend = truth.astype(np.float64).mean(1) - v_s
        bgs = np.stack([np.tile(np.clip(v_s + r * trend, VMIN, VMAX)[:, None], (1, nx)) for r in rhos])
        cols = [int(c) for c in np.round(np.linspace(0, nx - 1, ns))]
        out.append(dict(truth=truth, backgrounds=bgs.astype(np.float32), nt=nt, shot_cols=cols, v_s=v_s))
        total += ns * nb
        i += 1
    return out
