"""Generate the golden fixtures in this folder by running the REFERENCE itself.

Run from the repository root, in a container that has the ShotSweep source:

    python tests/golden/make_golden.py /path/to/ShotSweep

It imports ShotSweep's ``openfwi/physics/gpu.py`` and ``background.py``
unmodified, runs them on the CPU in float64 on seeded synthetic inputs, and
writes small ``.npz`` fixtures.  The fixtures pin both the CPU oracle
(``oracle/oracle.py``) and the CUDA path; nothing at test time needs the
reference source.

Fixtures:
  plain_small.npz  one seeded curved-layer model: reference gathers (5x1000x70),
                   its three backgrounds (surface velocity from the reference's
                   picker, depth trend over a 500-model synthetic population),
                   and the reference's muted images / gradients / illumination.
  fd_small.npz     the reference test's own inverse-crime case (2000 m/s, 2400
                   below row 8; tests/test_physics.py:26-33): gradients and
                   illumination with and without the 2000 m/s mute.
  ops_small.npz    lap / lap_adjoint on seeded 2x9x11 arrays, fold_edge_padding
                   on a seeded 2x150x150 array, and a subsampled mute table.
  fd_directions.npz  the reference test's five finite-difference directions
                   (tests/test_physics.py:43-61: interior, left, bottom and top
                   boundary strips, the velocity-dependent source cell) and its
                   muted bottom strip (:63-74), epsilon 0.1 m/s, central
                   differences of the reference's float64 loss, with the
                   reference's own float64 adjoint directional derivatives.
  calib_small.npz  the reference's calibrate() (gpu.py:213-221) on two seeded
                   models whose observed gathers carry a shaped source (the
                   Ricker rotated by 40 degrees of phase, delayed 3 samples and
                   scaled by 1.3), made by the reference simulator in float64.

    python tests/golden/make_golden.py /path/to/ShotSweep [fixture ...]

writes only the named fixtures (fd_directions, calib) when
any are given.
"""
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


FD_DIRECTIONS = {   # tests/test_physics.py:45-51 (the reference test's own strips and cells)
    'interior': (slice(10, 30), 35),
    'left_boundary': (slice(10, 30), 0),
    'bottom_boundary': (69, slice(25, 45)),
    'top_boundary': (0, slice(25, 45)),
    'velocity_dependent_source': (1, 34),
}


def fd_directions(gpu, sim):
    """Central differences of the reference's float64 loss along the reference test's directions."""
    velocity = np.full((1, 70, 70), 2000.0)
    truth = velocity.copy()
    truth[:, 8:] = 2400.0
    observed = sim.gathers(truth).astype(np.float32).astype(np.float64)   # what a float32 caller passes
    epsilon = 0.1
    gradient = sim.gradient(velocity, observed)[0].sum(1)
    out = {'velocity': velocity, 'observed': observed.astype(np.float32), 'epsilon': np.float64(epsilon)}

    def loss(v, weights=None):
        r = sim.gathers(v) - observed
        return 0.5 * np.sum((1.0 if weights is None else weights) * r * r)

    for name, loc in FD_DIRECTIONS.items():
        d = np.zeros_like(velocity)
        d[(0,) + loc] = 1.0
        out[f'fd_{name}'] = np.float64((loss(velocity + epsilon * d) - loss(velocity - epsilon * d)) / (2 * epsilon))
        out[f'adj_{name}'] = np.float64(np.sum(gradient * d))
    # muted case (tests/test_physics.py:63-74): bottom strip, mute velocity 2000 m/s
    mute = np.array([2000.0])
    g_muted = sim.gradient(velocity, observed, v_mute=mute)[0].sum(1)
    weights = sim.mute_weights(mute).cpu().numpy()
    d = np.zeros_like(velocity)
    d[:, 69, 25:45] = 1.0
    out['fd_muted_bottom'] = np.float64((loss(velocity + epsilon * d, weights) - loss(velocity - epsilon * d, weights))
                                        / (2 * epsilon))
    out['adj_muted_bottom'] = np.float64(np.sum(g_muted * d))
    out['names'] = np.array(list(FD_DIRECTIONS))
    np.savez_compressed(HERE / 'fd_directions.npz', **out)


def shaped_source(ricker, degrees=40.0, delay=3, scale=1.3):
    """The Ricker with a constant phase rotation, a delay of whole samples and a gain (a stand-in field source)."""
    n = len(ricker)
    spec = np.fft.rfft(ricker)
    f = np.arange(len(spec))
    spec = spec * np.exp(-1j * np.deg2rad(degrees)) * np.exp(-2j * np.pi * f * delay / n)
    return scale * np.fft.irfft(spec, n=n)


def calibration(gpu):
    from shotsweep_b200 import synth
    models = np.stack([synth.model('layered', [5, 0]), synth.model('textured', [5, 1])]).astype(np.float64)
    shaped = shaped_source(gpu.RICKER)
    observed = gpu.Sim(shaped, device='cpu', dtype=torch.float64).gathers(models).astype(np.float32)
    wavelet = gpu.calibrate(list(models), list(observed.astype(np.float64)))
    np.savez_compressed(HERE / 'calib_small.npz', models=models, observed=observed, shaped=shaped,
                        wavelet=np.asarray(wavelet, np.float64))


def main(ref_root, only=()):
    sys.path.insert(0, str(Path(ref_root) / 'openfwi' / 'physics'))
    import gpu                      # noqa: E402  (the reference module)
    import background as BG         # noqa: E402
    from shotsweep_b200 import synth

    torch.set_num_threads(8)
    sim = gpu.Sim(device='cpu', dtype=torch.float64)
    if only:
        if 'fd_directions' in only:
            fd_directions(gpu, sim)
        if 'calib' in only:
            gpu.DEV = torch.device('cpu')          # calibrate() builds Sim(RICKER) on the module default device
            calibration(gpu)
        print('wrote', ', '.join(only))
        return

    # --- plain small case -------------------------------------------------
    model = synth.small_model(0)
    gathers = sim.gathers(model[None].astype(np.float64))[0].astype(np.float32)
    trend = BG.depth_trend(synth.population(500))
    try:
        v_s = BG.estimate_surface_velocity(gathers.astype(np.float64))['velocity']
        picked = True
    except ValueError:
        v_s = float(model[0].mean())
        picked = False
    bgs = BG.backgrounds(v_s, trend)
    obs = np.repeat(gathers[None].astype(np.float64), 3, 0)
    mute = np.full(3, v_s)
    images, illum = sim.images(bgs, obs, v_mute=mute)
    grad, illum_g = sim.gradient(bgs, obs, v_mute=mute)
    images_nl, _ = sim.images(bgs, obs, v_mute=mute, laplacian=False)
    np.savez_compressed(HERE / 'plain_small.npz', model=model, gathers=gathers, trend=trend,
                        v_surface=np.float64(v_s), picked=picked, backgrounds=bgs,
                        images=images.astype(np.float32), images_nolap=images_nl.astype(np.float32),
                        illum=illum.astype(np.float32), grad=grad.astype(np.float32))
    assert np.allclose(illum, illum_g)

    # --- reference test's inverse-crime FD case ----------------------------
    velocity = np.full((1, 70, 70), 2000.0)
    truth = velocity.copy()
    truth[:, 8:] = 2400.0
    observed = sim.gathers(truth).astype(np.float32)
    g0, i0 = sim.gradient(velocity, observed.astype(np.float64))
    g1, i1 = sim.gradient(velocity, observed.astype(np.float64), v_mute=np.array([2000.0]))
    np.savez_compressed(HERE / 'fd_small.npz', velocity=velocity, truth=truth, observed=observed,
                        grad=g0.astype(np.float32), illum=i0.astype(np.float32),
                        grad_muted=g1.astype(np.float32), illum_muted=i1.astype(np.float32))

    # --- small operator pins ------------------------------------------------
    gen = torch.Generator().manual_seed(8)
    x = torch.randn(2, 9, 11, generator=gen, dtype=torch.float64)
    y = torch.randn(2, 9, 11, generator=gen, dtype=torch.float64)
    big = torch.randn(2, 150, 150, generator=gen, dtype=torch.float64)
    mute = sim.mute_weights(np.array([1800.0, 3100.0])).numpy()
    np.savez_compressed(HERE / 'ops_small.npz', x=x.numpy(), y=y.numpy(), lap_x=gpu.lap(x).numpy(),
                        lapT_y=gpu.lap_adjoint(y).numpy(), big=big.numpy(),
                        fold_big=gpu.fold_edge_padding(big, 40).numpy(),
                        mute_v=np.array([1800.0, 3100.0]), mute_sub=mute[:, :, ::7, :].astype(np.float32),
                        ricker=gpu.RICKER, src=np.array(gpu.SRC))
    fd_directions(gpu, sim)
    gpu.DEV = torch.device('cpu')
    calibration(gpu)
    print('wrote fixtures; surface velocity', v_s, 'picked' if picked else 'fallback')


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else '/root/reference', tuple(sys.argv[2:]))
