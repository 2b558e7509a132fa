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
"""
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def main(ref_root):
    sys.path.insert(0, str(Path(ref_root) / 'openfwi' / 'physics'))
    import gpu                      # noqa: E402  (the reference module)
    import background as BG         # noqa: E402
    from shotsweep_b200 import synth

    torch.set_num_threads(8)
    sim = gpu.Sim(device='cpu', dtype=torch.float64)

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
    print('wrote fixtures; surface velocity', v_s, 'picked' if picked else 'fallback')


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else '/root/reference')
