"""Generate tests/golden/process_small.npz by running the REFERENCE's surface-velocity picker.

    python tests/golden/make_golden_process.py /path/to/ShotSweep

Imports ShotSweep's ``openfwi/physics/gpu.py`` and ``background.py`` unmodified.
Gathers of three seeded models (curved, faulted, textured families) come from
the reference simulator in float64 and are stored rounded to float16 (to keep
the fixture small); the reference's ``estimate_surface_velocity`` runs on
exactly those values in float64.  So do the gathers of a model whose first
arrivals are too fast for its slope window.  Four more inputs, rebuilt by
``derived`` here and in the tests, exercise its error paths: all-zero gathers,
seeded white noise, gathers whose near-offset traces are zeroed in three shots,
and a single non-finite sample.  For each case the fixture holds
the reference's seven outputs, or its ValueError message.
"""
import sys
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

KEYS = ('velocity', 'confidence', 'fit_rmse_ms', 'short_offset_curvature', 'shot_slope_spread',
        'far_offset_velocity', 'possible_refraction')


SIMULATED = ('curved', 'faulted', 'textured', 'fast')
DERIVED = ('zeros', 'noise', 'near_zeroed', 'nonfinite')


def simulated(sim, synth):
    """Reference gathers of the three seeded models and the too-fast model, rounded to float16."""
    out = {}
    for name, seed in (('curved', [21, 0]), ('faulted', [21, 1]), ('textured', [21, 2])):
        model = synth.model(name, seed)
        out[name] = sim.gathers(model[None].astype(np.float64))[0]
    fast = np.full((1, 70, 70), 4400.0)
    fast[:, :3] = 4700.0                    # surface faster than the 1400-4600 m/s window
    out['fast'] = sim.gathers(fast)[0]
    return {k: v.astype(np.float16) for k, v in out.items()}


def derived(base):
    """The error-path inputs, rebuilt the same way here and in the tests (float32)."""
    out = {'zeros': np.zeros((5, 1000, 70), np.float32),
           'noise': np.random.default_rng(5).standard_normal((5, 1000, 70)).astype(np.float32)}
    g = base['curved'].astype(np.float32)
    for s in (0, 1, 2):                     # no 10-60 m traces in three shots
        cols = [r for r in range(70) if 10 <= abs(r * 10.0 - [0, 170, 340, 520, 690][s]) <= 60]
        g[s][:, cols] = 0
    out['near_zeroed'] = g
    g = base['faulted'].astype(np.float32)
    g[2, 500, 33] = np.nan
    out['nonfinite'] = g
    return out


def main(ref_root):
    sys.path.insert(0, str(Path(ref_root) / 'openfwi' / 'physics'))
    import gpu                      # noqa: E402  (the reference module)
    import background as BG         # noqa: E402
    from shotsweep_b200 import synth
    torch.set_num_threads(8)
    sim = gpu.Sim(device='cpu', dtype=torch.float64)
    base = simulated(sim, synth)
    data = {**{k: base[k].astype(np.float32) for k in SIMULATED}, **derived(base)}
    names = list(SIMULATED) + list(DERIVED)
    results = np.full((len(names), len(KEYS)), np.nan)
    errors = []
    for i, name in enumerate(names):
        try:
            est = BG.estimate_surface_velocity(data[name].astype(np.float64))
            results[i] = [float(est[k]) for k in KEYS]
            errors.append('')
        except ValueError as error:
            errors.append(str(error))
    np.savez_compressed(HERE / 'process_small.npz', names=np.array(names),
                        gathers=np.stack([base[n] for n in SIMULATED]), results=results,
                        errors=np.array(errors), keys=np.array(KEYS))
    for n, e, r in zip(names, errors, results):
        print(f'{n:12s} {e or r}')


if __name__ == '__main__':
    main(sys.argv[1] if len(sys.argv) > 1 else '/root/reference')
