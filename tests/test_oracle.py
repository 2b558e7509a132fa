"""The CPU oracle against golden vectors that the reference itself produced (tests/golden)."""
import numpy as np
from pathlib import Path
import pytest
import torch

from oracle import oracle as O

from .conftest import golden


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_small_operators_match_reference():
    g = golden('ops_small')
    x, y = torch.from_numpy(g['x']), torch.from_numpy(g['y'])
    np.testing.assert_allclose(O.lap(x).numpy(), g['lap_x'], rtol=0, atol=1e-12)
    np.testing.assert_allclose(O.lap_adjoint(y).numpy(), g['lapT_y'], rtol=0, atol=1e-12)
    np.testing.assert_allclose(O.fold_edge_padding(torch.from_numpy(g['big']), 40).numpy(), g['fold_big'],
                               rtol=1e-12, atol=1e-10)
    np.testing.assert_allclose(O.ricker(), g['ricker'], rtol=0, atol=1e-15)
    assert O.shot_columns(70, 5) == tuple(g['src'])
    sim = O.OracleSim()
    mute = sim.mute_weights(g['mute_v']).numpy()[:, :, ::7, :]
    np.testing.assert_allclose(mute, g['mute_sub'], rtol=0, atol=1e-7)


def test_laplacian_transpose_including_boundary():
    gen = torch.Generator().manual_seed(3)
    x = torch.randn(3, 13, 17, generator=gen, dtype=torch.float64)
    y = torch.randn(3, 13, 17, generator=gen, dtype=torch.float64)
    assert abs(float((O.lap(x) * y).sum() - (x * O.lap_adjoint(y)).sum())) < 1e-10


@pytest.fixture(scope='module')
def plain():
    return golden('plain_small')


def test_oracle_gathers_match_reference(plain):
    sim = O.OracleSim()
    out = sim.gathers(plain['model'][None].astype(np.float64))[0]
    assert rel(out, plain['gathers']) < 1e-6      # fixture stored as float32


def test_oracle_images_gradient_match_reference(plain):
    sim = O.OracleSim()
    bgs = plain['backgrounds']
    obs = np.repeat(plain['gathers'][None].astype(np.float64), 3, 0)
    mute = np.full(3, float(plain['v_surface']))
    grad, illum = sim.gradient(bgs, obs, v_mute=mute)
    assert rel(grad, plain['grad']) < 1e-6
    assert rel(illum, plain['illum']) < 1e-6
    img = O.image_epilogue(torch.from_numpy(grad), torch.from_numpy(illum)).numpy()
    assert rel(img, plain['images']) < 1e-6
    img_nl = O.image_epilogue(torch.from_numpy(grad), torch.from_numpy(illum), laplacian=False).numpy()
    assert rel(img_nl, plain['images_nolap']) < 1e-6


def test_oracle_inverse_crime_gradients_match_reference():
    g = golden('fd_small')
    sim = O.OracleSim()
    grad, illum = sim.gradient(g['velocity'], g['observed'].astype(np.float64))
    assert rel(grad, g['grad']) < 1e-6 and rel(illum, g['illum']) < 1e-6
    grad, illum = sim.gradient(g['velocity'], g['observed'].astype(np.float64), v_mute=np.array([2000.0]))
    assert rel(grad, g['grad_muted']) < 1e-6 and rel(illum, g['illum_muted']) < 1e-6


def test_oracle_background_helpers(plain):
    from shotsweep_b200 import synth
    trend = O.depth_trend(synth.population(500))
    np.testing.assert_allclose(trend, plain['trend'], rtol=1e-12)
    np.testing.assert_allclose(O.backgrounds(float(plain['v_surface']), trend), plain['backgrounds'], rtol=1e-12)


# ---- steps around the images: surface velocity, image cache, training inputs ----------------

def process_case(name):
    import importlib.util
    spec = importlib.util.spec_from_file_location('make_golden_process',
                                                  Path(__file__).parent / 'golden' / 'make_golden_process.py')
    mk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mk)
    g = golden('process_small')
    names = [str(n) for n in g['names']]
    base = {n: g['gathers'][i] for i, n in enumerate(mk.SIMULATED)}
    data = {**{k: v.astype(np.float32) for k, v in base.items()}, **mk.derived(base)}
    return names, data, g


def test_surface_velocity_oracle_matches_reference_outputs():
    from oracle import postprocess as PP
    names, data, g = process_case(None)
    keys = [str(k) for k in g['keys']]
    for i, name in enumerate(names):
        err = str(g['errors'][i])
        if err:
            with pytest.raises(ValueError) as info:
                PP.estimate_surface_velocity(data[name].astype(np.float64))
            assert str(info.value) == err, name
        else:
            est = PP.estimate_surface_velocity(data[name].astype(np.float64))
            got = np.array([float(est[k]) for k in keys])
            np.testing.assert_allclose(got, g['results'][i], rtol=1e-12, atol=1e-15, err_msg=name)


def test_image_cache_oracle_is_the_reference_epilogue():
    """The restatement applies 2_process.py:206-210 verbatim; check its properties on the reference images."""
    from oracle import postprocess as PP
    img = golden('plain_small')['images'][None]            # [1, 3, 5, 70, 70]
    cache, scale = PP.image_cache(img)
    assert cache.dtype == np.float16 and cache.shape == img.shape
    assert np.all(cache[..., :2, :] == 0) and np.abs(cache.astype(np.float32)).max() <= 4
    a = np.abs(img.copy())
    a[..., :2, :] = 0
    assert scale[0] == np.percentile(a.reshape(1, -1), 99, axis=1)[0]
    with pytest.raises(ValueError):
        PP.image_cache(np.zeros_like(img))


def test_oracle_calibrate_matches_reference():
    """calibrate() restated (gpu.py:213-221): float32 synthetics, pooled Wiener shaping of the Ricker."""
    c = golden('calib_small')
    torch.set_num_threads(max(1, torch.get_num_threads()))
    wavelet = O.calibrate(c['models'], c['observed'].astype(np.float64))
    assert rel(wavelet, c['wavelet']) < 1e-6


def test_oracle_finite_difference_matches_reference_top_strip():
    """The float64 oracle's loss gives the reference's own central difference along the top strip (the
    direction that edge padding folds onto the source row; tests/test_physics.py:48), epsilon 0.1 m/s."""
    fx = golden('fd_directions')
    velocity, observed = fx['velocity'], fx['observed'].astype(np.float64)
    eps = float(fx['epsilon'])
    sim = O.OracleSim()
    d = np.zeros_like(velocity)
    d[0, 0, 25:45] = 1.0

    def loss(v):
        r = sim.gathers(v) - observed
        return 0.5 * np.sum(r * r)

    fd = (loss(velocity + eps * d) - loss(velocity - eps * d)) / (2 * eps)
    assert abs(fd - float(fx['fd_top_boundary'])) <= 1e-8 * abs(fd)
