"""The steps around the images on the GPU: surface velocity, backgrounds, the float16 image cache
(2_process.py:193-213) and the training-input transforms (3_train.py:157-158,188-189,198).

Tolerances: surface-velocity diagnostics within 1e-9 relative of the reference's float64
results (its line fits use lstsq, these the normal equations) and the same ValueError
messages; image cache, backgrounds, batch gathers and targets bit-identical to the NumPy
restatement; stored gathers within one float16 unit (log1p of float32 on two libraries).
"""
import numpy as np
import pytest
import torch

from .conftest import golden
from .test_oracle import process_case

pytestmark = pytest.mark.gpu


def test_surface_velocity_matches_reference():
    from shotsweep_b200 import background as BG
    names, data, g = process_case(None)
    keys = [str(k) for k in g['keys']]
    for i, name in enumerate(names):
        err = str(g['errors'][i])
        if err:
            with pytest.raises(ValueError) as info:
                BG.estimate_surface_velocity(data[name])
            assert str(info.value) == err, name
        else:
            est = BG.estimate_surface_velocity(data[name])
            got = np.array([float(est[k]) for k in keys])
            np.testing.assert_allclose(got, g['results'][i], rtol=1e-9, atol=1e-12, err_msg=name)


def test_surface_velocity_batch_and_uneven_acquisition():
    from oracle import postprocess as PP
    from shotsweep_b200 import background as BG
    names, data, g = process_case(None)
    ok = [n for i, n in enumerate(names) if not str(g['errors'][i])]
    batch = np.stack([data[n] for n in ok])
    est = BG.estimate_surface_velocity_batch(batch)
    for e, n in zip(est, ok):
        ref = PP.estimate_surface_velocity(data[n].astype(np.float64))
        for k in BG.KEYS:
            np.testing.assert_allclose(float(e[k]), float(ref[k]), rtol=1e-9, atol=1e-12)
    with pytest.raises(ValueError, match='model 1: surface velocity unavailable: no nonzero onset traces'):
        BG.estimate_surface_velocity_batch(np.stack([data['curved'], data['zeros']]))
    # three shots of a 120-column survey at other positions, traces of 1400 samples
    from shotsweep_b200 import engine
    from oracle import oracle as O
    cols = (10, 60, 110)
    eng = engine.Engine(engine.geometry(50, 120, 700, 20, cols))
    truth = np.stack([np.tile(np.linspace(1800, 3000, 50, dtype=np.float32)[:, None], (1, 120))])
    obs = eng.forward(torch.tensor(truth, device=eng.device), engine.scaled_wavelet(O.ricker(700), eng.device))
    src_x = np.array(cols) * 10.0
    got = BG.surface_estimates(obs, src_x=src_x)[0]
    try:
        ref = PP.estimate_surface_velocity(obs[0].cpu().numpy().astype(np.float64), src_x=src_x)
        assert got.status == 0
        np.testing.assert_allclose(got.velocity, ref['velocity'], rtol=1e-9)
        np.testing.assert_allclose(got.confidence, ref['confidence'], rtol=1e-9)
    except ValueError:
        assert got.status != 0


def test_image_cache_bit_identical():
    from oracle import postprocess as PP
    from shotsweep_b200 import process
    img = golden('plain_small')['images'][None].astype(np.float32)
    rng = np.random.default_rng(3)
    extra = (rng.standard_normal((3, 3, 5, 70, 70)) * rng.uniform(1e-3, 1e3, (3, 1, 1, 1, 1))).astype(np.float32)
    extra[1, :, :, 10:20] = 0                                   # many ties at zero
    extra[2] = np.round(extra[2] * 4) / 4                        # repeated values around the percentile
    imgs = np.concatenate([img, extra])
    ref, ref_scale = PP.image_cache(imgs)
    got, scale = process.image_cache(torch.tensor(imgs, device='cuda'))
    np.testing.assert_array_equal(scale.cpu().numpy(), ref_scale)
    np.testing.assert_array_equal(got.cpu().numpy().view(np.uint16), ref.view(np.uint16))
    bad = imgs[:2].copy()
    bad[1, 0, 0, 30, 30] = np.inf
    with pytest.raises(ValueError, match=r'models \[1\]'):
        process.image_cache(torch.tensor(bad, device='cuda'))
    with pytest.raises(ValueError, match=r'models \[0\]'):
        process.image_cache(torch.zeros(1, 3, 5, 70, 70, device='cuda'))


def test_backgrounds_and_training_inputs():
    from oracle import oracle as O
    from oracle import postprocess as PP
    from shotsweep_b200 import background as BG, train_inputs as TI
    trend = golden('plain_small')['trend']
    v1 = np.array([1523.4, 1850.0, 2210.7])
    got = BG.backgrounds(v1, trend).cpu().numpy()
    ref = np.stack([O.backgrounds(v, trend) for v in v1]).astype(np.float32)
    np.testing.assert_array_equal(got, ref)
    g = golden('plain_small')['gathers'][None]
    stored = TI.stored_gathers(torch.tensor(g, device='cuda')).cpu().numpy()
    ref_stored = PP.signed_log1p(g)
    diff = np.abs(stored.view(np.uint16).astype(np.int32) - ref_stored.view(np.uint16).astype(np.int32))
    assert diff.max() <= 1 and (diff == 0).mean() > 0.999
    batch = TI.batch_gathers(torch.tensor(ref_stored, device='cuda'), 0.37).cpu().numpy()
    np.testing.assert_array_equal(batch, PP.scaled(ref_stored, 0.37))
    with pytest.raises(ValueError, match='scale'):
        TI.batch_gathers(torch.tensor(ref_stored, device='cuda'), float('nan'))
    y = golden('plain_small')['model'][None].astype(np.float32)
    np.testing.assert_array_equal(TI.targets(torch.tensor(y, device='cuda')).cpu().numpy(), PP.targets(y))
    v1f = v1.astype(np.float32)
    tr32 = trend.astype(np.float32)
    got = TI.vref(torch.tensor(v1f, device='cuda'), torch.tensor(tr32, device='cuda')).cpu().numpy()
    np.testing.assert_array_equal(got, PP.vref(v1f, tr32))


def test_process_batch_matches_oracle_chain():
    """Picks, backgrounds, images and cache together against the float64 oracle of the same steps."""
    from oracle import oracle as O
    from oracle import postprocess as PP
    from shotsweep_b200 import gpu, process
    names, data, g = process_case(None)
    obs = np.stack([data['curved'], data['textured']])
    trend = golden('plain_small')['trend']
    out = process.process_batch(gpu.Sim(device='cuda'), obs, trend)
    v1 = np.array([PP.estimate_surface_velocity(o.astype(np.float64))['velocity'] for o in obs])
    np.testing.assert_allclose(out['surface_velocity'], v1.astype(np.float32), rtol=1e-6)
    bgs = np.concatenate([O.backgrounds(v, trend) for v in v1])
    img, _ = O.OracleSim(checkpoint_interval=100).images(bgs, np.repeat(obs.astype(np.float64), 3, 0),
                                                         v_mute=np.repeat(v1, 3))
    ref, _ = PP.image_cache(img.reshape(2, 3, 5, 70, 70).astype(np.float32))
    got = out['images'].cpu().numpy().astype(np.float32)
    ref = ref.astype(np.float32)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-3
