"""CUDA path vs the reference (golden fixtures) and vs the CPU oracle (odd geometries).

Tolerances are relative L2 against float64 results (the reference's own
float32 run reaches 3.3e-6 on gathers and <5e-5 per shot-image):
    gathers <= 1e-5; each shot-image, gradient and illumination <= 2e-4.
"""
import numpy as np
import pytest
import torch

from .conftest import golden

pytestmark = pytest.mark.gpu

GATHER_TOL = 1e-5
IMAGE_TOL = 2e-4
FIELD_TOL = 5e-5     # whole padded wavefields (checkpoints), which include the weak far field


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def per_image_rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1, a.shape[-2] * a.shape[-1])
    b = np.asarray(b, np.float64).reshape(-1, b.shape[-2] * b.shape[-1])
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


@pytest.fixture(scope='module')
def gpu():
    from shotsweep_b200 import gpu as G
    assert torch.cuda.is_available()
    return G


@pytest.fixture(scope='module')
def plain():
    return golden('plain_small')


def test_gathers_match_reference(gpu, plain):
    out = gpu.Sim().gathers(plain['model'][None].astype(np.float64))
    assert out.shape == (1, 5, 1000, 70) and out.dtype == np.float32
    assert rel(out[0], plain['gathers']) <= GATHER_TOL


def test_images_gradient_illum_match_reference(gpu, plain):
    sim = gpu.Sim()
    obs = np.repeat(plain['gathers'][None].astype(np.float64), 3, 0)
    mute = np.full(3, float(plain['v_surface']))
    img, illum = sim.images(plain['backgrounds'], obs, v_mute=mute)
    assert img.shape == (3, 5, 70, 70)
    assert per_image_rel(img, plain['images']).max() <= IMAGE_TOL
    assert per_image_rel(illum, plain['illum']).max() <= IMAGE_TOL
    grad, illum2 = sim.gradient(plain['backgrounds'], obs, v_mute=mute)
    assert per_image_rel(grad, plain['grad']).max() <= IMAGE_TOL
    np.testing.assert_array_equal(illum, illum2)
    img_nl, _ = sim.images(plain['backgrounds'], obs, v_mute=mute, laplacian=False)
    assert per_image_rel(img_nl, plain['images_nolap']).max() <= IMAGE_TOL


def test_inverse_crime_gradients_match_reference(gpu):
    g = golden('fd_small')
    sim = gpu.Sim()
    grad, illum = sim.gradient(g['velocity'], g['observed'])
    assert rel(grad, g['grad']) <= IMAGE_TOL and rel(illum, g['illum']) <= IMAGE_TOL
    grad, illum = sim.gradient(g['velocity'], g['observed'], v_mute=np.array([2000.0]))
    assert rel(grad, g['grad_muted']) <= IMAGE_TOL and rel(illum, g['illum_muted']) <= IMAGE_TOL


def test_module_helpers_match_reference(gpu):
    g = golden('ops_small')
    x, y = torch.from_numpy(g['x']), torch.from_numpy(g['y'])
    np.testing.assert_allclose(gpu.lap(x).numpy(), g['lap_x'], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(gpu.lap_adjoint(y).numpy(), g['lapT_y'], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(gpu.fold_edge_padding(torch.from_numpy(g['big']), 40).numpy(), g['fold_big'],
                               rtol=1e-11, atol=1e-10)
    xf = x.float().cuda()
    assert gpu.lap(xf).device.type == 'cuda'
    np.testing.assert_allclose(gpu.lap(xf).cpu().numpy(), g['lap_x'], rtol=1e-5, atol=1e-5)
    mute = gpu.Sim().mute_weights(g['mute_v']).cpu().numpy()[:, :, ::7, :]
    np.testing.assert_allclose(mute, g['mute_sub'], rtol=0, atol=2e-6)


CALIBRATE_TOL = 1e-5


def test_calibrate_matches_reference(gpu):
    """Source calibration (gpu.py:213-221) against the reference's own output on two seeded models whose
    observed gathers carry a phase-rotated, delayed, scaled Ricker (tests/golden/calib_small.npz): the
    drop-in's forward modelling runs on the GPU, the pooled Wiener filter on the host."""
    c = golden('calib_small')
    wavelet = gpu.calibrate(list(c['models']), list(c['observed'].astype(np.float64)))
    assert wavelet.shape == c['wavelet'].shape and np.isfinite(wavelet).all()
    assert rel(wavelet, c['wavelet']) <= CALIBRATE_TOL
    # the estimate recovers the shaped source it was given (a property of the method, not only of the code)
    assert rel(wavelet, c['shaped']) <= 0.05


def test_process_batch_stays_within_memory_budget(gpu):
    """2_process sizes its batch as budget // imaging_memory_bytes(3 rows) (2_process.py:166-171).  A call on
    that many models, with NumPy gathers as 2_process passes them, allocates no more device memory than the
    model says (and so stays inside the default 2 GiB), and its images equal those of a call that keeps
    every co-resident cluster busy, bit for bit (each solve's arithmetic does not depend on its slot)."""
    from oracle import oracle as O
    from shotsweep_b200 import engine, synth
    budget = 2 * 1024 ** 3
    per_model = gpu.imaging_memory_bytes(3)
    n = int(budget // per_model)
    assert n >= 15
    models = synth.population(n).astype(np.float64)
    sim = gpu.Sim()
    obs = sim.gathers(models)
    trend = O.depth_trend(models)
    v_s = models[:, 0, :].mean(1)
    bgs = np.concatenate([O.backgrounds(v, trend) for v in v_s])
    obs_rows = np.repeat(obs, 3, 0)
    vm = np.repeat(v_s, 3)
    torch.cuda.synchronize()
    fresh = gpu.Sim()
    base = torch.cuda.memory_allocated()
    torch.cuda.reset_peak_memory_stats()
    img, illum = fresh.images(bgs, obs_rows, v_mute=vm)
    torch.cuda.synchronize()
    used = torch.cuda.max_memory_allocated() - base
    assert used <= n * per_model <= budget, (used, n * per_model)
    eng = fresh.engine
    assert eng.max_slots is None            # the cap applies to the call only
    dev = eng.device
    f32 = dict(dtype=torch.float32, device=dev)
    ref_img, ref_illum = eng.images(torch.tensor(bgs, **f32), engine.scaled_wavelet(gpu.RICKER, dev),
                                    torch.tensor(obs_rows, **f32), torch.tensor(vm, **f32))
    eng.status()
    assert np.array_equal(img, ref_img.cpu().numpy()) and np.array_equal(illum, ref_illum.cpu().numpy())


def test_tile_height_does_not_change_results(gpu):
    """Plans at 4 rows per thread (512 threads per CTA) give the same gathers, images and illumination as
    the default 5 (384 threads), bit for bit, on the OpenFWI grid and on an odd one."""
    import ctypes
    from shotsweep_b200 import _lib, engine, synth
    L = _lib.load()
    for geom_args in ((70, 70, 300, 40, (0, 17, 34, 52, 69)), (23, 37, 160, 9, (0, 18, 36))):
        nz, nx = geom_args[:2]
        eng = engine.Engine(engine.geometry(*geom_args))
        dev = eng.device
        f32 = dict(dtype=torch.float32, device=dev)
        truth = torch.tensor(np.stack([synth.model('curved', [7, i], nz, nx) for i in range(2)]), **f32)
        bg = torch.tensor(np.stack([np.tile(np.linspace(1700, 3300, nz)[:, None], (1, nx))] * 2), **f32)
        w = engine.scaled_wavelet(np.sin(np.arange(geom_args[2]) * 0.2) * np.exp(-np.arange(geom_args[2]) / 30.0), dev)
        out = {}
        try:
            for rows in (5, 4):
                for mode in range(4):
                    assert L.ss_set_rows_per_thread(mode, rows) == 0
                assert eng.plan(2, _lib.MODE_IMAGES)['rows_per_thread'] == rows
                obs = eng.forward(truth, w)
                img, illum = eng.images(bg, w, obs, torch.tensor([1800.0, 1900.0], **f32))
                eng.status()
                out[rows] = (obs, img, illum)
        finally:
            for mode in range(4):
                L.ss_set_rows_per_thread(mode, 0)
        for a, b in zip(out[5], out[4]):
            assert torch.equal(a, b), geom_args
    assert L.ss_set_rows_per_thread(2, 3) == _lib.ERR_INVALID


def test_forward_returns_reference_structures(gpu, plain):
    sim = gpu.Sim(checkpoint_interval=250)
    out, ck, c2 = sim.forward(plain['model'][None], store=True)
    assert out.is_cuda and tuple(out.shape) == (1, 5, 1000, 70)
    assert sorted(ck) == [0, 250, 500, 750]
    assert tuple(ck[250][0].shape) == (1, 5, 150, 150) and tuple(c2.shape) == (1, 1, 150, 150)
    from oracle import oracle as O
    osim = O.OracleSim(checkpoint_interval=250)
    o_out, o_ck, o_c2 = osim.forward(plain['model'][None].astype(np.float64), store=True)
    for it in (250, 750):
        for j in (0, 1):
            assert rel(ck[it][j].cpu().numpy(), o_ck[it][j].numpy()) <= FIELD_TOL
    assert rel(c2.cpu().numpy(), o_c2.numpy()) <= 1e-6


def test_nonfinite_and_bad_shapes_rejected(gpu, plain):
    sim = gpu.Sim()
    obs = np.repeat(plain['gathers'][None].astype(np.float32), 1, 0).copy()
    obs[0, 2, 500, 3] = np.nan
    with pytest.raises(ValueError, match='finite'):
        sim.gradient(plain['backgrounds'][:1], obs)
    with pytest.raises(ValueError, match='finite'):
        sim.images(plain['backgrounds'][:1], obs[:, :4])
    with pytest.raises(ValueError, match='velocities'):
        sim.gathers(-np.ones((1, 70, 70)))
    with pytest.raises(ValueError, match='eps'):
        sim.images(plain['backgrounds'][:1], obs, eps=0)
    # the call after a rejected one is clean
    obs[0, 2, 500, 3] = 0.0
    sim.gradient(plain['backgrounds'][:1], obs)


def test_batch_larger_than_resident_clusters_is_deterministic(gpu):
    """More solves than co-resident clusters: each result equals its solo run, bit for bit."""
    from shotsweep_b200 import synth
    sim = gpu.Sim()
    models = synth.population(48)
    obs = sim.gathers(models)
    bgs = np.stack([np.tile(np.linspace(1600, 3800, 70)[:, None], (1, 70)) + 10 * i for i in range(48)])
    img, illum = sim.images(bgs, obs, v_mute=np.full(48, 1700.0))
    for i in (0, 31, 47):
        img1, illum1 = sim.images(bgs[i:i + 1], obs[i:i + 1], v_mute=np.array([1700.0]))
        np.testing.assert_array_equal(img1[0], img[i])
        np.testing.assert_array_equal(illum1[0], illum[i])


def test_host_pipeline_equals_device_images(gpu):
    """The chunked host-observation pipeline (device velocities, or float32 / float64 host velocities; pinned
    or pageable gathers; uniform or growing chunks) gives the device-resident images bit for bit."""
    from shotsweep_b200 import engine, synth
    sim = gpu.Sim()
    eng = sim.engine
    models = synth.population(30)
    obs = torch.tensor(sim.gathers(models))
    bgs = torch.tensor(np.stack([np.tile(np.linspace(1600, 3800, 70)[:, None], (1, 70)) + 7 * i
                                 for i in range(30)]), dtype=torch.float32)
    vm = torch.full((30,), 1800.0, device=eng.device)
    w = engine.scaled_wavelet(gpu.RICKER, eng.device)
    ref_img, ref_illum = eng.images(bgs.to(eng.device), w, obs.to(eng.device), vm, 0.12)
    eng.status()
    assert [b - a for a, b in eng._chunks(30)][:2] == [9, 18]
    for vel, o, rows in ((bgs, obs.pin_memory(), None), (bgs.to(eng.device), obs, 7), (bgs.pin_memory(), obs, None),
                         (bgs.double(), obs.pin_memory(), 4)):
        img, illum = eng.images_from_host(vel, w, o, vm, 0.12, chunk_rows=rows)
        assert torch.equal(img, ref_img.cpu()) and torch.equal(illum, ref_illum.cpu())


ODD = [
    # nz, nx, nt, pad, shot columns, src_row
    (23, 37, 160, 9, (0, 18, 36), 1),
    (41, 19, 140, 6, (9,), 2),
    (12, 70, 120, 2, (0, 69), 1),
    (90, 31, 130, 12, (3, 15, 30, 5), 4),
    (150, 60, 110, 20, (0, 20, 40, 59), 1),
    (100, 300, 90, 40, (0, 150, 299), 1),
]


@pytest.mark.parametrize('case', ODD, ids=[f'{c[0]}x{c[1]}x{c[2]}p{c[3]}s{len(c[4])}' for c in ODD])
def test_odd_geometries_match_oracle(case):
    from oracle import oracle as O
    from shotsweep_b200 import engine, synth
    nz, nx, nt, pad, cols, src_row = case
    geom = O.Geometry(nz=nz, nx=nx, nt=nt, shot_cols=cols, src_row=src_row)
    rng = np.random.default_rng(nz * 1000 + nx)
    truth = np.stack([synth.model('textured', [7, i], nz, nx) for i in range(2)]).astype(np.float64)
    bg = np.stack([np.tile(np.linspace(1700, 3300, nz)[:, None], (1, nx)) + rng.uniform(-50, 50)
                   for _ in range(2)])
    wav = O.ricker(nt)
    osim = O.OracleSim(wavelet=wav, pad=pad, geom=geom, checkpoint_interval=17)
    obs = osim.gathers(truth)
    vm = np.array([1800.0, 2100.0])
    t_mute = 0.02 * nt * 1e-3          # short records: mute only the first fifth
    o_grad, o_illum = osim.gradient(bg, obs, v_mute=vm, t_mute=t_mute)
    o_img = O.image_epilogue(torch.from_numpy(o_grad), torch.from_numpy(o_illum)).numpy()

    eng = engine.Engine(engine.geometry(nz, nx, nt, pad, cols, src_row))
    dev = eng.device
    w = engine.scaled_wavelet(wav, dev)
    gat = eng.forward(torch.tensor(truth, dtype=torch.float32, device=dev), w).cpu().numpy()
    assert rel(gat, obs) <= GATHER_TOL
    v = torch.tensor(bg, dtype=torch.float32, device=dev)
    ob = torch.tensor(obs, dtype=torch.float32, device=dev)
    vmd = torch.tensor(vm, dtype=torch.float32, device=dev)
    grad, illum = eng.gradient(v, w, ob, vmd, t_mute)
    eng.status()
    assert per_image_rel(grad.cpu().numpy(), o_grad).max() <= IMAGE_TOL
    assert per_image_rel(illum.cpu().numpy(), o_illum).max() <= IMAGE_TOL
    img, illum2, grad2 = eng.images(v, w, ob, vmd, t_mute, want_grad=True)
    assert per_image_rel(img.cpu().numpy(), o_img).max() <= IMAGE_TOL
    np.testing.assert_array_equal(grad2.cpu().numpy(), grad.cpu().numpy())
    # no mute at all
    o_grad0, _ = osim.gradient(bg, obs)
    grad0, _ = eng.gradient(v, w, ob)
    assert per_image_rel(grad0.cpu().numpy(), o_grad0).max() <= IMAGE_TOL
