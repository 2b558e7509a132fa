"""Uneven batches: models of different grids, step counts, shots, pads and mutes in one launch sequence.

Every solve of a batch must give what the single-geometry entry points give for
its own geometry (those are pinned to the float64 oracle by tests/test_parity_gpu.py):
the arithmetic of a cell does not depend on how the grid is cut into bands, so
the comparison is exact.  One small model is also checked against the oracle
directly, at the parity tolerance of images (2e-4 relative L2 per shot-image).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

IMAGE_TOL = 2e-4


def shapes():
    from shotsweep_b200.batch import Shape, shot_columns
    return [
        Shape(23, 37, 160, [0, 18, 36], pad=9, v_mute=1800.0),
        Shape(30, 50, 130, shot_columns(50, 2), pad=12),
        Shape(17, 29, 190, [5], pad=6, src_row=2, v_mute=2000.0),
        Shape(40, 61, 100, shot_columns(61, 9), pad=20, v_mute=1900.0),
        Shape(60, 90, 120, shot_columns(90, 5), pad=40, v_mute=2100.0),   # a larger size class
        Shape(100, 300, 90, shot_columns(300, 3), pad=40),                 # a cluster of several CTAs
        Shape(26, 26, 150, shot_columns(26, 4), pad=10),
    ]


def models_for(shs, tag):
    from shotsweep_b200 import synth
    fams = ('layered', 'curved', 'faulted', 'textured')
    return [synth.model(fams[i % 4], [tag, i], s.nz, s.nx) for i, s in enumerate(shs)]


def backgrounds_for(truths):
    return [np.tile(np.linspace(1600.0, 3300.0, t.shape[0], dtype=np.float32)[:, None], (1, t.shape[1]))
            for t in truths]


@pytest.fixture(scope='module')
def case():
    from oracle import oracle as O
    from shotsweep_b200.batch import UnevenBatch
    shs = shapes()
    batch = UnevenBatch(shs)
    dev = batch.device
    max_nt = batch.max_nt
    wav = torch.tensor(O.ricker(max_nt) * 1e3, dtype=torch.float32, device=dev)
    truths = models_for(shs, 5)
    bgs = backgrounds_for(truths)
    vt = batch.pack_models(truths)
    vb = batch.pack_models(bgs)
    obs = batch.forward(vt, wav)
    img, illum, grad = batch.images(vb, wav, obs, t_mute=0.03, want_grad=True)
    torch.cuda.synchronize()
    batch.status()
    return dict(batch=batch, shapes=shs, wav=wav, truths=truths, bgs=bgs, vt=vt, vb=vb, obs=obs, img=img,
                illum=illum, grad=grad)


def engine_for(sh):
    from shotsweep_b200 import engine
    return engine.Engine(engine.geometry(sh.nz, sh.nx, sh.nt, sh.pad, sh.shot_cols, sh.src_row))


def test_batch_spans_several_size_classes(case):
    cls = case['batch'].classes()
    assert len(cls) >= 2
    assert sum(c['n_solves'] for c in cls) == sum(s.n_shots for s in case['shapes'])
    assert all(c['cluster'] >= c['min_cluster'] for c in cls)


def test_batch_forward_equals_single_geometry_forward(case):
    b = case['batch']
    for i, sh in enumerate(case['shapes']):
        eng = engine_for(sh)
        ref = eng.forward(torch.tensor(case['truths'][i][None], device=b.device), case['wav'][:sh.nt].contiguous())
        got = b.unpack_traces(case['obs'], i)
        assert torch.equal(got, ref[0]), f'model {i}: max diff {(got - ref[0]).abs().max().item()}'


def test_batch_images_equal_single_geometry_images(case):
    b = case['batch']
    for i, sh in enumerate(case['shapes']):
        eng = engine_for(sh)
        vm = torch.tensor([sh.v_mute], device=b.device) if sh.v_mute > 0 else None
        obs = b.unpack_traces(case['obs'], i)[None].contiguous()
        img, illum, grad = eng.images(torch.tensor(case['bgs'][i][None], device=b.device),
                                      case['wav'][:sh.nt].contiguous(), obs, vm, 0.03, want_grad=True)
        eng.status()
        for name, got, ref in (('img', case['img'], img), ('illum', case['illum'], illum),
                               ('grad', case['grad'], grad)):
            g = b.unpack_images(got, i)
            assert torch.equal(g, ref[0]), f'model {i} {name}: max diff {(g - ref[0]).abs().max().item()}'


def test_batch_images_match_oracle(case):
    from oracle import oracle as O
    i = 2                                     # 17 x 29, one shot at column 5, sources on row 2, muted
    sh = case['shapes'][i]
    geom = O.Geometry(nz=sh.nz, nx=sh.nx, nt=sh.nt, shot_cols=tuple(sh.shot_cols), src_row=sh.src_row)
    osim = O.OracleSim(wavelet=O.ricker(sh.nt), pad=sh.pad, geom=geom)
    obs = case['batch'].unpack_traces(case['obs'], i).cpu().numpy().astype(np.float64)[None]
    ref_img, ref_illum = osim.images(case['bgs'][i][None].astype(np.float64), obs,
                                     v_mute=np.array([sh.v_mute]), t_mute=0.03)
    got = case['batch'].unpack_images(case['img'], i).cpu().numpy()
    for s in range(sh.n_shots):
        r = np.linalg.norm(got[s] - ref_img[0, s]) / np.linalg.norm(ref_img[0, s])
        assert r <= IMAGE_TOL, (s, r)


def test_cluster_table_and_streams_do_not_change_results(case):
    from shotsweep_b200.batch import UnevenBatch
    b = case['batch']
    table = {c['min_cluster']: min(16, c['min_cluster'] + 1) for c in b.classes()}
    alt = UnevenBatch(case['shapes'], clusters=table, schedule=0)
    assert [c['cluster'] for c in alt.classes()] != [c['cluster'] for c in b.classes()]
    img, illum, _ = alt.images(case['vb'], case['wav'], case['obs'], t_mute=0.03)
    alt.status()
    assert torch.equal(img, case['img']) and torch.equal(illum, case['illum'])
    for sched in (1, 2):
        alt = UnevenBatch(case['shapes'], schedule=sched)
        img, illum, _ = alt.images(case['vb'], case['wav'], case['obs'], t_mute=0.03)
        alt.status()
        assert torch.equal(img, case['img']) and torch.equal(illum, case['illum']), sched


def test_graph_replay_equals_eager(case):
    b = case['batch']
    graph, img, illum = b.capture_images(case['vb'], case['wav'], case['obs'], t_mute=0.03)
    img.zero_()
    graph.replay()
    torch.cuda.synchronize()
    b.status()
    assert torch.equal(img, case['img']) and torch.equal(illum, case['illum'])


def test_autotuner_picks_a_fitting_launch_shape_per_class():
    """The tuner's table gives every size class a (cluster size, tile height) pair from the candidates it
    times: a tile height of 4-6 rows and a cluster from the smallest that fits every model of the class at
    that height to one above it (or 16 for classes of large grids)."""
    from shotsweep_b200 import autotune
    from shotsweep_b200.batch import TILE_ROWS
    shs = shapes()[:5]
    table = autotune.tune(shs, sample_nt=64, reps=1, extra=1)
    members = autotune.class_members(shs)
    assert set(table) == set(members)
    for c_min, (c, rows) in table.items():
        assert rows in TILE_ROWS
        lo = max(autotune.smallest_cluster(shs[i], rows) for i in members[c_min])
        assert lo <= c <= lo + 1 or (lo >= 10 and c == 16), (c_min, c, rows, lo)


def test_tile_heights_do_not_change_results(case):
    """Every class forced to 4 and to 6 rows per thread (at the smallest cluster that fits) gives the
    same images and illumination, bit for bit: a cell's arithmetic does not depend on the tile."""
    from shotsweep_b200.batch import UnevenBatch
    b = case['batch']
    for rows in (4, 6):
        table = {c['min_cluster']: (c['min_cluster'], rows) for c in b.classes()}
        alt = UnevenBatch(case['shapes'], clusters=table, schedule=0)
        assert all(c['rows_per_thread'] == rows for c in alt.classes())
        img, illum, _ = alt.images(case['vb'], case['wav'], case['obs'], t_mute=0.03)
        alt.status()
        assert torch.equal(img, case['img']) and torch.equal(illum, case['illum']), rows


def test_batch_rejects_bad_input(case):
    from shotsweep_b200.batch import Shape, UnevenBatch
    with pytest.raises(ValueError, match='src_row'):
        UnevenBatch([Shape(20, 20, 50, [3], pad=5, src_row=20)]).plan(2)
    with pytest.raises(ValueError, match='shot column'):
        UnevenBatch([Shape(20, 20, 50, [20], pad=5)]).plan(2)
    b = case['batch']
    with pytest.raises(ValueError, match='wavelet'):
        b.images(case['vb'], case['wav'][:10].contiguous(), case['obs'])
    with pytest.raises(ValueError, match='vel'):
        b.images(case['vb'][:-1].contiguous(), case['wav'], case['obs'])


def test_full_size_models_equal_single_geometry():
    """The largest grids and time axes of the uneven workload (200 x 300 cells over 3000 steps, 150 x 250 over
    2000): clusters of 14 and 9 CTAs in one batch, bit-identical to the single-geometry path."""
    from oracle import oracle as O
    from shotsweep_b200.batch import Shape, UnevenBatch, shot_columns
    shs = [Shape(200, 300, 3000, shot_columns(300, 2), v_mute=1900.0), Shape(150, 250, 2000, shot_columns(250, 3))]
    b = UnevenBatch(shs)
    assert sorted(c['cluster'] for c in b.classes()) == sorted(c['min_cluster'] for c in b.classes())
    assert max(c['cluster'] for c in b.classes()) >= 12
    wav = torch.tensor(O.ricker(b.max_nt) * 1e3, dtype=torch.float32, device=b.device)
    truths = models_for(shs, 8)
    bgs = backgrounds_for(truths)
    obs = b.forward(b.pack_models(truths), wav)
    img, illum, _ = b.images(b.pack_models(bgs), wav, obs, t_mute=0.1)
    b.status()
    for i, sh in enumerate(shs):
        eng = engine_for(sh)
        vm = torch.tensor([sh.v_mute], device=b.device) if sh.v_mute > 0 else None
        ref_img, ref_illum = eng.images(torch.tensor(bgs[i][None], device=b.device), wav[:sh.nt].contiguous(),
                                        b.unpack_traces(obs, i)[None].contiguous(), vm, 0.1)
        eng.status()
        assert torch.equal(b.unpack_images(img, i), ref_img[0]), i
        assert torch.equal(b.unpack_images(illum, i), ref_illum[0]), i
