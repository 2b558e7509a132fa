"""Batched L-BFGS FWI on the GPU against the NumPy restatement of the reference's iteration
(archive/toy/slopes/fwi.py:130-164).  Kernel checks use random data: directions, g.d and the
preconditioner within 1e-5 (float32 vectors, float64 dot products on both sides).  The whole loop
runs two iterations on one model against the float64 oracle simulator: misfits within 2e-4 and the
model within 2e-3 of the update (the float32 simulator's gradient differs from the float64 one by about
1e-4, which the curvature scaling of the second step carries into the update)."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_direction_and_preconditioner_kernels():
    from oracle import fwi_oracle as FO
    from shotsweep_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(0)
    B, n, mem = 7, 4900, 6
    g = rng.standard_normal((B, n)).astype(np.float32)
    S = rng.standard_normal((B, mem, n)).astype(np.float32) * 0.1
    Y = (S + 0.05 * rng.standard_normal((B, mem, n))).astype(np.float32)    # s.y > 0: a positive curvature pair
    count = np.array([0, 1, 2, 3, 6, 6, 4], np.int32)
    nxt = np.array([0, 1, 5, 3, 2, 0, 4], np.int32)
    g[6] = -np.abs(g[6])
    Y[6] = -Y[6]                                                           # forces a non-descent direction
    dev = torch.device('cuda')
    # every device array stays referenced until the call has run (a temporary's memory may be reused)
    g_d, S_d, Y_d = (torch.tensor(a, device=dev) for a in (g, S, Y))
    cnt, nxt_d, act = (torch.tensor(a, device=dev) for a in (count, nxt, np.ones(B, np.int32)))
    d = torch.empty(B, n, device=dev)
    gd = torch.empty(B, dtype=torch.float64, device=dev)
    _lib.check(L.ss_lbfgs_direction(_lib.ptr(g_d), _lib.ptr(S_d), _lib.ptr(Y_d), _lib.ptr(cnt), _lib.ptr(nxt_d),
                                    _lib.ptr(act), B, n, mem, 50.0, _lib.ptr(d), _lib.ptr(gd),
                                    _lib.stream_handle(dev)), 'ss_lbfgs_direction')
    torch.cuda.synchronize()
    d, gd, cnt = d.cpu().numpy(), gd.cpu().numpy(), cnt.cpu().numpy()
    for m in range(B):
        slots = [(nxt[m] - count[m] + j) % mem for j in range(count[m])]
        ref, ref_gd, keep = FO.direction(g[m].astype(np.float64), [S[m, s].astype(np.float64) for s in slots],
                                         [Y[m, s].astype(np.float64) for s in slots])
        assert np.abs(d[m] - ref).max() <= 1e-5 * np.abs(ref).max(), m
        assert abs(gd[m] - ref_gd) <= 1e-5 * abs(ref_gd), m
        assert (cnt[m] == count[m]) == keep or (count[m] == 0 and cnt[m] == 0), m
    grads = rng.standard_normal((3, 5, 70, 70)).astype(np.float32)
    out = torch.empty(3, 70, 70, device=dev)
    grads_d = torch.tensor(grads, device=dev)
    _lib.check(L.ss_fwi_precondition(_lib.ptr(grads_d), 3, 5, 70, 70, 2.0, _lib.ptr(out), _lib.stream_handle(dev)),
               'ss_fwi_precondition')
    for m in range(3):
        ref = FO.precondition(grads[m].sum(0).astype(np.float64), 2.0)
        assert np.abs(out[m].cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()


def test_fwi_loop_matches_oracle_two_iterations():
    from oracle import fwi_oracle as FO
    from oracle import oracle as O
    from shotsweep_b200 import engine, gpu, synth
    from shotsweep_b200.fwi import BatchFWI
    truth = synth.model('layered', [77, 0])
    v0 = np.tile(np.linspace(1800, 3600, 70)[:, None], (1, 70))
    sim = gpu.Sim(device='cuda')
    eng = sim.engine
    w = engine.scaled_wavelet(gpu.RICKER, eng.device)
    obs = eng.forward(torch.tensor(truth[None], device=eng.device), w)
    fwi = BatchFWI(eng, w, obs)
    v, hist = fwi.run(torch.tensor(v0[None], dtype=torch.float32, device=eng.device), iters=2)
    ref_v, ref_J = FO.fwi(O.OracleSim(checkpoint_interval=100), obs[0].cpu().numpy().astype(np.float64), v0, 2)
    got_J = [h[1][0] for h in hist]
    assert len(ref_J) == 3
    np.testing.assert_allclose(got_J, ref_J, rtol=2e-4)
    step = np.abs(ref_v - v0).max()                      # the size of the two updates (about 100 m/s)
    assert np.abs(v[0].cpu().numpy() - ref_v).max() <= 2e-3 * step
    assert got_J[-1] < got_J[0]


def test_per_model_wavelets_equal_single_model_runs():
    """One wavelet per model in one launch: each model's gathers and gradient equal its own run, bit for bit."""
    from oracle import oracle as O
    from shotsweep_b200 import engine, gpu, synth
    from shotsweep_b200.fwi import scaled
    eng = gpu.Sim(device='cuda').engine
    dev = eng.device
    models = torch.tensor(np.stack([synth.model(f, [91, i]) for i, f in enumerate(('layered', 'curved', 'faulted'))]),
                          dtype=torch.float32, device=dev)
    rick = [O.ricker(1000, f0=f0) for f0 in (15.0, 11.0, 19.0)]
    wav = torch.stack([scaled(r) for r in rick]).to(dev)
    obs = eng.forward(models, scaled(rick[0]).to(dev))
    bg = torch.tensor(np.tile(np.linspace(1700, 3500, 70, dtype=np.float32)[:, None], (3, 1, 70)), device=dev)
    got = eng.forward(models, wav)
    g_all, il_all = eng.gradient(bg, wav, obs)
    eng.status()
    for i in range(3):
        ref = eng.forward(models[i:i + 1].contiguous(), wav[i].contiguous())
        g, il = eng.gradient(bg[i:i + 1].contiguous(), wav[i].contiguous(), obs[i:i + 1].contiguous())
        eng.status()
        assert torch.equal(got[i], ref[0]), i
        assert torch.equal(g_all[i], g[0]) and torch.equal(il_all[i], il[0]), i
    with pytest.raises(ValueError, match='wavelet'):
        eng.forward(models, wav[:2].contiguous())


def test_band_loop_matches_oracle():
    """Two bands (8 Hz low-pass, then full), one iteration each, on one model: the estimated wavelets, the
    misfits and the model against the float64 restatement of the reference's multiscale loop."""
    from oracle import fwi_oracle as FO
    from oracle import oracle as O
    from shotsweep_b200 import engine, gpu, synth
    from shotsweep_b200.fwi import BatchFWI
    truth = synth.model('curved', [78, 0])
    v0 = np.tile(np.linspace(1800, 3600, 70)[:, None], (1, 70))
    eng = gpu.Sim(device='cuda').engine
    w = engine.scaled_wavelet(gpu.RICKER, eng.device)
    obs = eng.forward(torch.tensor(truth[None], device=eng.device), w)
    fwi = BatchFWI(eng, w, obs)
    v, hist = fwi.run_bands(torch.tensor(v0[None], dtype=torch.float32, device=eng.device), gpu.RICKER,
                            iters=(1, 1))
    ref_v, ref_bands = FO.fwi_bands(lambda wav: O.OracleSim(wavelet=wav, checkpoint_interval=100),
                                    obs[0].cpu().numpy().astype(np.float64), v0, gpu.RICKER, iters=(1, 1))
    for k, ref_w, ref_J in ref_bands:
        got_w = fwi.wavelets[k][0].double().cpu().numpy() / 1e3
        assert np.abs(got_w - ref_w).max() <= 1e-4 * np.abs(ref_w).max(), k
        got_J = [h[1][0] for h in hist if h[2] == k]
        np.testing.assert_allclose(got_J, ref_J, rtol=2e-4)
    step = np.abs(ref_v - v0).max()
    assert np.abs(v[0].cpu().numpy() - ref_v).max() <= 2e-3 * step
