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
