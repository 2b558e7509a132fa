"""What the trained network gains over the method without it, at a reduced size (2048 training
models, 1000 AdamW steps of 32, 32 held-out models, 8 full-band L-BFGS iterations, as the full-size
workload runs 50): its proposals are closer to the true models than the medium backgrounds plain FWI
starts from, in model space (normalised MAE) and in data misfit, and FWI from the accepted proposals
ends at a lower misfit than plain FWI.  (The multiscale schedule is checked against the oracle in
tests/test_fwi_gpu.py; at this size its low band leaves the two starts too close to compare.)"""
import pytest

pytestmark = pytest.mark.gpu


def test_trained_proposal_gains_over_plain_fwi():
    from shotsweep_b200 import learned
    res = learned.run(n_train=2048, n_test=32, steps=1000, batch=32, iters=8, log=None)
    assert res['losses'][-1][1] < 0.1
    assert res['mae_proposal'] < 0.5 * res['mae_background']
    assert res['J_proposal'] < res['J_background']
    assert res['accepted'] > 16
    assert res['learned_final_misfit'] < res['plain_final_misfit']
    assert res['mae_learned_fwi'] < res['mae_plain_fwi']


def test_multiscale_learned_side_accounts_for_the_fallback():
    """With several bands, refused proposals run plain FWI over every band first (their time counts), and
    accepted ones go straight to the full band; each group's models end where a run of that group alone
    ends (L-BFGS is per model), and the curve adds the fallback group's final full-band misfit."""
    import numpy as np
    import torch
    from shotsweep_b200 import engine, gpu, learned, synth
    from shotsweep_b200.fwi import BatchFWI
    dev = torch.device('cuda', torch.cuda.current_device())
    eng = gpu.Sim(device=dev).engine
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    truth = torch.tensor(synth.population(6, tag=33), device=dev)
    obs = eng.forward(truth, w)
    bg = torch.tensor(np.stack([np.tile(np.linspace(1800, 3800, 70)[:, None], (1, 70))] * 6), dtype=torch.float32,
                      device=dev)
    prop = (0.7 * truth + 0.3 * bg).contiguous()
    use = np.array([True, False, True, True, False, True])
    bands, iters = (8.0, None), (2, 2)
    v, curve = learned.learned_multiscale(eng, w, obs, prop, bg, use, bands, iters, propose_s=0.5)
    rej = torch.tensor(np.flatnonzero(~use), device=dev)
    acc = torch.tensor(np.flatnonzero(use), device=dev)
    v_r, h_r = BatchFWI(eng, w, obs[rej].contiguous()).run_bands(bg[rej].contiguous(), gpu.RICKER, bands, iters)
    v_a, h_a = BatchFWI(eng, w, obs[acc].contiguous()).run_bands(prop[acc].contiguous(), gpu.RICKER, (None,), (4,))
    assert torch.equal(v[rej], v_r) and torch.equal(v[acc], v_a)
    assert len(curve) == len(h_a) and curve[0][0] >= 0.5 + h_r[-1][0] * 0.5
    j_rej = float(h_r[-1][1].sum())
    for (t, j), h in zip(curve, h_a):
        assert abs(j - (j_rej + float(h[1].sum()))) <= 1e-6 * j
    assert all(t1 >= t0 for (t0, _), (t1, _) in zip(curve, curve[1:]))
