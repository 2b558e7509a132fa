"""What the trained network gains over the method without it, at a reduced size (2048 training
models, 600 AdamW steps of 32, 32 held-out models, 8 full-band L-BFGS iterations, as the full-size
workload runs 50): its proposals are closer to the true models than the medium backgrounds plain FWI
starts from, in model space (normalised MAE) and in data misfit, and FWI from the accepted proposals
ends at a lower misfit than plain FWI.  (The multiscale schedule is checked against the oracle in
tests/test_fwi_gpu.py; at this size its low band leaves the two starts too close to compare.)"""
import pytest

pytestmark = pytest.mark.gpu


def test_trained_proposal_gains_over_plain_fwi():
    from shotsweep_b200 import learned
    res = learned.run(n_train=2048, n_test=32, steps=600, batch=32, iters=8, log=None)
    assert res['losses'][-1][1] < 0.1
    assert res['mae_proposal'] < 0.5 * res['mae_background']
    assert res['J_proposal'] < res['J_background']
    assert res['accepted'] > 16
    assert res['learned_final_misfit'] < res['plain_final_misfit']
    assert res['mae_learned_fwi'] < res['mae_plain_fwi']
