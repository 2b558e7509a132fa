"""CPU checks of the multiscale FWI's host-side signal steps (no GPU): the Gaussian low-pass and the
per-model Wiener wavelet estimate of shotsweep_b200.fwi against the NumPy restatement of the
reference's lowpass / estimate_source (archive/toy/slopes/fwi.py:78-90).  Both run float64 FFTs, so
they agree to rounding (1e-12 relative)."""
import numpy as np
import torch


def test_lowpass_matches_restatement():
    from oracle import fwi_oracle as FO
    from oracle import oracle as O
    from shotsweep_b200 import fwi
    rng = np.random.default_rng(4)
    x = rng.standard_normal((2, 3, 1000, 7)).astype(np.float32)
    for fc in (4.0, 8.0, None):
        got = fwi.lowpass(torch.tensor(x), fc).numpy()
        ref = np.stack([FO.lowpass(x[i].astype(np.float64), fc) for i in range(2)]).astype(np.float32)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-6 * np.abs(ref).max())
    ric = O.ricker()
    np.testing.assert_allclose(fwi.lowpass(ric, 8.0), FO.lowpass(ric[None, :, None], 8.0)[0, :, 0], rtol=1e-12,
                               atol=1e-14)
    assert fwi.lowpass(ric, None) is ric


def test_wavelet_estimate_per_model_matches_restatement():
    from oracle import fwi_oracle as FO
    from oracle import oracle as O
    from shotsweep_b200 import fwi
    rng = np.random.default_rng(5)
    ric = O.ricker()
    sim = rng.standard_normal((3, 2, 1000, 6))
    obs = sim * np.array([0.5, 1.5, -2.0])[:, None, None, None] + 0.1 * rng.standard_normal(sim.shape)
    got = fwi.estimate_wavelets(torch.tensor(sim), torch.tensor(obs), ric).numpy()
    for m in range(3):
        ref = FO.estimate_source(sim[m], obs[m], ric)
        assert np.abs(got[m] - ref).max() <= 1e-12 * np.abs(ref).max()
    w = fwi.scaled(torch.tensor(got))
    assert w.dtype == torch.float32 and w.is_contiguous()
    np.testing.assert_array_equal(w.numpy(), (got * 1e3).astype(np.float32))
