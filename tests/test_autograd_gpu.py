"""Differentiation: gathers(v) as a torch.autograd.Function with sqrt(nt) checkpoints and segment recompute.

Checks, with J = 0.5 * sum (F(v) - obs)^2 (the unmuted misfit of Sim.gradient):
  * the autograd gradient equals the fused gradient kernel's (summed over shots),
  * it matches the reference's own float64 gradient (golden vectors),
  * it does not depend on the checkpoint interval (tests/test_physics.py:76-79 in the reference),
  * directional derivatives match central finite differences of the reference's float64
    loss along the reference test's five directions (tests/test_physics.py:41-74), epsilon
    0.1 m/s, relative 1e-4 (the reference's own bar), for the fused and the autograd gradient.
"""
import numpy as np
import pytest
import torch

from .conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope='module')
def fd_case():
    return golden('fd_small')


def test_autograd_matches_fused_gradient_and_reference(fd_case):
    from shotsweep_b200 import autograd as AD, engine, gpu
    eng = AD.default_engine()
    dev = eng.device
    v = torch.tensor(fd_case['velocity'], dtype=torch.float32, device=dev)
    obs = torch.tensor(fd_case['observed'], dtype=torch.float32, device=dev)
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    J, g = AD.misfit_gradient(v, obs, eng, w)
    assert g.shape == v.shape and torch.isfinite(g).all()
    fused, _ = eng.gradient(v, w, obs)
    assert rel(g.cpu().numpy(), fused.sum(1).cpu().numpy()) <= 1e-4
    assert rel(g.cpu().numpy(), fd_case['grad'].sum(1)) <= 2e-4


def test_checkpoint_interval_invariance():
    from shotsweep_b200 import autograd as AD, engine, gpu, synth
    eng = AD.default_engine()
    dev = eng.device
    truth = torch.tensor(synth.population(4)[:2], dtype=torch.float32, device=dev)
    v = torch.tensor(np.stack([np.tile(np.linspace(1700, 3400, 70)[:, None], (1, 70))] * 2), dtype=torch.float32,
                     device=dev)
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    obs = eng.forward(truth, w)
    grads = [AD.misfit_gradient(v, obs, eng, w, interval)[1].cpu().numpy() for interval in (32, 73, 1000)]
    assert rel(grads[1], grads[0]) <= 1e-5
    assert rel(grads[2], grads[0]) <= 1e-5


def _directional(g, loc):
    d = np.zeros((70, 70))
    d[loc] = 1.0
    return float(np.sum(np.asarray(g, np.float64).reshape(70, 70) * d))


def test_directional_derivatives_match_reference_finite_differences():
    """The reference test's five directions (tests/test_physics.py:43-61) at its own bar: central differences
    of the reference's float64 loss with epsilon = 0.1 m/s (stored by tests/golden/make_golden.py), against
    the fused Sim.gradient summed over shots and against the autograd (checkpoint + recompute) gradient;
    |fd - adjoint| / max(|fd|, 1) < 1e-4.  The top strip is where edge padding folds onto the source row."""
    from shotsweep_b200 import autograd as AD, engine, gpu
    fx = golden('fd_directions')
    velocity, observed = fx['velocity'], fx['observed']
    fused = gpu.Sim().gradient(velocity, observed)[0].sum(1)[0]
    eng = AD.default_engine()
    dev = eng.device
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    _, g = AD.misfit_gradient(torch.tensor(velocity, dtype=torch.float32, device=dev),
                              torch.tensor(observed, dtype=torch.float32, device=dev), eng, w)
    auto = g.cpu().numpy()[0]
    directions = {
        'interior': (slice(10, 30), 35),
        'left_boundary': (slice(10, 30), 0),
        'bottom_boundary': (69, slice(25, 45)),
        'top_boundary': (0, slice(25, 45)),
        'velocity_dependent_source': (1, 34),
    }
    assert sorted(directions) == sorted(str(n) for n in fx['names'])
    for name, loc in directions.items():
        numerical = float(fx[f'fd_{name}'])
        for label, grad in (('fused', fused), ('autograd', auto)):
            adjoint = _directional(grad, loc)
            assert abs(numerical - adjoint) / max(abs(numerical), 1.0) < 1e-4, (name, label, numerical, adjoint)


def test_muted_directional_derivative_matches_reference_finite_difference():
    """The reference's muted case (tests/test_physics.py:63-74): bottom strip, mute velocity 2000 m/s, mute
    weights fixed; the fused gradient against the reference's float64 central difference, relative 1e-4."""
    from shotsweep_b200 import gpu
    fx = golden('fd_directions')
    grad = gpu.Sim().gradient(fx['velocity'], fx['observed'], v_mute=np.array([2000.0]))[0].sum(1)[0]
    numerical = float(fx['fd_muted_bottom'])
    adjoint = _directional(grad, (69, slice(25, 45)))
    assert abs(numerical - adjoint) / abs(numerical) < 1e-4, (numerical, adjoint)


def test_textured_batch_gradient_and_random_cell_finite_differences():
    """64 textured models from the medium background: the autograd gradient of every model equals the
    fused kernel's, and central differences of the float64 oracle (h = 1e-3 v) on 32 random cells agree.
    Per cell: |fd - adjoint| <= 1e-3 |fd| + 1e-5 max|grad of that model| (the gradient spans five orders
    of magnitude over the grid, so cells near zero are held to the model's scale)."""
    from oracle import oracle as O
    from shotsweep_b200 import autograd as AD, engine, gpu, synth
    eng = AD.default_engine()
    dev = eng.device
    truth_np = np.stack([synth.model('textured', [64, i]) for i in range(64)]).astype(np.float32)
    trend = O.depth_trend(truth_np)
    start_np = np.stack([O.backgrounds(m[0].mean(), trend)[1] for m in truth_np]).astype(np.float32)
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    truth = torch.tensor(truth_np, device=dev)
    start = torch.tensor(start_np, device=dev)
    obs = eng.forward(truth, w)
    _, g = AD.misfit_gradient(start, obs, eng, w)
    fused, _ = eng.gradient(start, w, obs)
    g = g.cpu().numpy().astype(np.float64)
    fused = fused.sum(1).cpu().numpy()
    for b in range(64):
        assert rel(g[b], fused[b]) <= 1e-4, b

    rng = np.random.default_rng(2024)
    models = np.arange(0, 64, 2)
    cells = rng.integers(0, 70, size=(32, 2))
    plus, minus = [], []
    for m, (z, x) in zip(models, cells):
        h = 1e-3 * float(start_np[m, z, x])
        for sign, out in ((1, plus), (-1, minus)):
            vv = start_np[m].astype(np.float64).copy()
            vv[z, x] += sign * h
            out.append(vv)
    osim = O.OracleSim()
    ob = obs.cpu().numpy().astype(np.float64)[models]
    rp = osim.gathers(np.stack(plus)) - ob
    rm = osim.gathers(np.stack(minus)) - ob
    jp = 0.5 * (rp * rp).sum(axis=(1, 2, 3))
    jm = 0.5 * (rm * rm).sum(axis=(1, 2, 3))
    for j, (m, (z, x)) in enumerate(zip(models, cells)):
        h = 1e-3 * float(start_np[m, z, x])
        fd = (jp[j] - jm[j]) / (2 * h)
        adj = g[m, z, x]
        assert abs(fd - adj) <= 1e-3 * abs(fd) + 1e-5 * np.abs(g[m]).max(), (int(m), int(z), int(x), fd, adj)
