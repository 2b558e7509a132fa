"""Failure detection on the GPU without a fault: a bounded device wait runs out and reports it.

ss_wait_probe runs the simulation kernels' bounded mbarrier wait on a barrier that nothing arrives on.
It must record SS_ERR_TIMEOUT after its limit and return, and the context must stay usable: a small
solve afterwards still matches the oracle.  Host-side failures (bad shapes, non-finite or non-positive
inputs) are covered by the parity and ABI tests.
"""
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_the_context_stays_usable():
    from oracle import oracle as O
    from shotsweep_b200 import _lib, engine
    L = _lib.load()
    dev = torch.device('cuda', torch.cuda.current_device())
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _lib.check(L.ss_wait_probe(_lib.ptr(status), 50.0, _lib.stream_handle(dev)), 'ss_wait_probe')
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert status.item() == _lib.ERR_TIMEOUT
    assert 0.05 <= elapsed < 5.0
    # the same context still computes correctly
    nz, nx, nt, pad, cols = 17, 29, 120, 6, (3, 25)
    geom = O.Geometry(nz=nz, nx=nx, nt=nt, shot_cols=cols)
    v = np.tile(np.linspace(1800, 2600, nz)[:, None], (1, nx))[None]
    ref = O.OracleSim(wavelet=O.ricker(nt), pad=pad, geom=geom).gathers(v)
    eng = engine.Engine(engine.geometry(nz, nx, nt, pad, cols), dev)
    got = eng.forward(torch.tensor(v, dtype=torch.float32, device=dev), engine.scaled_wavelet(O.ricker(nt), dev))
    eng.status()
    got = got.cpu().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-5
