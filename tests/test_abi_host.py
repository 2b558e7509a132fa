"""CPU-only checks: the C ABI library loads and exports what include/shotsweep.h declares,
and the host-side layer mirrors the reference's argument checks and errors."""
import re
from pathlib import Path
from unittest import mock

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope='module')
def lib():
    from shotsweep_b200 import _lib, build
    build.build()
    return _lib.load()


def header_symbols():
    text = (ROOT / 'include' / 'shotsweep.h').read_text()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(ss_[a-z0-9_]+)\s*\(', text)))


def test_library_exports_every_declared_symbol(lib):
    from shotsweep_b200 import _lib
    declared = header_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(_lib.exported_symbols()) == declared


def test_version_and_error_string_without_gpu(lib):
    assert b'sm_100a' in lib.ss_version()
    assert lib.ss_last_error() is not None


def test_invalid_geometry_rejected_before_any_device_work(lib):
    import ctypes
    from shotsweep_b200 import _lib
    g = _lib.make_geometry(70, 70, 1000, 1, (0, 17))      # pad < 2
    rc = lib.ss_forward(ctypes.byref(g), 1, None, None, None, None, 0, None, 0, None)
    assert rc == _lib.ERR_INVALID
    assert b'pad' in lib.ss_last_error()
    g = _lib.make_geometry(70, 70, 1000, 40, (0, 70))     # shot outside the model
    assert lib.ss_gradient(ctypes.byref(g), 1, None, None, None, None, 0.12, None, None, None, 0, None) == _lib.ERR_INVALID
    with pytest.raises(ValueError):
        _lib.make_geometry(70, 70, 1000, 40, tuple(range(17)))


def test_sim_argument_checks_match_reference():
    from shotsweep_b200 import gpu
    with pytest.raises(ValueError, match='pad must be'):
        gpu.Sim(pad=1)
    with pytest.raises(ValueError, match='checkpoint_interval'):
        gpu.Sim(checkpoint_interval=0)
    with pytest.raises(ValueError, match='wavelet'):
        gpu.Sim(wavelet=np.zeros(1000))
    with pytest.raises(ValueError, match='wavelet'):
        gpu.Sim(wavelet=np.ones(999))
    with pytest.raises(ValueError, match='float32'):
        gpu.Sim(dtype=torch.float64)
    assert gpu.SRC == [0, 17, 34, 52, 69]
    assert gpu.RICKER.shape == (1000,)
    assert gpu.torch is torch


def test_explicit_unavailable_device_fails():
    from shotsweep_b200 import gpu
    with mock.patch.object(torch.cuda, 'is_available', return_value=False):
        with pytest.raises(RuntimeError, match='CUDA was requested'):
            gpu.resolve_device('cuda')
    with pytest.raises(ValueError):
        gpu.resolve_device('xla')


@pytest.mark.skipif(torch.cuda.is_available(), reason='checks the no-GPU failure mode')
def test_no_cpu_fallback():
    from shotsweep_b200 import gpu
    sim = gpu.Sim(device='cpu')
    with pytest.raises(RuntimeError, match='CUDA'):
        sim.gathers(np.full((1, 70, 70), 2000.0))
    with pytest.raises(RuntimeError, match='CUDA'):
        gpu.lap(torch.zeros(3, 9, 9))


def test_velocity_validation_happens_on_host():
    from shotsweep_b200 import gpu
    with pytest.raises(ValueError, match='velocities'):
        gpu.Sim._velocity(np.full((1, 70, 69), 2000.0))
    with pytest.raises(ValueError, match='velocities'):
        gpu.Sim._velocity(np.full((1, 70, 70), np.nan))


def test_memory_model_is_bounded():
    from shotsweep_b200 import gpu
    full_history = 24 * 5 * 1000 * 150 * 150 * 4
    assert gpu.imaging_memory_bytes(24) < full_history         # history is shared by solves in flight
    assert gpu.imaging_memory_bytes(1) < gpu.imaging_memory_bytes(300)
