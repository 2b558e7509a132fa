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
    """The reference's own bound (tests/test_physics.py:81-83), and a model linear in the rows."""
    from shotsweep_b200 import gpu
    full_history = 24 * 5 * 1000 * 150 * 150 * 4
    assert gpu.imaging_memory_bytes(24) < full_history / 5
    assert gpu.imaging_memory_bytes(1) < gpu.imaging_memory_bytes(300)
    for rows in (3, 6, 30, 300):
        assert abs(gpu.imaging_memory_bytes(2 * rows) - 2 * gpu.imaging_memory_bytes(rows)) <= 2


def test_process_budget_formula_batches_many_models():
    """2_process.py:166-171 sizes its batch as budget // imaging_memory_bytes(3 rows): at the default 2 GiB
    that admits at least 15 models, and the scratch of a call on that batch (at most rows*5/10 solves in
    flight, each with its own history) stays inside the budget with the call's row tensors."""
    import ctypes
    from shotsweep_b200 import _lib, engine, gpu
    L = _lib.load()
    per_model = gpu.imaging_memory_bytes(3)
    max_batch = int(2.0 * 1024 ** 3 // per_model)
    assert max_batch >= 15
    rows = 3 * max_batch
    slots = gpu.max_solves_in_flight(rows)
    g = engine.geometry()
    ws = L.ss_workspace_bytes_slots(ctypes.byref(g), _lib.MODE_IMAGES, slots)
    row_tensors = rows * (5 * (1000 * 70 + 2 * 70 * 70) + 70 * 70) * 4
    assert ws + row_tensors <= max_batch * per_model <= 2.0 * 1024 ** 3
    assert 20 <= slots <= 45


def test_workspace_per_slot_is_linear(lib):
    """ss_workspace_bytes_slots needs no device and grows by one solve's scratch per slot."""
    import ctypes
    from shotsweep_b200 import _lib, engine
    g = engine.geometry()
    sizes = [lib.ss_workspace_bytes_slots(ctypes.byref(g), _lib.MODE_IMAGES, k) for k in (1, 2, 3, 45)]
    step = sizes[1] - sizes[0]
    assert abs(sizes[2] - sizes[1] - step) <= 1024 and abs(sizes[3] - sizes[0] - 44 * step) <= 44 * 1024
    assert sizes == sorted(sizes)                  # (regions are 256-byte aligned, so steps differ by bytes)
    assert 88e6 < step < 90e6                      # 1000 steps x 150 rows x 148 columns x 4 bytes, + rows
    assert lib.ss_workspace_bytes_slots(ctypes.byref(g), _lib.MODE_IMAGES, 0) == 0
    assert lib.ss_workspace_bytes_slots(ctypes.byref(g), _lib.MODE_FORWARD, 45) == 256


def test_workspace_size_gives_back_its_solves_in_flight(lib):
    """A workspace sized for k solves runs k at once, one byte less runs k - 1 (the regions' 256-byte
    alignment makes the growth per solve uneven, so this is exact arithmetic, not a division)."""
    import ctypes
    from shotsweep_b200 import _lib, engine
    for g in (engine.geometry(), engine.geometry(23, 37, 160, 9, (0, 18, 36))):
        for mode in (_lib.MODE_GRADIENT, _lib.MODE_IMAGES):
            for k in (1, 2, 3, 7, 44, 45, 46, 200, 4096):
                b = lib.ss_workspace_bytes_slots(ctypes.byref(g), mode, k)
                assert lib.ss_workspace_slots(ctypes.byref(g), mode, b) == k
                assert lib.ss_workspace_slots(ctypes.byref(g), mode, b - 1) == k - 1


def test_host_pipeline_chunks_cover_rows_in_whole_rounds():
    """The host-observation pipeline's chunks: contiguous, covering every row once, whole rounds of the
    persistent clusters except the last, growing x6 from one round, capped at a third of the rows and 1 GiB."""
    from shotsweep_b200 import engine
    eng = engine.Engine.__new__(engine.Engine)          # host logic only: no device
    eng.g = engine.geometry()
    eng.plan = lambda n_models, mode: {'slots': 45}
    per_round = 9                                        # 45 clusters / 5 shots
    for B in (1, 8, 9, 10, 48, 100, 1500, 20000):
        ch = eng._chunks(B)
        assert ch[0][0] == 0 and ch[-1][1] == B
        assert all(a2 == b1 for (_, b1), (a2, _) in zip(ch, ch[1:])) and all(b > a for a, b in ch)
        assert all((b - a) % per_round == 0 for a, b in ch[:-1])
        assert max(b - a for a, b in ch) * 5 * 1000 * 70 * 4 <= max(1 << 30, per_round * 5 * 1000 * 70 * 4)
    assert [(b - a) // per_round for a, b in eng._chunks(1500)][:4] == [1, 6, 36, 56]
    assert eng._chunks(100, chunk_rows=30) == [(0, 30), (30, 60), (60, 90), (90, 100)]


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors have the sizes and field offsets that a C compiler gives the header's structs."""
    import ctypes
    import shutil
    import subprocess
    from shotsweep_b200 import _lib
    cc = shutil.which('gcc') or shutil.which('cc')
    if cc is None:
        pytest.skip('no C compiler')
    structs = {'ss_geometry': _lib.Geometry, 'ss_batch_item': _lib.BatchItem, 'ss_physics': _lib.Physics,
               'ss_batch_class_info': _lib.BatchClassInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "shotsweep.h"', 'int main(void) {']
    expect = []
    for cname, py in structs.items():
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        expect.append(ctypes.sizeof(py))
        for fname, _ in py._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append(getattr(py, fname).offset)
    lines += ['  return 0;', '}']
    src = tmp_path / 'layout.c'
    src.write_text('\n'.join(lines))
    exe = tmp_path / 'layout'
    subprocess.run([cc, '-std=c99', f'-I{ROOT / "include"}', str(src), '-o', str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect


def test_batch_size_class_and_plan_validation_without_gpu(lib):
    """The size class of a model is host arithmetic; plans reject bad items before touching a device."""
    import ctypes
    from shotsweep_b200 import _lib
    from shotsweep_b200.batch import Shape, make_items, physics
    items, _ = make_items([Shape(70, 70, 1000, [0, 17, 34, 52, 69])])
    assert lib.ss_batch_min_cluster(items, _lib.MODE_IMAGES) == 3      # 150 x 150 padded: three 50-row bands
    items, _ = make_items([Shape(100, 300, 90, [0, 150, 299])])
    assert lib.ss_batch_min_cluster(items, _lib.MODE_IMAGES) == 9      # 95 column groups: 20-row bands
    items, _ = make_items([Shape(20, 20, 50, [3], pad=5, src_row=20)])
    assert lib.ss_batch_min_cluster(items, _lib.MODE_IMAGES) == _lib.ERR_INVALID
    pb, wb = ctypes.c_size_t(0), ctypes.c_size_t(0)
    rc = lib.ss_batch_plan(ctypes.byref(physics()), _lib.MODE_IMAGES, items, 1, None, 1, None, ctypes.byref(pb),
                           ctypes.byref(wb))
    assert rc == _lib.ERR_INVALID and b'src_row' in lib.ss_last_error()
    rc = lib.ss_batch_plan(ctypes.byref(physics()), 7, items, 1, None, 1, None, ctypes.byref(pb), ctypes.byref(wb))
    assert rc == _lib.ERR_INVALID and b'mode' in lib.ss_last_error()
