"""ss_images_noalloc: RTM images for callers that cannot allocate device memory.

Such callers (a plugin host that passes only input and output buffers, a
framework whose allocator owns all device memory, a service that must not
allocate after start-up) get the same images from a fixed 32 MiB scratch
array inside the library.  This test calls the entry point through the C ABI
twice in a row and compares each result with ss_images (the workspace entry
point), and checks that a geometry too large for the array is refused.
It lives in a file that pytest collects last and needs nothing from the other
tests, so it runs the same alone in a fresh process and after the others.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

IMAGE_TOL = 2e-4     # the tolerance of the parity tests (relative L2 per shot-image)


def per_image_rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1, a.shape[-2] * a.shape[-1])
    b = np.asarray(b, np.float64).reshape(-1, b.shape[-2] * b.shape[-1])
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-30)


def test_noalloc_images_match_workspace_entry_point_twice():
    from oracle import oracle as O
    from shotsweep_b200 import _lib, engine, synth
    nz, nx, nt, pad, cols = 23, 37, 160, 9, (0, 18, 36)
    geom = engine.geometry(nz, nx, nt, pad, cols)
    eng = engine.Engine(geom)
    dev = eng.device
    f32 = dict(dtype=torch.float32, device=dev)
    truth = torch.tensor(np.stack([synth.model('textured', [11, i], nz, nx) for i in range(3)]), **f32)
    bg = torch.tensor(np.stack([np.tile(np.linspace(1700 + 40 * i, 3200, nz)[:, None], (1, nx)) for i in range(3)]),
                      **f32)
    w = engine.scaled_wavelet(O.ricker(nt), dev)
    obs = eng.forward(truth, w)
    vm = torch.tensor([1800.0, 1900.0, 2000.0], **f32)
    t_mute = 0.03
    ref_img, ref_illum, ref_grad = eng.images(bg, w, obs, vm, t_mute, want_grad=True)
    eng.status()

    L = _lib.load()
    for call in range(2):
        img = torch.full_like(ref_img, float('nan'))
        illum = torch.full_like(ref_img, float('nan'))
        grad = torch.full_like(ref_img, float('nan'))
        with torch.cuda.device(dev):
            rc = L.ss_images_noalloc(ctypes.byref(geom), 3, _lib.ptr(bg), _lib.ptr(w), _lib.ptr(obs), _lib.ptr(vm),
                                     t_mute, 1e-4, 1, _lib.ptr(img), _lib.ptr(illum), _lib.ptr(grad),
                                     _lib.stream_handle(dev))
        assert rc == 0, L.ss_last_error()
        for got, ref in ((img, ref_img), (illum, ref_illum), (grad, ref_grad)):
            got, ref = got.cpu().numpy(), ref.cpu().numpy()
            assert np.isfinite(got).all(), f'call {call}: unwritten output'
            assert per_image_rel(got, ref).max() <= IMAGE_TOL, f'call {call}'


def test_noalloc_refuses_geometry_beyond_its_scratch():
    from shotsweep_b200 import _lib, engine
    geom = engine.geometry()                     # 70x70, 1000 steps: about 90 MB of scratch per solve
    dev = torch.device('cuda', torch.cuda.current_device())
    L = _lib.load()
    x = torch.zeros(1, 5, 1000, 70, device=dev)
    v = torch.full((1, 70, 70), 2000.0, device=dev)
    w = torch.zeros(1000, device=dev)
    out = torch.empty(1, 5, 70, 70, device=dev)
    rc = L.ss_images_noalloc(ctypes.byref(geom), 1, _lib.ptr(v), _lib.ptr(w), _lib.ptr(x), None, 0.12, 1e-4, 1,
                             _lib.ptr(out), _lib.ptr(out.clone()), None, _lib.stream_handle(dev))
    assert rc == _lib.ERR_UNSUPPORTED
    assert b'scratch' in L.ss_last_error()


def test_noalloc_refuses_stream_capture():
    """The call ends by waiting for its own work, which a CUDA graph cannot record: on a capturing stream it
    returns SS_ERR_UNSUPPORTED before it enqueues anything, and the capture ends cleanly."""
    from shotsweep_b200 import _lib, engine
    geom = engine.geometry(23, 37, 160, 9, (0, 18, 36))
    dev = torch.device('cuda', torch.cuda.current_device())
    L = _lib.load()
    x = torch.zeros(1, 3, 160, 37, device=dev)
    v = torch.full((1, 23, 37), 2000.0, device=dev)
    w = torch.zeros(160, device=dev)
    img = torch.empty(1, 3, 23, 37, device=dev)
    illum = torch.empty_like(img)
    side = torch.cuda.Stream(dev)
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(side):
        graph.capture_begin()
        try:
            rc = L.ss_images_noalloc(ctypes.byref(geom), 1, _lib.ptr(v), _lib.ptr(w), _lib.ptr(x), None, 0.03, 1e-4,
                                     1, _lib.ptr(img), _lib.ptr(illum), None, ctypes.c_void_p(side.cuda_stream))
        finally:
            graph.capture_end()
    assert rc == _lib.ERR_UNSUPPORTED
    assert b'captured' in L.ss_last_error()
