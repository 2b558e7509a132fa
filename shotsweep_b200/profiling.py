"""Small fixed workloads for profiling with ncu.

    python -m shotsweep_b200.profiling [n_models]
    python -m shotsweep_b200.profiling learned [batch]
    python -m shotsweep_b200.profiling uneven [solves]
    python -m shotsweep_b200.profiling uneven-classes [CxR ...]
    python -m shotsweep_b200.profiling gemm

`uneven-classes` times every size class of the uneven bench workload (2000 solves, full time axes) alone at its
tuned launch shape and at the extra (cluster x rows per thread) shapes given, then the whole batch under each
stream schedule.

The last form times the tensor-core GEMM on square BF16 problems (4096^3, 8192^3; BF16 and F32 outputs)
beside torch.matmul on the same device.

The second form: `batch` simulated models (default 64), three training steps of the learned
proposal (warm-up), then five timed steps; each step launches the network's 38 tensor-core
GEMMs in the same order (13 forward, then per layer from the top the weight gradient and,
below the first layer, the input gradient).

Runs, on cuda:0, with `n_models` seeded synthetic models (default 9, i.e.
45 solves, one round of three-CTA clusters on a B200):
  1. forward of the true models (observed gathers),
  2. images, 3. forward          (warm-up),
  4. forward, 5. images          (the launches to capture: ncu -s 3 -c 2),
and prints their CUDA-event times.
"""
import sys

import numpy as np
import torch

from . import engine, gpu, synth


def main(n_models=9):
    eng = engine.Engine(engine.geometry())
    dev = eng.device
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    vt = torch.tensor(synth.population(max(n_models, 4))[:n_models], dtype=torch.float32, device=dev)
    obs = eng.forward(vt, w)
    bg = torch.tensor(np.stack([np.tile(np.linspace(1600, 3600, 70)[:, None], (1, 70))] * n_models),
                      dtype=torch.float32, device=dev)
    vm = torch.full((n_models,), 1700.0, device=dev)
    eng.images(bg, w, obs, vm)
    eng.forward(vt, w)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    eng.forward(vt, w)
    ev[1].record()
    ev[2].record()
    eng.images(bg, w, obs, vm)
    ev[3].record()
    torch.cuda.synchronize()
    eng.status()
    print(f'models={n_models} solves={5 * n_models} forward {ev[0].elapsed_time(ev[1]):.3f} ms '
          f'images {ev[2].elapsed_time(ev[3]):.3f} ms')


def learned(batch=64):
    from . import train_inputs as TI
    from .proposal import ProposalNet
    eng = engine.Engine(engine.geometry())
    dev = eng.device
    models = synth.population(batch, tag=7)
    g = eng.forward(torch.tensor(models, device=dev), engine.scaled_wavelet(gpu.RICKER, dev))
    stored = TI.stored_gathers(g)
    scale = float(stored.abs().max().item())
    y = TI.targets(torch.tensor(models, device=dev))
    net = ProposalNet(batch, device=dev)
    net.ids.copy_(torch.arange(batch, dtype=torch.int32))
    for _ in range(3):
        net.train_step(stored, scale, y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        net.train_step(stored, scale, y)
    e1.record()
    torch.cuda.synchronize()
    net.check()
    print(f'batch={batch} training step {e0.elapsed_time(e1) / 5:.3f} ms, L1 {net.loss_sum.item() / (batch * 4900):.4f}')


def uneven(n_solves=48):
    """A seeded uneven batch (time axes capped at 600 steps), forward then images twice (the second timed)."""
    import dataclasses
    from .batch import Shape, UnevenBatch
    wl = synth.uneven_workload(n_solves, seed=9)
    shapes, bgs, truths = [], [], []
    for m in wl:
        nz, nx = m['truth'].shape
        for bg in m['backgrounds']:
            shapes.append(Shape(nz, nx, min(m['nt'], 600), m['shot_cols'], v_mute=m['v_s']))
            bgs.append(bg)
            truths.append(m['truth'])
    b = UnevenBatch(shapes)
    dev = b.device
    t = np.arange(b.max_nt) * 1e-3
    a = (np.pi * 15.0 * (t - 1.2 / 15.0)) ** 2
    w = torch.tensor((1 - 2 * a) * np.exp(-a) * 1e3, dtype=torch.float32, device=dev)
    obs = b.forward(b.pack_models(truths), w)
    vb = b.pack_models(bgs)
    b.images(vb, w, obs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.images(vb, w, obs)
    e1.record()
    torch.cuda.synchronize()
    b.status()
    print(f'solves={b.n_solves} classes={[(c["cluster"], c["n_solves"]) for c in b.classes()]} '
          f'images {e0.elapsed_time(e1):.3f} ms')


def uneven_classes(extra=(), n_solves=2000, seed=2):
    """Per-class CUDA-event times of the uneven bench workload (see the module docstring)."""
    from . import autotune
    from .batch import Shape, UnevenBatch
    dev = torch.device('cuda', torch.cuda.current_device())
    shapes = []
    for m in synth.uneven_workload(n_solves, seed=seed):
        nz, nx = m['truth'].shape
        shapes += [Shape(nz, nx, m['nt'], m['shot_cols'], v_mute=m['v_s']) for _ in m['backgrounds']]
    table = autotune.tune(shapes, device=dev)
    total = 0.0
    for c_min, idx in sorted(autotune.class_members(shapes).items()):
        sub = [shapes[i] for i in idx]
        for shape in [table[c_min]] + [s for s in extra if s != table[c_min]]:
            try:
                secs, work = autotune._time_class(sub, shape, c_min, dev, 10 ** 6, 2)
            except RuntimeError:      # the class does not fit this launch shape
                continue
            b = UnevenBatch(sub, device=dev, clusters={c_min: shape}, schedule=0)
            inflight = sum(c['slots'] for c in b.classes())
            del b
            total += secs if shape == table[c_min] else 0.0
            print(f'class {c_min:2d} {"tuned" if shape == table[c_min] else "other"} {shape}: {len(sub)} rows, '
                  f'{sum(s.n_shots for s in sub)} solves, {inflight} in flight, {secs * 1e3:.1f} ms, '
                  f'{work / secs / 1e9:.1f} Gcell-steps/s, {work / secs / 1e9 / (inflight * shape[0]):.2f} per SM',
                  flush=True)
    print(f'sum over classes at the tuned shapes: {total * 1e3:.1f} ms')
    rng = np.random.default_rng(0)
    for sched in UnevenBatch.SCHEDULES:
        b = UnevenBatch(shapes, device=dev, clusters=table, schedule=sched)
        vel = b.pack_models([np.full((s.nz, s.nx), 2500.0, np.float32) for s in shapes])
        obs = b.pack_traces([rng.standard_normal((s.n_shots, s.nt, s.nx)).astype(np.float32) for s in shapes])
        w = torch.zeros(b.max_nt, dtype=torch.float32, device=dev)
        w[:40] = 1.0
        out = (b._empty(b.n_out), b._empty(b.n_out), None)
        b.images(vel, w, obs, out=out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.images(vel, w, obs, out=out)
        e1.record()
        e1.synchronize()
        b.status()
        print(f'whole batch, schedule {sched}: {e0.elapsed_time(e1):.1f} ms')
        del b, vel, obs, out


def gemm():
    from . import _lib
    L = _lib.load()
    dev = torch.device('cuda', torch.cuda.current_device())

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 10

    for n in (4096, 8192):
        A = torch.randn(n, n, device=dev).to(torch.bfloat16)
        B = torch.randn(n, n, device=dev).to(torch.bfloat16)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        for epi, dt in ((_lib.EPI_BIAS_LRELU_BF16, torch.bfloat16), (_lib.EPI_F32, torch.float32)):
            C = torch.empty(n, n, dtype=dt, device=dev)
            ms = timed(lambda: _lib.check(L.ss_gemm_bf16(_lib.ptr(A), n, _lib.ptr(B), n, n, n, n, epi, _lib.ptr(C), n,
                                                         None, 1.0, 1, _lib.ptr(err), _lib.stream_handle(dev)),
                                          'ss_gemm_bf16'))
            print(f'n={n} ss_gemm_bf16 {"bf16" if epi == _lib.EPI_BIAS_LRELU_BF16 else "f32"} out: {ms:.3f} ms, '
                  f'{2 * n ** 3 / ms / 1e9:.0f} TFLOP/s, status {err.item()}')
        ref = torch.empty(n, n, dtype=torch.bfloat16, device=dev)
        ms = timed(lambda: torch.matmul(A, B.T, out=ref))
        print(f'n={n} torch.matmul bf16 out: {ms:.3f} ms, {2 * n ** 3 / ms / 1e9:.0f} TFLOP/s')


if __name__ == '__main__':
    if len(sys.argv) > 1 and sys.argv[1] == 'learned':
        learned(int(sys.argv[2]) if len(sys.argv) > 2 else 64)
    elif len(sys.argv) > 1 and sys.argv[1] == 'gemm':
        gemm()
    elif len(sys.argv) > 1 and sys.argv[1] == 'uneven-classes':
        uneven_classes(tuple(tuple(int(v) for v in a.split('x')) for a in sys.argv[2:]))
    elif len(sys.argv) > 1 and sys.argv[1] == 'uneven':
        uneven(int(sys.argv[2]) if len(sys.argv) > 2 else 48)
    else:
        main(int(sys.argv[1]) if len(sys.argv) > 1 else 9)
