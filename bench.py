#!/usr/bin/env python
"""RTM shot-image throughput of the B200 path, one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step"): 500 seeded OpenFWI-shaped synthetic velocity models
(equal mix of layered / curved / faulted / textured families) x 3 laterally
constant backgrounds (surface velocity + 0.6 / 1.0 / 1.4 x the population's
mean depth trend) x 5 shots = 7500 shot-images, each one forward + one exact
adjoint solve of 1000 steps on the 150x150 padded grid plus the image
epilogue, in one kernel launch.  Observed gathers are simulated from the
true models.  No OpenFWI data exists offline; the synthetic models have its
shapes, spacing and velocity range.

value     shot-images/s with inputs resident in HBM (CUDA events, max over ranks)
e2e       the same metric through gpu.Sim.images with host inputs (pinned gathers),
          host->device and device->host copies inside the timed region
roofline  FP32 CUDA-core throughput: 0.81 GFLOP per shot-image (150^2 cells x
          1000 steps x 36 flops) over the launch time, against an FMA peak
          measured live on this GPU
cpu_baseline  the oracle's float32 restatement of the reference CPU path
          (PyTorch eager, all host threads) on a bounded sample

With torchrun, every rank simulates its own 500 models (weak scaling); the
ranks exchange nothing on the data path.

--workload uneven: the uneven batch instead: 2000 seeded (model, background,
shot) solves on grids of 70-200 x 70-300 cells, 1000-3000 steps, 1-9 shots and
1-3 backgrounds per model, planned into size classes, cluster sizes from the
autotuner, replayed as one CUDA graph per step (shot-images/s and padded
cell-steps/s; no CPU arm, the reference runs one fixed geometry only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = 'RTM shot-images/s (70x70, 1000 steps)'
UNIT = 'shot-images/s'
N_MODELS = 500
RHOS = (0.6, 1.0, 1.4)
FLOP_PER_SHOT_IMAGE = 150 * 150 * 1000 * 36
WORKLOAD = ('RTM images: 500 seeded OpenFWI-shaped synthetic models x 3 backgrounds x 5 shots = 7500 shot-images, '
            '70x70 cells + 40-cell absorbing pad, 1000 steps, one launch')
CPU_BEST_ROWS = 12           # background rows (4 models x 3) per CPU call: the CPU path's best batch
CPU_PROCESS_ROWS = 3         # 2_process's defaults (--batch 1: one model x 3 backgrounds, --threads 2),
CPU_PROCESS_THREADS = 2      # 2_process.py:115,118
TRAFFIC_FILE = ROOT / 'profiles' / 'images_kernel_dram.json'


def parse():
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', choices=('ours', 'reference'), default='ours')
    ap.add_argument('--models', type=int, default=N_MODELS, help='velocity models per GPU')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--workload', choices=('openfwi', 'uneven', 'process', 'learned'), default='openfwi')
    ap.add_argument('--train-models', type=int, default=20000, help='learned workload: training models')
    ap.add_argument('--train-steps', type=int, default=6000, help='learned workload: AdamW steps (batch 64)')
    ap.add_argument('--test-models', type=int, default=256, help='learned workload: held-out models')
    ap.add_argument('--fwi-iters', default='50',
                    help='learned workload: L-BFGS iterations, one count (full band) or two (8 Hz low-pass band, '
                         'then full band, as the reference\'s multiscale FWI with 10,25)')
    ap.add_argument('--solves', type=int, default=2000, help='uneven workload: solves per GPU')
    ap.add_argument('--schedule', type=int, default=-1, choices=(-1, 0, 1, 2),
                    help='uneven workload: stream schedule (-1: autotuned)')
    return ap.parse_args()


def population_slice(start, stop, total):
    """Models [start, stop) of a seeded population of `total` (family mix as synth.population)."""
    from shotsweep_b200 import synth
    return np.stack([synth.model(synth.FAMILIES[i * len(synth.FAMILIES) // total], [1, i]) for i in range(start, stop)])


def backgrounds_for(models, trend):
    """Per model: surface velocity (top-row mean) + rho x trend, clipped, laterally constant (3 rows each)."""
    v_s = models[:, 0, :].astype(np.float64).mean(1)
    rows = [np.tile(np.clip(v + r * trend, 1500.0, 4500.0)[:, None], (1, models.shape[2])) for v in v_s for r in RHOS]
    return np.stack(rows), np.repeat(v_s, len(RHOS))


def depth_trend(models):
    m = np.asarray(models, np.float64)
    return (m.mean(2) - m[:, :1, :].mean(2)).mean(0)


class ClockSampler:
    """nvidia-smi clock / throttle samples every 200 ms while the timed region runs."""
    QUERY = ('index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, bus_id):
        self.bus_id = (bus_id or '').lower()
        self.file = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={self.QUERY}', '--format=csv,noheader,nounits',
                                          '-lms', '200'], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        sm, mx, reasons = [], None, set()
        names = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')
        for line in self.file:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 10:
                continue
            if self.bus_id and self.bus_id not in f[1].lower():
                continue
            try:
                sm.append(float(f[2]))
                mx = float(f[3])
            except ValueError:
                continue
            for name, val in zip(names, f[6:10]):
                if val.lower() == 'active':
                    reasons.add(name)
        os.unlink(self.file.name)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['no samples']}
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': mx, 'reasons': sorted(reasons), 'samples': len(sm)}


def fp32_peak(device):
    """Measured FP32 FMA throughput (TFLOP/s): max of scalar and packed FP32x2 probes over all SMs."""
    import ctypes
    import torch
    from shotsweep_b200 import _lib
    L = _lib.load()
    out = torch.zeros(1, device=device)
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    best = 0.0
    for packed in (0, 1):
        for _ in range(2):
            flops = ctypes.c_double()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.check(L.ss_fp32_probe(_lib.ptr(out), sms * 8, 20000, packed, ctypes.byref(flops),
                                       _lib.stream_handle(device)), 'ss_fp32_probe')
            e1.record()
            torch.cuda.synchronize()
            best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def dram_bytes_per_solve():
    """(bytes, source): DRAM read + write bytes per solve of the images kernel, from one ncu capture of a
    small case (one round of solves) recorded in a committed data file, or (None, reason)."""
    try:
        rec = json.loads(TRAFFIC_FILE.read_text())
        return float(rec['dram_bytes_per_solve']), rec.get('capture', '')
    except (OSError, ValueError, KeyError):
        return None, 'no traffic record'


def cpu_model():
    try:
        with open('/proc/cpuinfo') as f:
            for line in f:
                if line.startswith('model name'):
                    return line.split(':', 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or 'unknown'


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_port_rate(obs_rows, bgs, vm, rows, threads, repeats=3):
    """shot-images/s of the oracle's float32 CPU restatement of Sim.images on `rows` background rows."""
    import torch
    from oracle import oracle as O
    torch.set_num_threads(threads)
    sim = O.OracleSim(dtype=torch.float32)
    sim.images(bgs[:1], obs_rows[:1], v_mute=vm[:1])            # warm-up (allocator, threads)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        sim.images(bgs[:rows], obs_rows[:rows], v_mute=vm[:rows])
        times.append(time.perf_counter() - t0)
    return rows * 5 / statistics.median(times)


def run_reference(args):
    """CPU arm: the oracle port of the reference path on the host cores, rank 0 only."""
    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return 0
    import torch
    from oracle import oracle as O
    threads = host_threads()
    torch.set_num_threads(threads)
    rows = CPU_BEST_ROWS
    models = population_slice(0, rows // len(RHOS), N_MODELS)
    trend = depth_trend(population_slice(0, N_MODELS, N_MODELS))
    bgs, vm = backgrounds_for(models, trend)
    osim = O.OracleSim(dtype=torch.float32)
    obs = np.repeat(osim.gathers(models.astype(np.float64)), len(RHOS), 0)
    for _ in range(args.warmup):
        osim.images(bgs[:rows], obs[:rows], v_mute=vm[:rows])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        osim.images(bgs[:rows], obs[:rows], v_mute=vm[:rows])
    elapsed = time.perf_counter() - t0
    value = rows * 5 * args.steps / elapsed
    sample = (f'{rows} background rows (the first {rows // len(RHOS)} models x 3 backgrounds) x 5 shots = '
              f'{rows * 5} shot-images per step from the same workload, float32 PyTorch eager on {threads} host '
              f'threads ({cpu_model()})')
    print(json.dumps({
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': args.gpus,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': elapsed / args.steps * 1e3,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': WORKLOAD, 'sample': sample},
        'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': threads, 'kind': 'port', 'sample': sample,
                         'cpu_model': cpu_model()},
        'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }), flush=True)
    return 0


def run_ours(args):
    import torch
    from shotsweep_b200 import dist as D
    from shotsweep_b200 import engine, gpu
    rank, world, local = D.init('nccl' if args.gpus > 1 else 'gloo', timeout_s=300)
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    per = args.models
    a, b = D.shard(per * world, rank, world)
    models = population_slice(a, b, per * world) if world > 1 else population_slice(0, per, per)
    trend = depth_trend(population_slice(0, N_MODELS, N_MODELS))
    bgs, vm = backgrounds_for(models, trend)
    n_rows = len(bgs)
    shot_images = n_rows * 5

    sim = gpu.Sim(device=dev)
    eng = sim.engine
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    obs_models = eng.forward(torch.tensor(models, dtype=torch.float32, device=dev), w)
    obs = obs_models.repeat_interleave(len(RHOS), dim=0).contiguous()
    del obs_models
    bg_d = torch.tensor(bgs, dtype=torch.float32, device=dev)
    vm_d = torch.tensor(vm, dtype=torch.float32, device=dev)
    img = torch.empty(n_rows, 5, 70, 70, dtype=torch.float32, device=dev)
    illum = torch.empty_like(img)

    def eager():
        eng.images(bg_d, w, obs, vm_d, out=(img, illum))

    for _ in range(args.warmup):
        eager()
    torch.cuda.synchronize()
    eng.status()
    # the timed step: the persistent launch replayed as a captured CUDA graph
    graph = torch.cuda.CUDAGraph()
    try:
        with torch.cuda.graph(graph):
            eager()
        graph.replay()
        torch.cuda.synchronize()
        eng.status()
        step, captured = graph.replay, True
    except RuntimeError as error:
        print(f'graph capture unavailable ({error}); timing eager launches', file=sys.stderr)
        step, captured = eager, False
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    props = torch.cuda.get_device_properties(dev)
    bus = None
    if hasattr(props, 'pci_bus_id'):
        bus = f'{getattr(props, "pci_domain_id", 0):08X}:{props.pci_bus_id:02X}:{getattr(props, "pci_device_id", 0):02X}.0'
    D.barrier()
    torch.cuda.synchronize()
    with ClockSampler(bus) as clk:
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        t_all0.record()
        for e0, e1 in events:
            e0.record()
            step()
            e1.record()
        t_all1.record()
        torch.cuda.synchronize()
    D.barrier()
    eng.status()
    elapsed_ms = D.reduce(t_all0.elapsed_time(t_all1), 'max', dev if world > 1 else None)
    launch_ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in events)
    value = world * shot_images * args.steps / (elapsed_ms * 1e-3)
    clocks = clk.summary()

    # end to end through the public API: pinned host gathers in, numpy images out
    obs_host = obs.cpu().pin_memory()
    h2d = obs_host.numel() * 4 + bgs.size * 8 + vm.size * 8
    d2h = img.numel() * 4 * 2
    sim.images(bgs, obs_host, v_mute=vm)
    e2e_steps = max(1, min(args.steps, 10))
    D.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.images(bgs, obs_host, v_mute=vm)
    e2e_s = D.reduce(time.perf_counter() - t0, 'max', dev if world > 1 else None)
    e2e = world * shot_images * e2e_steps / e2e_s
    # the same call with pageable NumPy gathers (what the reference's callers pass); the first call
    # allocates the pinned staging buffers (the host allocator keeps them for later calls)
    obs_np = obs_host.numpy().copy()
    del obs_host
    sim.images(bgs, obs_np, v_mute=vm)
    D.barrier()
    t0 = time.perf_counter()
    for _ in range(2):
        sim.images(bgs, obs_np, v_mute=vm)
    e2e_np = world * shot_images * 2 / D.reduce(time.perf_counter() - t0, 'max', dev if world > 1 else None)
    # driven as 2_process drives it (2_process.py:166-204): models in batches of
    # budget // imaging_memory_bytes(3) at the default 2 GiB, float64 NumPy gathers repeated per background
    per_call = int(2.0 * 1024 ** 3 // gpu.imaging_memory_bytes(len(RHOS)))
    obs_models = obs_np[::len(RHOS)].astype(np.float64)
    del obs_np
    sim.images(bgs[:per_call * len(RHOS)], np.repeat(obs_models[:per_call], len(RHOS), 0),
               v_mute=vm[:per_call * len(RHOS)])
    D.barrier()
    t0 = time.perf_counter()
    for i in range(0, per, per_call):
        j = min(per, i + per_call)
        sim.images(bgs[i * len(RHOS):j * len(RHOS)], np.repeat(obs_models[i:j], len(RHOS), 0),
                   v_mute=vm[i * len(RHOS):j * len(RHOS)])
    e2e_proc = world * shot_images / D.reduce(time.perf_counter() - t0, 'max', dev if world > 1 else None)
    del obs_models

    peak = fp32_peak(dev)
    achieved = FLOP_PER_SHOT_IMAGE * shot_images / (launch_ms * 1e-3) / 1e12
    per_solve, traffic_src = dram_bytes_per_solve()
    roofline = {'bound': 'fp32', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s', 'frac': achieved / peak,
                'traffic': per_solve * shot_images if per_solve else None,
                'peak_source': 'measured live: max of scalar FFMA and packed FFMA2 probes on all SMs '
                               '(the measured HBM and BF16 peaks carry no FP32 figure)',
                'algorithmic': '36 flops per padded cell per step (16 forward + 20 adjoint), 150^2 cells, 1000 steps; '
                               'traffic = ncu dram read + write bytes per solve x solves',
                'traffic_source': traffic_src,
                'hbm_gbs_of_traffic': per_solve * shot_images / (launch_ms * 1e-3) / 1e9 if per_solve else None}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import torch as _t
        threads = host_threads()
        rows = CPU_BEST_ROWS
        obs_rows = obs[:rows].cpu().double().numpy()
        rate = cpu_port_rate(obs_rows, bgs, vm, rows, threads)
        rate_proc = cpu_port_rate(obs_rows, bgs, vm, CPU_PROCESS_ROWS, CPU_PROCESS_THREADS)
        _t.set_num_threads(threads)
        cpu = {'value': rate, 'unit': UNIT, 'cores': threads, 'kind': 'port', 'cpu_model': cpu_model(),
               'sample': f'{rows} background rows (4 models x 3 backgrounds) x 5 shots of the same workload, median '
                         f'of 3 calls: the oracle\'s float32 PyTorch-eager restatement of Sim.images on {threads} '
                         f'host threads',
               'process_defaults': {'value': rate_proc, 'unit': UNIT, 'cores': CPU_PROCESS_THREADS,
                                    'sample': f'{CPU_PROCESS_ROWS} background rows (one model, 2_process --batch 1) '
                                              f'on {CPU_PROCESS_THREADS} threads (2_process --threads 2)'}}
    if rank == 0:
        print(json.dumps({
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': elapsed_ms / args.steps, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
            'data': 'synthetic: seeded OpenFWI-shaped velocity models, gathers simulated from the true models',
            'config': {'workload': WORKLOAD, 'models_per_gpu': per, 'backgrounds_per_model': len(RHOS),
                       'shots': 5, 'shot_images_per_gpu': shot_images, 'nz': 70, 'nx': 70, 'nt': 1000, 'pad': 40,
                       'parallelism': f'{world} independent ranks (weak scaling, no data-path collective)',
                       'l2': 'inputs larger than L2 (2.1 GB of gathers per step per GPU)',
                       'cuda_graph': captured, 'plan': eng.plan(n_rows, 2)},
            'roofline': roofline, 'cpu_baseline': cpu,
            'e2e': {'value': e2e, 'unit': UNIT, 'h2d_bytes_per_step': int(h2d), 'd2h_bytes_per_step': int(d2h),
                    'api': 'shotsweep_b200.gpu.Sim.images (pinned torch gathers, numpy velocities in; numpy out)',
                    'steps': e2e_steps,
                    'numpy_pageable': {'value': e2e_np, 'unit': UNIT,
                                       'api': 'Sim.images with pageable float32 NumPy gathers (staged per chunk)'},
                    'process_batches': {'value': e2e_proc, 'unit': UNIT, 'models_per_call': per_call,
                                        'api': 'Sim.images on budget // imaging_memory_bytes(3) models per call at '
                                               '2 GiB, float64 NumPy gathers repeated per background, as '
                                               '2_process.py:166-204'}},
            'clocks': clocks, 'gpu_launches': args.steps,
        }), flush=True)
    del graph
    D.finish()
    return 0


def bus_id(dev):
    import torch
    props = torch.cuda.get_device_properties(dev)
    if hasattr(props, 'pci_bus_id'):
        return f'{getattr(props, "pci_domain_id", 0):08X}:{props.pci_bus_id:02X}:{getattr(props, "pci_device_id", 0):02X}.0'
    return None


def run_uneven(args):
    """Uneven batch: forward of the true models, then RTM images of every (model, background) in one graph."""
    import torch
    from shotsweep_b200 import autotune, synth
    from shotsweep_b200 import dist as D
    from shotsweep_b200.batch import Shape, UnevenBatch
    rank, world, local = D.init('nccl' if args.gpus > 1 else 'gloo', timeout_s=600)
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    wl = synth.uneven_workload(args.solves, seed=2 + rank)
    max_nt = max(m['nt'] for m in wl)
    t = np.arange(max_nt) * 1e-3
    a = (np.pi * 15.0 * (t - 1.2 / 15.0)) ** 2
    wav = torch.tensor((1 - 2 * a) * np.exp(-a) * 1e3, dtype=torch.float32, device=dev)
    fb = UnevenBatch([Shape(m['truth'].shape[0], m['truth'].shape[1], m['nt'], m['shot_cols']) for m in wl], device=dev)
    gathers = fb.forward(fb.pack_models([m['truth'] for m in wl]), wav)
    shapes, bgs, obs_parts = [], [], []
    for i, m in enumerate(wl):
        nz, nx = m['truth'].shape
        for bg in m['backgrounds']:
            shapes.append(Shape(nz, nx, m['nt'], m['shot_cols'], v_mute=m['v_s']))
            bgs.append(bg)
            obs_parts.append(fb.unpack_traces(gathers, i).reshape(-1))
    obs = torch.cat(obs_parts).contiguous()
    del obs_parts, gathers
    n_solves = sum(s.n_shots for s in shapes)
    cell_steps = sum(s.cell_steps() for s in shapes)
    table = autotune.tune(shapes, device=dev)
    schedule = autotune.tune_schedule(shapes, table, device=dev) if args.schedule < 0 else args.schedule
    ib = UnevenBatch(shapes, device=dev, clusters=table, schedule=schedule)
    vb = ib.pack_models(bgs)
    graph, img, illum = ib.capture_images(vb, wav, obs)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    ib.status()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    D.barrier()
    torch.cuda.synchronize()
    with ClockSampler(bus_id(dev)) as clk:
        for e0, e1 in events:
            e0.record()
            graph.replay()
            e1.record()
        torch.cuda.synchronize()
    D.barrier()
    ib.status()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in events]
    total_ms = D.reduce(sum(step_ms), 'max', dev if world > 1 else None)
    value = world * n_solves * args.steps / (total_ms * 1e-3)
    # end to end: every step's gathers cross from pinned host memory and its images and illumination come back.
    # Two device buffer sets (two captured graphs over the same plan and workspace) let a copy stream upload
    # step k+1's gathers and download step k-1's images while step k is imaged.
    obs_host = obs.cpu().pin_memory()
    img_host = torch.empty(img.shape, dtype=img.dtype, pin_memory=True)
    illum_host = torch.empty_like(img_host)
    obs2 = torch.empty_like(obs)
    graph2, img2, illum2 = ib.capture_images(vb, wav, obs2)
    sets = ((obs, graph, img, illum), (obs2, graph2, img2, illum2))
    compute, copy = torch.cuda.current_stream(dev), torch.cuda.Stream(dev)
    copied = [torch.cuda.Event() for _ in sets]
    imaged = [torch.cuda.Event() for _ in sets]
    fetched = [torch.cuda.Event() for _ in sets]

    def upload(k):
        o = sets[k % 2][0]
        with torch.cuda.stream(copy):
            if k >= 2:
                copy.wait_event(imaged[k % 2])        # the graph that read this buffer two steps ago is done
            o.copy_(obs_host, non_blocking=True)
            copied[k % 2].record(copy)

    D.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(compute)
    copy.wait_event(e0)
    upload(0)
    for k in range(args.steps):
        _, g_k, img_k, illum_k = sets[k % 2]
        compute.wait_event(copied[k % 2])
        if k >= 2:
            compute.wait_event(fetched[k % 2])        # this set's images of two steps ago have left
        g_k.replay()
        imaged[k % 2].record(compute)
        if k + 1 < args.steps:
            upload(k + 1)
        with torch.cuda.stream(copy):
            copy.wait_event(imaged[k % 2])
            img_host.copy_(img_k, non_blocking=True)
            illum_host.copy_(illum_k, non_blocking=True)
            fetched[k % 2].record(copy)
    compute.wait_stream(copy)
    e1.record(compute)
    torch.cuda.synchronize()
    e2e_ms = D.reduce(e0.elapsed_time(e1), 'max', dev if world > 1 else None)
    e2e = world * n_solves * args.steps / (e2e_ms * 1e-3)
    peak = fp32_peak(dev)
    achieved = cell_steps * 36 / (statistics.mean(step_ms) * 1e-3) / 1e12
    classes = ib.classes()
    if rank == 0:
        print(json.dumps({
            'metric': 'RTM shot-images/s (uneven batch: 70-200 x 70-300 cells, 1000-3000 steps, 1-9 shots)',
            'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': total_ms / args.steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32', 'data': 'synthetic: seeded models of uneven size, gathers simulated from the true models',
            'cell_steps_per_s': world * cell_steps * args.steps / (total_ms * 1e-3),
            'config': {'workload': f'{n_solves} solves per GPU from {len(wl)} models ({len(shapes)} background rows), '
                                   'one CUDA graph per step', 'solves_per_gpu': n_solves,
                       'padded_cell_steps_per_gpu': cell_steps,
                       'l2': f'inputs larger than L2 ({obs.numel() * 4 / 1e9:.1f} GB of gathers per step per GPU)',
                       'autotune': {str(k): v for k, v in sorted(table.items())}, 'schedule': schedule,
                       'classes': [{k: c[k] for k in ('min_cluster', 'cluster', 'rows_per_thread', 'n_solves', 'threads',
                                                      'slots',
                                                      'stream')} for c in classes]},
            'roofline': {'bound': 'fp32', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                         'frac': achieved / peak, 'traffic': None,
                         'algorithmic': '36 flops per padded cell per step (16 forward + 20 adjoint) over every solve'},
            'cpu_baseline': None,
            'e2e': {'value': e2e, 'unit': UNIT, 'h2d_bytes_per_step': obs.numel() * 4,
                    'd2h_bytes_per_step': img.numel() * 8,
                    'api': 'UnevenBatch graph replays with pinned host gathers in, images and illumination out, '
                           'copies of neighbouring steps overlapped with imaging (two buffer sets)'},
            'clocks': clk.summary(), 'gpu_launches': len(classes) * args.steps,
        }), flush=True)
    del graph, graph2
    D.finish()
    return 0


def run_process(args):
    """2_process's per-batch work for the 500-model population: picks, backgrounds, images, float16 cache."""
    import torch
    from oracle import postprocess as PP
    from shotsweep_b200 import background as BG
    from shotsweep_b200 import dist as D
    from shotsweep_b200 import engine, gpu, process
    rank, world, local = D.init('nccl' if args.gpus > 1 else 'gloo', timeout_s=300)
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    per = args.models
    a, b = D.shard(per * world, rank, world)
    # the first `per` models of a seeded pool whose first arrivals the picker accepts (2_process refuses a
    # batch with any rejected model)
    pool = population_slice(2 * a, 2 * b, 2 * per * world)
    trend = depth_trend(population_slice(0, N_MODELS, N_MODELS))
    sim = gpu.Sim(device=dev)
    eng = sim.engine
    pool_g = eng.forward(torch.tensor(pool, dtype=torch.float32, device=dev), engine.scaled_wavelet(gpu.RICKER, dev))
    ok = np.flatnonzero([e.status == 0 for e in BG.surface_estimates(pool_g)])[:per]
    if len(ok) < per:
        raise SystemExit(f'only {len(ok)} of {len(pool)} pool models have usable first arrivals')
    gathers = pool_g[torch.tensor(ok, device=dev)].contiguous()
    del pool_g
    v1 = np.array([e['velocity'] for e in BG.estimate_surface_velocity_batch(gathers)])
    bgs = BG.backgrounds(v1, trend, device=dev).reshape(per * 3, 70, 70)
    img, _ = eng.images(bgs, sim._wavelet(), gathers.repeat_interleave(3, dim=0),
                        torch.tensor(np.repeat(v1, 3), dtype=torch.float32, device=dev))
    times = {'surface': [], 'cache': [], 'batch': []}

    def timed(name, fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        times[name].append(e0.elapsed_time(e1))
        return r

    for step in range(args.warmup + args.steps):
        est = timed('surface', lambda: BG.surface_estimates(gathers))
        cache = timed('cache', lambda: process.image_cache(img.view(per, 3, 5, 70, 70)))
        out = timed('batch', lambda: process.process_batch(sim, gathers, trend))
        if step < args.warmup:
            for k in times:
                times[k].clear()
    eng.status()
    ms = {k: D.reduce(statistics.mean(v), 'max', dev if world > 1 else None) for k, v in times.items()}
    value = world * per / (ms['batch'] * 1e-3)
    # CPU: the NumPy restatement of the picks and the cache on a sample of 20 models, one thread each step
    g_host = gathers[:20].cpu().numpy().astype(np.float64)
    t0 = time.perf_counter()
    for k in range(20):
        try:
            PP.estimate_surface_velocity(g_host[k])
        except ValueError:
            pass
    cpu_surface = 20 / (time.perf_counter() - t0)
    im_host = out['images'][:20].float().cpu().numpy()
    t0 = time.perf_counter()
    PP.image_cache(im_host)
    cpu_cache = 20 / (time.perf_counter() - t0)
    if rank == 0:
        print(json.dumps({
            'metric': '2_process models/s (surface picks + 3 backgrounds + 15 RTM images + float16 cache per model)',
            'value': value, 'unit': 'models/s', 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': ms['batch'], 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32', 'data': 'synthetic: the 500-model OpenFWI-shaped population, gathers simulated',
            'config': {'workload': f'{per} models per GPU per step (the first with usable first arrivals of a '
                                   f'{len(pool)}-model seeded pool)', 'models_per_gpu': per},
            'kernels': {'surface_velocity_models_per_s': per / (ms['surface'] * 1e-3),
                        'image_cache_models_per_s': per / (ms['cache'] * 1e-3)},
            'cpu_baseline': {'surface_velocity_models_per_s': cpu_surface, 'image_cache_models_per_s': cpu_cache,
                             'unit': 'models/s', 'cores': 1, 'kind': 'port',
                             'sample': '20 models, NumPy restatement of background.py:19-83 and 2_process.py:206-210'},
            'gpu_launches': None,
        }), flush=True)
    D.finish()
    return 0


def run_learned(args):
    """Learned proposal + FWI vs plain FWI on held-out models: time-to-misfit (the reference's second metric)."""
    import torch
    from shotsweep_b200 import dist as D
    from shotsweep_b200 import learned
    rank, world, local = D.init('nccl' if args.gpus > 1 else 'gloo', timeout_s=1800)
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    iters = tuple(int(x) for x in str(args.fwi_iters).split(','))
    bands = (8.0, None) if len(iters) == 2 else (None,) * len(iters)
    if len(iters) not in (1, 2):
        raise SystemExit('--fwi-iters: one count (full band) or two (8 Hz band, full band)')
    with ClockSampler(bus_id(dev)) as clk:
        res = learned.run(n_train=args.train_models, n_test=args.test_models, steps=args.train_steps,
                          iters=iters, bands=bands, seed=rank, log=None)
    if rank == 0:
        print(json.dumps({
            'metric': 'time-to-misfit: learned-proposal FWI to reach plain FWI\'s final data misfit, / plain FWI time',
            'value': res['time_ratio'], 'unit': 'fraction of plain FWI wall time', 'n_gpus': world,
            'steps': sum(iters), 'warmup': 0, 'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'bf16 network (f32 accumulate), f32 physics',
            'data': 'synthetic: seeded models of the four families, gathers simulated by this library',
            'config': {'workload': f'{args.train_models} training models, {args.train_steps} AdamW steps of 64, '
                                   f'{args.test_models} held-out models, L-BFGS iterations per band '
                                   f'{iters} (bands {bands}: Hz of the low-pass, None = full band)',
                       'parameters': 2961536},
            'time_ratio_inclusive': res['time_ratio_inclusive'],
            'plain_fwi_seconds': res['plain_seconds'], 'learned_time_to_plain_misfit_s': res['learned_time_to_plain_misfit'],
            'propose_seconds': res['propose_seconds'], 'train_seconds': res['train_seconds'],
            'train_steps_per_s': res['train_steps_per_s'], 'data_seconds': res['data_seconds'],
            'misfit': {'background': res['J_background'], 'proposal': res['J_proposal'],
                       'plain_final': res['plain_final_misfit'], 'learned_final': res['learned_final_misfit']},
            'normalised_mae': {'background': res['mae_background'], 'proposal': res['mae_proposal'],
                               'plain_fwi': res['mae_plain_fwi'], 'learned_fwi': res['mae_learned_fwi']},
            'accepted_proposals': res['accepted'], 'picker_refused': res['picker_refused'],
            'final_train_l1': res['losses'][-1][1] if res['losses'] else None,
            'clocks': clk.summary(),
        }), flush=True)
    D.finish()
    return 0


def main():
    args = parse()
    if args.warmup < 0 or args.steps < 1:
        raise SystemExit('--steps must be positive and --warmup non-negative')
    if args.impl == 'reference':
        return run_reference(args)
    if args.workload == 'uneven':
        return run_uneven(args)
    if args.workload == 'process':
        return run_process(args)
    if args.workload == 'learned':
        return run_learned(args)
    return run_ours(args)


if __name__ == '__main__':
    sys.exit(main())
