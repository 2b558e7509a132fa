"""Autotuner for uneven batches: the launch shape of each size class, its cluster
size (CTAs per solve) and tile height (rows of the band per thread) together.

A size class is the set of models whose smallest fitting cluster is the same
(``batch.min_cluster``).  A larger cluster cuts each CTA's band of the grid
(fewer rows per thread block, fewer threads per CTA, more synchronisation per
cell) and changes how many solves fit on the GPU at once; a shorter tile puts
more threads (warps) on each band, a taller one reuses more vertical
neighbours from registers and needs fewer threads, so a grid too large for a
small cluster at one height may fit it at another.  The best pair depends on
the grids in the class.  For every class the tuner times the class's own
models, with their time axes shortened to `sample_nt` steps, at tile heights
4, 5 and 6, each at the smallest cluster that fits every model of the class
at that height and up to `extra` sizes above it (and 16 when that smallest
cluster is 10 or more), and keeps the pair with the most padded cell-steps
per second.  Results are cached per device name and class signature (in
memory, and in a JSON file when `cache_path` is given).

    table = tune(shapes)                 # {min_cluster: (cluster, rows per thread)}
    schedule = tune_schedule(shapes, table)
    batch = UnevenBatch(shapes, clusters=table, schedule=schedule)

``tune_schedule`` then times the whole batch, its time axes scaled down by
`nt_scale`, under each stream schedule of ``UnevenBatch`` and keeps the fastest.
"""
from __future__ import annotations

import dataclasses
import json
import os
from pathlib import Path

import numpy as np
import torch

from . import _lib
from .batch import TILE_ROWS, UnevenBatch, make_items, min_cluster

_MEMO = {}


def class_members(shapes, mode=_lib.MODE_IMAGES):
    """{min_cluster: [indices of shapes]}."""
    out = {}
    for i, sh in enumerate(shapes):
        out.setdefault(min_cluster(sh, mode), []).append(i)
    return out


def _signature(shapes):
    nz = [s.nz for s in shapes]
    nx = [s.nx for s in shapes]
    return (len(shapes), min(nz), max(nz), min(nx), max(nx), sum(s.n_shots for s in shapes))


def smallest_cluster(shape, rows, mode=_lib.MODE_IMAGES):
    """The smallest cluster that fits one solve of `shape` at `rows` rows per thread (0: none does)."""
    items, _ = make_items([shape])
    rc = _lib.load().ss_batch_min_cluster_rows(items, mode, rows)
    return rc if rc > 0 else 0


def _time_class(shapes, shape, c_min, device, sample_nt, reps):
    """Seconds of one images run of `shapes` (time axes capped at sample_nt) at launch shape
    (cluster, rows per thread)."""
    short = [dataclasses.replace(s, nt=min(s.nt, sample_nt)) for s in shapes]
    batch = UnevenBatch(short, device=device, clusters={c_min: shape}, schedule=0)
    if any((c['cluster'], c['rows_per_thread']) != tuple(shape) for c in batch.classes()):
        raise RuntimeError('the class does not fit this launch shape')
    rng = np.random.default_rng(0)
    vel = batch.pack_models([np.full((s.nz, s.nx), 2500.0, np.float32) for s in short])
    obs = batch.pack_traces([rng.standard_normal((s.n_shots, s.nt, s.nx)).astype(np.float32) for s in short])
    wav = torch.zeros(max(s.nt for s in short), dtype=torch.float32, device=batch.device)
    wav[:40] = 1.0
    out = (batch._empty(batch.n_out), batch._empty(batch.n_out), None)
    batch.images(vel, wav, obs, out=out)                 # warm-up (and plan)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(reps):
        start.record()
        batch.images(vel, wav, obs, out=out)
        stop.record()
        stop.synchronize()
        times.append(start.elapsed_time(stop) * 1e-3)
    batch.status()
    return float(np.median(times)), sum(s.cell_steps() for s in short)


def tune(shapes, device=None, extra=2, sample_nt=192, reps=3, cache_path=None, verbose=False):
    """{min_cluster: (best cluster, best rows per thread)} for the size classes of `shapes` (images mode)."""
    device = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
    name = torch.cuda.get_device_name(device)
    members = class_members(shapes)
    cache = {}
    if cache_path and Path(cache_path).exists():
        cache = json.loads(Path(cache_path).read_text())
    table, report = {}, {}
    for c_min, idx in sorted(members.items()):
        sub = [shapes[i] for i in idx]
        key = f'{name}|{c_min}|{_signature(sub)}|{sample_nt}'
        if key in _MEMO or key in cache:
            table[c_min] = tuple(int(x) for x in _MEMO.get(key, cache.get(key)))
            continue
        best, results = None, {}
        for rows in TILE_ROWS:
            # the smallest cluster that fits every model of the class at this height, sizes just
            # above it, and for large grids the largest cluster, which may pack the GPU's processing
            # clusters better than one just above
            need = [smallest_cluster(sh, rows) for sh in {(s.nz, s.nx, s.nt, s.pad): s for s in sub}.values()]
            if min(need) == 0:
                continue
            lo = max(need)
            sizes = set(range(lo, min(_lib.MAX_CLUSTER, lo + extra) + 1))
            if lo >= 10:
                sizes.add(_lib.MAX_CLUSTER)
            for c in sorted(sizes):
                try:
                    secs, work = _time_class(sub, (c, rows), c_min, device, sample_nt, reps)
                except RuntimeError:          # this launch shape does not fit: skip it
                    continue
                results[(c, rows)] = work / secs
                if best is None or results[(c, rows)] > results[best]:
                    best = (c, rows)
        if best is None:
            raise RuntimeError(f'no launch shape could run size class {c_min}')
        table[c_min] = best
        _MEMO[key] = list(best)
        cache[key] = list(best)
        report[c_min] = {f'{c}x{h}': f'{r / 1e9:.2f} Gcell-steps/s' for (c, h), r in results.items()}
        if verbose:
            print(f'size class {c_min} ({len(sub)} models): {report[c_min]} -> {best}')
    if cache_path:
        Path(cache_path).parent.mkdir(parents=True, exist_ok=True)
        tmp = Path(str(cache_path) + f'.{os.getpid()}')
        tmp.write_text(json.dumps(cache, indent=1))
        tmp.replace(cache_path)
    return table


def tune_schedule(shapes, table, device=None, nt_scale=0.1, reps=2, verbose=False):
    """The fastest stream schedule (UnevenBatch.SCHEDULES) for the whole batch at cluster table `table`."""
    device = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
    short = [dataclasses.replace(s, nt=max(16, int(round(s.nt * nt_scale)))) for s in shapes]
    rng = np.random.default_rng(1)
    times = {}
    vel = obs = wav = None
    for sched in UnevenBatch.SCHEDULES:
        batch = UnevenBatch(short, device=device, clusters=table, schedule=sched)
        if vel is None:
            vel = batch.pack_models([np.full((s.nz, s.nx), 2500.0, np.float32) for s in short])
            obs = batch.pack_traces([rng.standard_normal((s.n_shots, s.nt, s.nx)).astype(np.float32) for s in short])
            wav = torch.zeros(batch.max_nt, dtype=torch.float32, device=batch.device)
            wav[:40] = 1.0
        out = (batch._empty(batch.n_out), batch._empty(batch.n_out), None)
        batch.images(vel, wav, obs, out=out)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ts = []
        for _ in range(reps):
            start.record()
            batch.images(vel, wav, obs, out=out)
            stop.record()
            stop.synchronize()
            ts.append(start.elapsed_time(stop))
        batch.status()
        times[sched] = float(np.median(ts))
        del batch
    if verbose:
        print('schedules (ms):', times)
    return min(times, key=times.get)
