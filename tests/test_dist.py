"""Multi-process plumbing on CPU (gloo, world size 2): shards cover the work once, timings reduce to the max."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from shotsweep_b200 import dist as D


def test_shard_covers_every_unit_once():
    for n in (0, 1, 7, 500, 1501):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                a, b = D.shard(n, r, world)
                assert 0 <= a <= b <= n
                seen.extend(range(a, b))
            assert seen == list(range(n))
            sizes = [D.shard(n, r, world)[1] - D.shard(n, r, world)[0] for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        D.shard(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    r, w, _ = D.init('gloo', timeout_s=60)
    a, b = D.shard(1500, r, w)
    D.barrier()
    slowest = D.reduce(1.0 + r, 'max')
    total = D.reduce(b - a, 'sum')
    q.put((r, a, b, slowest, total))
    D.finish()


def test_two_ranks_split_and_reduce():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1:3] == (0, 750) and out[1][1:3] == (750, 1500)
    assert all(o[3] == 2.0 and o[4] == 1500.0 for o in out)


def _bench_worker(rank, world, port, q):
    """One rank of bench.py's data-path split: its contiguous share of the seeded model population and
    the backgrounds built from it, returned to the parent for comparison with one process's view."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    r, w, _ = D.init('gloo', timeout_s=60)
    per = 6
    a, b = D.shard(per * w, r, w)
    models = bench.population_slice(a, b, per * w)
    trend = bench.depth_trend(bench.population_slice(0, 40, 40))
    bgs, vm = bench.backgrounds_for(models, trend)
    D.barrier()
    q.put((r, a, b, models, bgs, vm))
    D.finish()


def test_two_ranks_take_disjoint_shares_of_the_bench_population():
    """Under torchrun every rank images its own contiguous slice of one seeded population (weak scaling,
    no data-path collective): the slices of two gloo ranks are disjoint, cover the population, and hold
    exactly the models and backgrounds that one process builds for those indices."""
    import sys
    from pathlib import Path
    import numpy as np
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [(o[1], o[2]) for o in out] == [(0, 6), (6, 12)]
    full = bench.population_slice(0, 12, 12)
    trend = bench.depth_trend(bench.population_slice(0, 40, 40))
    bgs, vm = bench.backgrounds_for(full, trend)
    assert np.array_equal(np.concatenate([o[3] for o in out]), full)
    assert np.array_equal(np.concatenate([o[4] for o in out]), bgs)
    assert np.array_equal(np.concatenate([o[5] for o in out]), vm)
