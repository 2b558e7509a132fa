"""One process per GPU: rank discovery, work split and max-over-ranks timing.

Every (velocity model, background, shot) solve is independent, so several
GPUs split the list of velocity models into contiguous shards and exchange
nothing on the data path.  The only collectives are the timing barrier and
the max/sum reductions that turn per-rank timings into one number.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env():
    """(rank, world_size, local_rank) from the torchrun environment (defaults: single process)."""
    return (int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1)),
            int(os.environ.get('LOCAL_RANK', 0)))


def init(backend='nccl', timeout_s=120):
    """Join the process group when launched with more than one rank; returns (rank, world, local_rank)."""
    rank, world, local = env()
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault('MASTER_ADDR', '127.0.0.1')
        kwargs = {'timeout': datetime.timedelta(seconds=timeout_s)}
        if backend == 'nccl':
            kwargs['device_id'] = torch.device('cuda', local)
        dist.init_process_group(backend, **kwargs)
    return rank, world, local


def shard(n_units, rank, world):
    """Contiguous [start, stop) slice of n_units for this rank; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError('rank must lie in [0, world)')
    base, extra = divmod(n_units, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def barrier():
    if dist.is_initialized():
        dist.barrier()


def reduce(value, op='max', device=None):
    """max / sum of a float over ranks (identity on one rank)."""
    if not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == 'max' else dist.ReduceOp.SUM)
    return float(t.item())


def finish():
    if dist.is_initialized():
        dist.destroy_process_group()
