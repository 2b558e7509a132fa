"""Uneven batches: models of different grid size, step count and shot count in one launch sequence.

The reference's ``Sim`` runs one fixed geometry (70x70 cells, 1000 steps, 5 shots;
openfwi/physics/gpu.py:59,95-96,103,126-128).  ``UnevenBatch`` takes a list of
models, each with its own grid, time axis, shot columns, absorbing-layer width
and mute velocity, packs their arrays end to end in device memory, and runs
forward modelling, gradients or RTM images for all of them through
``ss_batch_plan`` / ``ss_batch_run``: one persistent launch per size class
(the solves that need the same cluster of CTAs), the classes spread over two
streams (``schedule``), optionally replayed as one CUDA graph.  Every solve computes what
the single-geometry entry points compute for its own geometry.

    shapes = [Shape(nz=120, nx=200, nt=2000, shot_cols=shot_columns(200, 3)), ...]
    batch = UnevenBatch(shapes, clusters=autotune.tune(shapes))
    vel = batch.pack_models(models)                 # list of [nz, nx] arrays
    gathers = batch.forward(vel, wavelet)           # packed [n_shots, nt, nx] per model
    img, illum, grad = batch.images(vel, wavelet, gathers)
    batch.unpack_images(img, i)                     # [n_shots, nz, nx] of model i
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib


def shot_columns(nx, n_shots):
    """Evenly spread source columns round(linspace(0, nx - 1, n)); [0, 17, 34, 52, 69] for nx = 70, n = 5."""
    return [int(c) for c in np.round(np.linspace(0, nx - 1, n_shots))]


@dataclass
class Shape:
    """Grid and acquisition of one model (one background row) of a batch."""
    nz: int
    nx: int
    nt: int
    shot_cols: list = field(default_factory=list)
    pad: int = 40
    src_row: int = 1
    v_mute: float = 0.0          # direct-wave mute velocity (m/s); 0: no mute

    @property
    def n_shots(self):
        return len(self.shot_cols)

    def cell_steps(self):
        """Padded cells x steps x shots: the solves' work."""
        return (self.nz + 2 * self.pad) * (self.nx + 2 * self.pad) * self.nt * self.n_shots


def physics(dx=10.0, dt=1e-3, r_coef=1e-5, vmax_damping=4500.0, amp_ref=2000.0):
    p = _lib.Physics()
    p.dx, p.dt, p.r_coef, p.vmax_damping, p.amp_ref = dx, dt, r_coef, vmax_damping, amp_ref
    return p


def make_items(shapes):
    """ss_batch_item array with the packed offsets of velocities, traces and images."""
    items = (_lib.BatchItem * len(shapes))()
    vo = to = oo = 0
    for it, sh in zip(items, shapes):
        if not 1 <= sh.n_shots <= _lib.MAX_SHOTS:
            raise ValueError(f'between 1 and {_lib.MAX_SHOTS} shots per model are supported')
        it.nz, it.nx, it.nt, it.pad = sh.nz, sh.nx, sh.nt, sh.pad
        it.n_shots, it.src_row = sh.n_shots, sh.src_row
        for i, c in enumerate(sh.shot_cols):
            it.shot_cols[i] = int(c)
        it.vel_offset, it.obs_offset, it.out_offset = vo, to, oo
        it.v_mute = float(sh.v_mute)
        vo += sh.nz * sh.nx
        to += sh.n_shots * sh.nt * sh.nx
        oo += sh.n_shots * sh.nz * sh.nx
    return items, (vo, to, oo)


MAX_CLASSES = 32          # (cluster size, tile height) launches of one plan, at most
TILE_ROWS = (4, 5, 6)     # tile heights (rows per thread) of the batch kernels


def launch_shape_code(shape):
    """A size class's launch shape for ss_batch_plan: a cluster size, or (cluster size, rows per thread)."""
    if isinstance(shape, (tuple, list)):
        c, h = int(shape[0]), int(shape[1])
        if h not in TILE_ROWS:
            raise ValueError(f'rows per thread must be one of {TILE_ROWS}')
        return c | (h << 8)
    return int(shape)


def min_cluster(shape, mode=_lib.MODE_IMAGES):
    """The size class of a model: the smallest cluster of CTAs that fits one of its solves."""
    items, _ = make_items([shape])
    L = _lib.load()
    rc = L.ss_batch_min_cluster(items, mode)
    if rc < 0:
        _lib.check(rc, 'ss_batch_min_cluster')
    return rc


class UnevenBatch:
    """A planned uneven batch on one device (one plan per mode, built on first use)."""

    # schedule: 0 one stream; 1 classes alternate between two streams; 2 classes
    # whose large clusters leave SMs idle on one stream, the others beside them
    SCHEDULES = (0, 1, 2)

    def __init__(self, shapes, device=None, clusters=None, schedule=2, phys=None):
        """clusters: {size class (smallest cluster at 5 rows per thread): cluster size or (cluster size,
        rows per thread)}, e.g. from autotune.tune; classes not listed run at their smallest cluster."""
        if not shapes:
            raise ValueError('an uneven batch needs at least one model')
        self.shapes = list(shapes)
        self.device = torch.device('cuda', torch.cuda.current_device()) if device is None else torch.device(device)
        _lib.require_cuda(self.device)
        if self.device.index is None:
            self.device = torch.device('cuda', torch.cuda.current_device())
        self.L = _lib.load()
        self.items, (self.n_vel, self.n_trace, self.n_out) = make_items(self.shapes)
        self.phys = physics() if phys is None else phys
        self.clusters = dict(clusters or {})
        if int(schedule) not in self.SCHEDULES:
            raise ValueError(f'schedule must be one of {self.SCHEDULES}')
        self.schedule = int(schedule)
        self.max_nt = max(s.nt for s in self.shapes)
        self.n_solves = sum(s.n_shots for s in self.shapes)
        self._plans = {}
        self._ws = None

    # -- planning -------------------------------------------------------------
    def plan(self, mode):
        """(host plan bytes, device copy, workspace bytes) for `mode`, built once."""
        if mode in self._plans:
            return self._plans[mode]
        table = (ctypes.c_int32 * (_lib.MAX_CLUSTER + 1))()
        for k, v in self.clusters.items():
            table[int(k)] = launch_shape_code(v)
        pb, wb = ctypes.c_size_t(0), ctypes.c_size_t(0)
        args = (ctypes.byref(self.phys), mode, self.items, len(self.items), table, self.schedule)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ss_batch_plan(*args, None, ctypes.byref(pb), ctypes.byref(wb)), 'ss_batch_plan')
            host = np.zeros(pb.value, np.uint8)
            _lib.check(self.L.ss_batch_plan(*args, host.ctypes.data_as(ctypes.c_void_p), ctypes.byref(pb),
                                            ctypes.byref(wb)), 'ss_batch_plan')
        dev = torch.from_numpy(host).to(self.device)
        self._plans[mode] = (host, dev, wb.value)
        return self._plans[mode]

    def classes(self, mode=_lib.MODE_IMAGES):
        host, _, _ = self.plan(mode)
        out = (_lib.BatchClassInfo * MAX_CLASSES)()
        n = ctypes.c_int32(0)
        _lib.check(self.L.ss_batch_classes(host.ctypes.data_as(ctypes.c_void_p), out, MAX_CLASSES,
                                           ctypes.byref(n)), 'ss_batch_classes')
        keys = ('min_cluster', 'cluster', 'rows_per_thread', 'n_solves', 'threads', 'smem_bytes', 'slots', 'stream',
                'cell_steps')
        return [{k: getattr(out[i], k) for k in keys} for i in range(n.value)]

    def workspace(self, mode):
        need = self.plan(mode)[2]
        if self._ws is None or self._ws.numel() < need:
            self._ws = None
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        return self._ws

    def status(self):
        if self._ws is not None:
            with torch.cuda.device(self.device):
                _lib.check(self.L.ss_workspace_status(_lib.ptr(self._ws), _lib.stream_handle(self.device)),
                           'device status')

    # -- packing ----------------------------------------------------------------
    def pack_models(self, models):
        """Velocities of every model ([nz, nx] each) in one float32 device array."""
        if len(models) != len(self.shapes):
            raise ValueError(f'expected {len(self.shapes)} models, got {len(models)}')
        parts = []
        for m, sh in zip(models, self.shapes):
            a = torch.as_tensor(m, dtype=torch.float32)
            if tuple(a.shape) != (sh.nz, sh.nx):
                raise ValueError(f'model of shape {tuple(a.shape)} where {(sh.nz, sh.nx)} was planned')
            parts.append(a.reshape(-1).to(self.device))
        return torch.cat(parts).contiguous()

    def pack_traces(self, traces):
        parts = []
        for t, sh in zip(traces, self.shapes):
            a = torch.as_tensor(t, dtype=torch.float32)
            if tuple(a.shape) != (sh.n_shots, sh.nt, sh.nx):
                raise ValueError(f'traces of shape {tuple(a.shape)} where {(sh.n_shots, sh.nt, sh.nx)} was planned')
            parts.append(a.reshape(-1).to(self.device))
        return torch.cat(parts).contiguous()

    def unpack_traces(self, packed, i):
        it, sh = self.items[i], self.shapes[i]
        n = sh.n_shots * sh.nt * sh.nx
        return packed[it.obs_offset:it.obs_offset + n].view(sh.n_shots, sh.nt, sh.nx)

    def unpack_images(self, packed, i):
        it, sh = self.items[i], self.shapes[i]
        n = sh.n_shots * sh.nz * sh.nx
        return packed[it.out_offset:it.out_offset + n].view(sh.n_shots, sh.nz, sh.nx)

    # -- compute ----------------------------------------------------------------
    def _run(self, mode, vel, wavelet, obs=None, t_mute=0.12, eps=1e-4, laplacian=True, gathers=None, img=None,
             illum=None, grad=None):
        self._check(vel, self.n_vel, 'vel')
        self._check(wavelet, None, 'wavelet')
        if wavelet.numel() < self.max_nt:
            raise ValueError(f'the wavelet needs at least {self.max_nt} samples')
        if obs is not None:
            self._check(obs, self.n_trace, 'obs')
        host, dev, _ = self.plan(mode)
        ws = self.workspace(mode)
        with torch.cuda.device(self.device):
            rc = self.L.ss_batch_run(host.ctypes.data_as(ctypes.c_void_p), _lib.ptr(dev), _lib.ptr(vel),
                                     _lib.ptr(wavelet), _lib.ptr(obs), float(t_mute), float(eps), int(bool(laplacian)),
                                     _lib.ptr(gathers), _lib.ptr(img), _lib.ptr(illum), _lib.ptr(grad), _lib.ptr(ws),
                                     ws.numel(), _lib.stream_handle(self.device))
        _lib.check(rc, 'ss_batch_run')

    def _check(self, t, n, name):
        if not isinstance(t, torch.Tensor) or t.device != self.device or t.dtype != torch.float32 \
                or not t.is_contiguous():
            raise ValueError(f'{name} must be a contiguous float32 tensor on {self.device}')
        if n is not None and t.numel() != n:
            raise ValueError(f'{name} must hold {n} values, got {t.numel()}')

    def _empty(self, n):
        return torch.empty(n, dtype=torch.float32, device=self.device)

    def forward(self, vel, wavelet, out=None):
        """Packed gathers ([n_shots, nt, nx] per model, in model order)."""
        out = self._empty(self.n_trace) if out is None else out
        self._run(_lib.MODE_FORWARD, vel, wavelet, gathers=out)
        return out

    def gradient(self, vel, wavelet, obs, t_mute=0.12, out=None):
        """Packed per-shot gradients and illuminations of 0.5 sum w (sim - obs)^2 (mute from each Shape)."""
        grad, illum = (self._empty(self.n_out), self._empty(self.n_out)) if out is None else out
        self._run(_lib.MODE_GRADIENT, vel, wavelet, obs, t_mute=t_mute, illum=illum, grad=grad)
        return grad, illum

    def images(self, vel, wavelet, obs, t_mute=0.12, eps=1e-4, laplacian=True, want_grad=False, out=None):
        """Packed RTM images, illuminations (and gradients) per shot."""
        if out is None:
            img, illum = self._empty(self.n_out), self._empty(self.n_out)
            grad = self._empty(self.n_out) if want_grad else None
        else:
            img, illum, grad = out
        self._run(_lib.MODE_IMAGES, vel, wavelet, obs, t_mute=t_mute, eps=eps, laplacian=laplacian, img=img,
                  illum=illum, grad=grad)
        return img, illum, grad

    def capture_images(self, vel, wavelet, obs, t_mute=0.12, eps=1e-4, laplacian=True):
        """A CUDA graph of one images run over these buffers: (graph, img, illum); graph.replay() reruns it."""
        img, illum = self._empty(self.n_out), self._empty(self.n_out)
        self.plan(_lib.MODE_IMAGES)
        self.workspace(_lib.MODE_IMAGES)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):      # warm-up outside capture
            self.images(vel, wavelet, obs, t_mute, eps, laplacian, out=(img, illum, None))
        torch.cuda.current_stream(self.device).wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.images(vel, wavelet, obs, t_mute, eps, laplacian, out=(img, illum, None))
        return graph, img, illum
