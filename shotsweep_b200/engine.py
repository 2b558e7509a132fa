"""Geometry-generic device entry points over the C ABI.

``Engine(geometry)`` runs forward modelling, gradients and RTM images for any
grid / time axis / shot layout that the kernels plan for (the reference's
``Sim`` hard-wires 70x70, 1000 steps, 5 shots; ``shotsweep_b200.gpu.Sim`` is a
thin layer over this class with that geometry).  Arguments are CUDA float32
tensors; outputs are new CUDA tensors.  The per-step history workspace is
allocated once and reused while it is large enough.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib


def geometry(nz=70, nx=70, nt=1000, pad=40, shot_cols=(0, 17, 34, 52, 69), src_row=1, dx=10.0, dt=1e-3,
             R=1e-5):
    return _lib.make_geometry(nz, nx, nt, pad, shot_cols, src_row, dx, dt, R)


class Engine:
    def __init__(self, geom, device=None):
        self.g = geom
        self.device = torch.device('cuda') if device is None else torch.device(device)
        _lib.require_cuda(self.device)
        if self.device.index is None:
            self.device = torch.device('cuda', torch.cuda.current_device())
        self.L = _lib.load()
        self._ws = None

    # -- plumbing -----------------------------------------------------------
    @property
    def shape(self):
        return self.g.nz, self.g.nx

    @property
    def n_shots(self):
        return self.g.n_shots

    @property
    def padded(self):
        return self.g.nz + 2 * self.g.pad, self.g.nx + 2 * self.g.pad

    def plan(self, n_models, mode):
        out = (ctypes.c_int64 * 8)()
        with torch.cuda.device(self.device):
            _lib.check(self.L.ss_plan_info(ctypes.byref(self.g), n_models, mode, out), 'ss_plan_info')
        keys = ('cluster', 'threads', 'smem', 'band_rows', 'col_groups', 'rows_per_thread', 'max_clusters', 'slots')
        return dict(zip(keys, list(out)))

    def workspace(self, n_models, mode):
        with torch.cuda.device(self.device):
            need = self.L.ss_workspace_bytes(ctypes.byref(self.g), n_models, mode)
        if need == 0:
            _lib.check(_lib.ERR_UNSUPPORTED, 'ss_workspace_bytes')
        if self._ws is None or self._ws.numel() < need:
            self._ws = None
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        return self._ws

    def _stream(self):
        return _lib.stream_handle(self.device)

    def _check_in(self, t, shape, name):
        if not isinstance(t, torch.Tensor) or t.device != self.device or t.dtype != torch.float32:
            raise ValueError(f'{name} must be a float32 tensor on {self.device}')
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f'{name} must have shape {tuple(shape)}, got {tuple(t.shape)}')
        return t.contiguous()

    def status(self):
        """Raise if the last simulation on this engine recorded a device-side failure."""
        if self._ws is None:
            return
        with torch.cuda.device(self.device):
            rc = self.L.ss_workspace_status(_lib.ptr(self._ws), self._stream())
        if rc == _lib.ERR_NONFINITE:
            raise ValueError('observations must be finite')
        _lib.check(rc, 'device status')

    # -- entry points ----------------------------------------------------------
    def forward(self, vel, wavelet, ckpt_interval=None, out=None):
        """Gathers [B, S, nt, nx] (+ checkpoints [B, S, n_ck, 2, nzp, nxp] if ckpt_interval)."""
        g = self.g
        B = vel.shape[0]
        vel = self._check_in(vel, (B, g.nz, g.nx), 'vel')
        wavelet = self._check_in(wavelet, (g.nt,), 'wavelet')
        if out is None:
            out = torch.empty(B, g.n_shots, g.nt, g.nx, dtype=torch.float32, device=self.device)
        ck = None
        if ckpt_interval:
            n_ck = math.ceil(g.nt / ckpt_interval)
            ck = torch.zeros(B, g.n_shots, n_ck, 2, *self.padded, dtype=torch.float32, device=self.device)
        ws = self.workspace(B, _lib.MODE_FORWARD)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ss_forward(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(wavelet), _lib.ptr(out),
                                         _lib.ptr(ck), int(ckpt_interval or 0), _lib.ptr(ws), ws.numel(),
                                         self._stream()), 'ss_forward')
        return (out, ck) if ckpt_interval else out

    def gradient(self, vel, wavelet, obs, v_mute=None, t_mute=0.12):
        """(grad, illum), each [B, S, nz, nx]."""
        g = self.g
        B = vel.shape[0]
        vel = self._check_in(vel, (B, g.nz, g.nx), 'vel')
        wavelet = self._check_in(wavelet, (g.nt,), 'wavelet')
        obs = self._check_in(obs, (B, g.n_shots, g.nt, g.nx), 'obs')
        if v_mute is not None:
            v_mute = self._check_in(v_mute, (B,), 'v_mute')
        grad = torch.empty(B, g.n_shots, g.nz, g.nx, dtype=torch.float32, device=self.device)
        illum = torch.empty_like(grad)
        ws = self.workspace(B, _lib.MODE_GRADIENT)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ss_gradient(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(wavelet), _lib.ptr(obs),
                                          _lib.ptr(v_mute), float(t_mute), _lib.ptr(grad), _lib.ptr(illum),
                                          _lib.ptr(ws), ws.numel(), self._stream()), 'ss_gradient')
        return grad, illum

    def images_from_host(self, vel, wavelet, obs_host, v_mute=None, t_mute=0.12, eps=1e-4, laplacian=True,
                         chunk_rows=None):
        """Images of host-resident observations with the copies overlapped (pinned host img, illum).

        The rows are imaged in chunks: chunk k+1's gathers move to the device on a copy stream while chunk k
        is imaged (two device buffers), and each chunk's images return to pinned host memory behind it, so
        that an end-to-end call costs about the imaging time plus one chunk's copy.  obs_host: CPU tensor
        [B, S, nt, nx] float32, pinned or not (pageable rows are staged through pinned buffers).
        """
        g = self.g
        B = vel.shape[0]
        shape = (B, g.n_shots, g.nt, g.nx)
        if not isinstance(obs_host, torch.Tensor) or obs_host.device.type != 'cpu' or obs_host.dtype != torch.float32:
            raise ValueError('obs_host must be a float32 CPU tensor')
        if tuple(obs_host.shape) != shape:
            raise ValueError(f'obs must have shape {shape}, got {tuple(obs_host.shape)}')
        obs_host = obs_host.contiguous()
        if chunk_rows:
            chunk = int(chunk_rows)
        else:   # about six chunks, each a whole number of rounds of the persistent clusters
            slots = self.plan(B, _lib.MODE_IMAGES)['slots']
            per_round = slots // math.gcd(slots, g.n_shots)          # rows whose solves fill whole rounds
            chunk = max(1, min(B, math.ceil(math.ceil(B / 6) / per_round) * per_round))
        n_chunks = math.ceil(B / chunk)
        dev = self.device
        compute = torch.cuda.current_stream(dev)
        if getattr(self, '_copy_stream', None) is None:
            self._copy_stream = torch.cuda.Stream(dev)
        copy = self._copy_stream
        f32 = dict(dtype=torch.float32, device=dev)
        dev_obs = [torch.empty(chunk, *shape[1:], **f32) for _ in range(min(2, n_chunks))]
        pinned = obs_host.is_pinned()
        staging = [] if pinned else [torch.empty(chunk, *shape[1:], dtype=torch.float32, pin_memory=True)
                                     for _ in range(min(2, n_chunks))]
        img_dev = torch.empty(B, g.n_shots, g.nz, g.nx, **f32)
        illum_dev = torch.empty_like(img_dev)
        img = torch.empty(img_dev.shape, dtype=torch.float32, pin_memory=True)
        illum = torch.empty_like(img, pin_memory=True)
        flags = torch.zeros(n_chunks, dtype=torch.int32, device=dev)
        copied = [torch.cuda.Event() for _ in dev_obs]
        imaged = [torch.cuda.Event() for _ in dev_obs]
        for k in range(n_chunks):
            a, b = k * chunk, min(B, (k + 1) * chunk)
            buf = k % len(dev_obs)
            src = obs_host[a:b]
            if not pinned:
                if k >= len(staging):
                    copied[buf].synchronize()          # the staging buffer's previous rows have left
                staging[buf][:b - a].copy_(src)
                src = staging[buf][:b - a]
            with torch.cuda.stream(copy):
                if k >= len(dev_obs):
                    copy.wait_event(imaged[buf])       # the device buffer's previous chunk is imaged
                dev_obs[buf][:b - a].copy_(src, non_blocking=True)
                copied[buf].record(copy)
            compute.wait_event(copied[buf])
            self.images(vel[a:b], wavelet, dev_obs[buf][:b - a], None if v_mute is None else v_mute[a:b], t_mute, eps,
                        laplacian, out=(img_dev[a:b], illum_dev[a:b]))
            flags[k:k + 1].copy_(self._ws[:4].view(torch.int32))   # this chunk's device status, kept
            imaged[buf].record(compute)
            with torch.cuda.stream(copy):
                copy.wait_event(imaged[buf])
                img[a:b].copy_(img_dev[a:b], non_blocking=True)
                illum[a:b].copy_(illum_dev[a:b], non_blocking=True)
        copy.synchronize()
        compute.synchronize()
        bad = flags.cpu().numpy()
        if (bad == _lib.ERR_NONFINITE).any():
            raise ValueError('observations must be finite')
        if bad.any():
            _lib.check(int(bad[bad != 0][0]), 'device status')
        return img, illum

    def images(self, vel, wavelet, obs, v_mute=None, t_mute=0.12, eps=1e-4, laplacian=True, want_grad=False,
               out=None):
        """(img, illum[, grad]), each [B, S, nz, nx]."""
        if not eps > 0:
            raise ValueError('illumination regularization eps must be positive')
        g = self.g
        B = vel.shape[0]
        vel = self._check_in(vel, (B, g.nz, g.nx), 'vel')
        wavelet = self._check_in(wavelet, (g.nt,), 'wavelet')
        obs = self._check_in(obs, (B, g.n_shots, g.nt, g.nx), 'obs')
        if v_mute is not None:
            v_mute = self._check_in(v_mute, (B,), 'v_mute')
        if out is None:
            img = torch.empty(B, g.n_shots, g.nz, g.nx, dtype=torch.float32, device=self.device)
            illum = torch.empty_like(img)
        else:
            img, illum = out
        grad = torch.empty_like(img) if want_grad else None
        ws = self.workspace(B, _lib.MODE_IMAGES)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ss_images(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(wavelet), _lib.ptr(obs),
                                        _lib.ptr(v_mute), float(t_mute), float(eps), int(bool(laplacian)),
                                        _lib.ptr(img), _lib.ptr(illum), _lib.ptr(grad), _lib.ptr(ws), ws.numel(),
                                        self._stream()), 'ss_images')
        return (img, illum, grad) if want_grad else (img, illum)

    # -- checkpointed adjoint (differentiation) --------------------------------
    def segment_workspace(self, n_models, interval):
        with torch.cuda.device(self.device):
            need = self.L.ss_segment_workspace_bytes(ctypes.byref(self.g), n_models, int(interval))
        if need == 0:
            _lib.check(_lib.ERR_UNSUPPORTED, 'ss_segment_workspace_bytes')
        if self._ws is None or self._ws.numel() < need:
            self._ws = None
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        return self._ws

    def adjoint_from_checkpoints(self, vel, wavelet, ckpt, interval, res):
        """Per-shot gradient and illumination from forward checkpoints and an adjoint source.

        ckpt [B, S, n_ck, 2, nzp, nxp] from forward(..., ckpt_interval=interval);
        res [B, S, nt, nx] = dJ/d(gathers).  Segments run last-first, each
        recomputing `interval` steps from its checkpoint (gpu.py:169-184).
        """
        g = self.g
        B = vel.shape[0]
        vel = self._check_in(vel, (B, g.nz, g.nx), 'vel')
        wavelet = self._check_in(wavelet, (g.nt,), 'wavelet')
        res = self._check_in(res, (B, g.n_shots, g.nt, g.nx), 'res')
        n_ck = math.ceil(g.nt / interval)
        if tuple(ckpt.shape) != (B, g.n_shots, n_ck, 2, *self.padded):
            raise ValueError('checkpoints do not match the geometry and interval')
        f32 = dict(dtype=torch.float32, device=self.device)
        theta = torch.zeros(B, g.n_shots, 2, *self.padded, **f32)
        gacc = torch.zeros(B, g.n_shots, *self.padded, **f32)
        illum_acc = torch.zeros(B, g.n_shots, g.nz, g.nx, **f32)
        src_acc = torch.zeros(B, g.n_shots, **f32)
        ws = self.segment_workspace(B, interval)
        with torch.cuda.device(self.device):
            for k in range(n_ck - 1, -1, -1):
                _lib.check(self.L.ss_adjoint_segment(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(wavelet),
                                                     _lib.ptr(ckpt), int(interval), k, _lib.ptr(res), _lib.ptr(theta),
                                                     _lib.ptr(gacc), _lib.ptr(illum_acc), _lib.ptr(src_acc),
                                                     _lib.ptr(ws), ws.numel(), self._stream()), 'ss_adjoint_segment')
            grad = torch.empty(B, g.n_shots, g.nz, g.nx, **f32)
            illum = torch.empty_like(grad)
            _lib.check(self.L.ss_gradient_finish(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(gacc), _lib.ptr(src_acc),
                                                 _lib.ptr(illum_acc), _lib.ptr(grad), _lib.ptr(illum), self._stream()),
                       'ss_gradient_finish')
        self.status()
        return grad, illum

    def mute_weights(self, v_mute, t_mute=0.12):
        g = self.g
        v_mute = self._check_in(v_mute, (v_mute.shape[0],), 'v_mute')
        out = torch.empty(v_mute.shape[0], g.n_shots, g.nt, g.nx, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ss_mute_weights(ctypes.byref(g), v_mute.shape[0], _lib.ptr(v_mute), float(t_mute),
                                              _lib.ptr(out), self._stream()), 'ss_mute_weights')
        return out

    def c2_field(self, vel):
        g = self.g
        out = torch.empty(vel.shape[0], *self.padded, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.L.ss_c2_field(ctypes.byref(g), vel.shape[0], _lib.ptr(vel), _lib.ptr(out),
                                          self._stream()), 'ss_c2_field')
        return out


def scaled_wavelet(wavelet, device):
    """The reference injects wavelet*1e3 (gpu.py:94), computed in float64 then cast."""
    return torch.as_tensor(np.asarray(wavelet, np.float64) * 1e3, dtype=torch.float32).to(device)
