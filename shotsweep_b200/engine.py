"""Geometry-generic device entry points over the C ABI.

``Engine(geometry)`` runs forward modelling, gradients and RTM images for any
grid / time axis / shot layout that the kernels plan for (the reference's
``Sim`` hard-wires 70x70, 1000 steps, 5 shots; ``shotsweep_b200.gpu.Sim`` is a
thin layer over this class with that geometry).  Arguments are CUDA float32
tensors; outputs are new CUDA tensors.  The per-step history workspace is
allocated once and reused while it is large enough.  ``max_slots`` caps the
solves in flight (each holds its own history, about 89 MB for the OpenFWI
grid), which bounds the workspace of a call.
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
        self.max_slots = None     # None: every co-resident cluster gets a solve

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
        info = dict(zip(keys, list(out)))
        if self.max_slots is not None and mode != _lib.MODE_FORWARD:
            info['slots'] = max(1, min(info['slots'], int(self.max_slots)))
        return info

    def workspace(self, n_models, mode):
        """The workspace of a call: a view of the engine's buffer, exactly as long as the call's plan needs
        (the library keeps as many solves in flight as the workspace it is given holds)."""
        with torch.cuda.device(self.device):
            if self.max_slots is not None and mode != _lib.MODE_FORWARD:
                slots = self.plan(n_models, mode)['slots']
                need = self.L.ss_workspace_bytes_slots(ctypes.byref(self.g), mode, slots)
            else:
                need = self.L.ss_workspace_bytes(ctypes.byref(self.g), n_models, mode)
        if need == 0:
            _lib.check(_lib.ERR_UNSUPPORTED, 'ss_workspace_bytes')
        if self._ws is None or self._ws.numel() < need:
            self._ws = None
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        return self._ws[:need]

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
    def _wavelet_in(self, wavelet, B):
        """(wavelet, per_model): one wavelet [nt] for every model, or one per model [B, nt]."""
        per_model = isinstance(wavelet, torch.Tensor) and wavelet.dim() == 2
        shape = (B, self.g.nt) if per_model else (self.g.nt,)
        return self._check_in(wavelet, shape, 'wavelet'), per_model

    def forward(self, vel, wavelet, ckpt_interval=None, out=None):
        """Gathers [B, S, nt, nx] (+ checkpoints [B, S, n_ck, 2, nzp, nxp] if ckpt_interval).

        wavelet: [nt] for every model, or [B, nt] (one per model; no checkpoints)."""
        g = self.g
        B = vel.shape[0]
        vel = self._check_in(vel, (B, g.nz, g.nx), 'vel')
        wavelet, per_model = self._wavelet_in(wavelet, B)
        if per_model and ckpt_interval:
            raise ValueError('checkpoints are kept with one wavelet for every model only')
        if out is None:
            out = torch.empty(B, g.n_shots, g.nt, g.nx, dtype=torch.float32, device=self.device)
        ck = None
        if ckpt_interval:
            n_ck = math.ceil(g.nt / ckpt_interval)
            ck = torch.zeros(B, g.n_shots, n_ck, 2, *self.padded, dtype=torch.float32, device=self.device)
        ws = self.workspace(B, _lib.MODE_FORWARD)
        with torch.cuda.device(self.device):
            if per_model:
                _lib.check(self.L.ss_forward_wavelets(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(wavelet),
                                                      _lib.ptr(out), _lib.ptr(ws), ws.numel(), self._stream()),
                           'ss_forward_wavelets')
            else:
                _lib.check(self.L.ss_forward(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(wavelet), _lib.ptr(out),
                                             _lib.ptr(ck), int(ckpt_interval or 0), _lib.ptr(ws), ws.numel(),
                                             self._stream()), 'ss_forward')
        return (out, ck) if ckpt_interval else out

    def gradient(self, vel, wavelet, obs, v_mute=None, t_mute=0.12):
        """(grad, illum), each [B, S, nz, nx]; wavelet [nt], or [B, nt] (one per model)."""
        g = self.g
        B = vel.shape[0]
        vel = self._check_in(vel, (B, g.nz, g.nx), 'vel')
        wavelet, per_model = self._wavelet_in(wavelet, B)
        obs = self._check_in(obs, (B, g.n_shots, g.nt, g.nx), 'obs')
        if v_mute is not None:
            v_mute = self._check_in(v_mute, (B,), 'v_mute')
        grad = torch.empty(B, g.n_shots, g.nz, g.nx, dtype=torch.float32, device=self.device)
        illum = torch.empty_like(grad)
        ws = self.workspace(B, _lib.MODE_GRADIENT)
        entry = self.L.ss_gradient_wavelets if per_model else self.L.ss_gradient
        with torch.cuda.device(self.device):
            _lib.check(entry(ctypes.byref(g), B, _lib.ptr(vel), _lib.ptr(wavelet), _lib.ptr(obs), _lib.ptr(v_mute),
                             float(t_mute), _lib.ptr(grad), _lib.ptr(illum), _lib.ptr(ws), ws.numel(),
                             self._stream()), 'ss_gradient_wavelets' if per_model else 'ss_gradient')
        return grad, illum

    def images_from_host(self, vel, wavelet, obs_host, v_mute=None, t_mute=0.12, eps=1e-4, laplacian=True,
                         chunk_rows=None):
        """Images of host-resident observations with the copies overlapped (pinned host img, illum).

        The rows are imaged in chunks.  Gathers (and, for host velocities, the model rows) move to the
        device on one copy stream, at most two chunks ahead of the imaging (two device buffers); images
        return to pinned host memory on a second copy stream behind each chunk.  The chunks grow from one
        round of the persistent clusters, so that imaging starts after a short first copy, and the last one
        is small, so that little is left to copy back at the end: a call costs about the imaging time.
        vel: [B, nz, nx], float32 on the device, or float32 / float64 on the host (each chunk's rows are
        converted into a pinned float32 buffer just before its copy, while the previous chunk is imaged).
        obs_host: CPU tensor [B, S, nt, nx], float32 (pinned or not) or float64; pageable or float64 rows are
        staged (and converted) through pinned float32 buffers chunk by chunk, while the previous chunk is
        imaged.  `chunk_rows` fixes a uniform chunk size instead.
        """
        g = self.g
        B = vel.shape[0]
        shape = (B, g.n_shots, g.nt, g.nx)
        if (not isinstance(obs_host, torch.Tensor) or obs_host.device.type != 'cpu'
                or obs_host.dtype not in (torch.float32, torch.float64)):
            raise ValueError('obs_host must be a float32 or float64 CPU tensor')
        if tuple(obs_host.shape) != shape:
            raise ValueError(f'obs must have shape {shape}, got {tuple(obs_host.shape)}')
        obs_host = obs_host.contiguous()
        dev = self.device
        f32 = dict(dtype=torch.float32, device=dev)
        host_vel = isinstance(vel, torch.Tensor) and vel.device.type == 'cpu'
        if host_vel:
            if vel.dtype not in (torch.float32, torch.float64) or tuple(vel.shape) != (B, g.nz, g.nx):
                raise ValueError(f'vel must be a float32 or float64 tensor of shape {(B, g.nz, g.nx)}')
            vel_host = vel.contiguous()
            vel = torch.empty(B, g.nz, g.nx, **f32)
        else:
            vel = self._check_in(vel, (B, g.nz, g.nx), 'vel')
        bounds = self._chunks(B, chunk_rows)
        n_chunks = len(bounds)
        chunk = max(b - a for a, b in bounds)
        compute = torch.cuda.current_stream(dev)
        if getattr(self, '_copy_streams', None) is None:
            self._copy_streams = (torch.cuda.Stream(dev), torch.cuda.Stream(dev))
        h2d, d2h = self._copy_streams
        h2d.wait_stream(compute)          # inputs and outputs made on the caller's stream are ready
        dev_obs = [torch.empty(chunk, *shape[1:], **f32) for _ in range(min(2, n_chunks))]
        pinned = obs_host.dtype == torch.float32 and obs_host.is_pinned()
        staging = [] if pinned else [torch.empty(chunk, *shape[1:], dtype=torch.float32, pin_memory=True)
                                     for _ in range(min(2, n_chunks))]
        vel_staging = [torch.empty(chunk, g.nz, g.nx, dtype=torch.float32, pin_memory=True)
                       for _ in range(min(2, n_chunks))] if host_vel else []
        img_dev = torch.empty(B, g.n_shots, g.nz, g.nx, **f32)
        illum_dev = torch.empty_like(img_dev)
        img = torch.empty(img_dev.shape, dtype=torch.float32, pin_memory=True)
        illum = torch.empty_like(img, pin_memory=True)
        flags = torch.zeros(n_chunks, dtype=torch.int32, device=dev)
        copied = [torch.cuda.Event() for _ in dev_obs]
        imaged = [torch.cuda.Event() for _ in dev_obs]
        for k, (a, b) in enumerate(bounds):
            buf = k % len(dev_obs)
            src = obs_host[a:b]
            if (not pinned or host_vel) and k >= len(dev_obs):
                copied[buf].synchronize()              # the staging buffers' previous rows have left
            if not pinned:
                staging[buf][:b - a].copy_(src)
                src = staging[buf][:b - a]
            if host_vel:
                vel_staging[buf][:b - a].copy_(vel_host[a:b])
            with torch.cuda.stream(h2d):
                if k >= len(dev_obs):
                    h2d.wait_event(imaged[buf])        # the device buffer's previous chunk is imaged
                dev_obs[buf][:b - a].copy_(src, non_blocking=True)
                if host_vel:
                    vel[a:b].copy_(vel_staging[buf][:b - a], non_blocking=True)
                copied[buf].record(h2d)
            compute.wait_event(copied[buf])
            self.images(vel[a:b], wavelet, dev_obs[buf][:b - a], None if v_mute is None else v_mute[a:b], t_mute, eps,
                        laplacian, out=(img_dev[a:b], illum_dev[a:b]))
            flags[k:k + 1].copy_(self._ws[:4].view(torch.int32))   # this chunk's device status, kept
            imaged[buf].record(compute)
            with torch.cuda.stream(d2h):
                d2h.wait_event(imaged[buf])
                img[a:b].copy_(img_dev[a:b], non_blocking=True)
                illum[a:b].copy_(illum_dev[a:b], non_blocking=True)
        h2d.synchronize()
        d2h.synchronize()
        compute.synchronize()
        bad = flags.cpu().numpy()
        if (bad == _lib.ERR_NONFINITE).any():
            raise ValueError('observations must be finite')
        if bad.any():
            _lib.check(int(bad[bad != 0][0]), 'device status')
        return img, illum

    def _chunks(self, B, chunk_rows=None):
        """Row ranges [(a, b), ...] of the host-observation pipeline.

        Default: whole rounds of the persistent clusters (rows whose solves fill every cluster), growing
        from one round by x6 per chunk (a chunk's gathers cross PCIe several times faster than the previous
        chunk is imaged) up to a third of the rows or 1 GiB of gathers; the last chunk takes what is left.
        """
        if chunk_rows:
            c = int(chunk_rows)
            return [(a, min(B, a + c)) for a in range(0, B, c)]
        slots = self.plan(B, _lib.MODE_IMAGES)['slots']
        per_round = slots // math.gcd(slots, self.g.n_shots)
        row_bytes = self.g.n_shots * self.g.nt * self.g.nx * 4
        cap = max(1, min(math.ceil(math.ceil(B / per_round) / 3), (1 << 30) // (row_bytes * per_round)))
        out, a, n = [], 0, 1
        while a < B:
            b = min(B, a + min(n, cap) * per_round)
            out.append((a, b))
            a, n = b, n * 6
        return out

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
