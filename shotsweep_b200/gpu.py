"""Drop-in replacement for ShotSweep's ``openfwi/physics/gpu.py`` on B200.

Same module surface as the reference (``DEV``, ``SRC``, ``RICKER``, ``torch``,
``resolve_device``, ``lap``, ``lap_adjoint``, ``fold_edge_padding``,
``imaging_memory_bytes``, ``Sim``, ``calibrate``), same argument meaning,
return types and exceptions; the arithmetic runs in hand-written sm_100a
kernels of ``libshotsweep.so`` reached through its C ABI (``_lib``).  There is
no CPU path: a ``Sim`` on a non-CUDA device raises.

Differences a caller can observe:
  * ``dtype`` must be ``torch.float32`` (the kernels compute in FP32, like the
    reference's default); float64 raises ``ValueError``.
  * ``checkpoint_interval`` only shapes ``forward(store=True)``'s checkpoint
    dictionary: the adjoint keeps a full per-step history in device memory
    instead of recomputing segments, so its results do not depend on it (the
    reference's own test pins that invariance, tests/test_physics.py:76-79).
  * ``imaging_memory_bytes`` reports this implementation's device storage,
    and ``images`` / ``gradient`` keep their storage within it by running at
    most rows*5/SOLVES_PER_SLOT solves at once (a call on 90 or more rows,
    30 models at 3 backgrounds, fills the 45 co-resident clusters of a B200).
"""
from __future__ import annotations

import contextlib
import math

import numpy as np
import torch

from . import _lib, engine
from .constants import DX, DT, NX, NZ, NT, F0, SRC_X

DEV = torch.device('cuda' if torch.cuda.is_available() else 'cpu')    # gpu.py:13 (no MPS on this target)
SRC = [int(round(x / DX)) for x in SRC_X]                               # gpu.py:14
_t = np.arange(NT) * DT
_a = (np.pi * F0 * (_t - 1.2 / F0)) ** 2
RICKER = (1 - 2 * _a) * np.exp(-_a)                                    # gpu.py:15-17


def resolve_device(name='auto'):
    """Same contract as gpu.py:20-30: explicit unavailable devices raise."""
    if name == 'auto':
        return torch.device('cuda' if torch.cuda.is_available() else 'cpu')
    device = torch.device(name)
    if device.type == 'cuda' and not torch.cuda.is_available():
        raise RuntimeError('CUDA was requested, but this PyTorch installation has no available CUDA device')
    if device.type == 'mps' and not torch.backends.mps.is_available():
        raise RuntimeError('MPS was requested, but no MPS device is available')
    if device.type not in ('cpu', 'cuda', 'mps'):
        raise ValueError(f'unsupported device: {name}')
    return device


def _device_op(p, fn32, fn64, out_shape, extra=()):
    """Run a helper kernel on a tensor of any device; the result returns to p's device."""
    if p.dtype not in (torch.float32, torch.float64):
        raise TypeError('only float32 and float64 tensors are supported')
    dev = p.device if p.device.type == 'cuda' else torch.device('cuda')
    _lib.require_cuda(dev)
    x = p.to(dev).contiguous()
    out = torch.empty(out_shape, dtype=p.dtype, device=dev)
    fn = fn32 if p.dtype == torch.float32 else fn64
    with torch.cuda.device(dev):
        _lib.check(fn(_lib.ptr(x), _lib.ptr(out), *extra, _lib.stream_handle(dev)), fn.__name__)
    return out.to(p.device)


def lap(p):
    """4th-order Laplacian x dx^2 with a 2-cell zero border (gpu.py:33-37)."""
    L = _lib.load()
    batch = int(np.prod(p.shape[:-2])) if p.dim() > 2 else 1
    return _device_op(p, L.ss_lap_f32, L.ss_lap_f64, p.shape, (batch, p.shape[-2], p.shape[-1]))


def lap_adjoint(p):
    """Transpose of lap, including its two-cell zero-output boundary (gpu.py:40-53)."""
    L = _lib.load()
    batch = int(np.prod(p.shape[:-2])) if p.dim() > 2 else 1
    return _device_op(p, L.ss_lap_adjoint_f32, L.ss_lap_adjoint_f64, p.shape, (batch, p.shape[-2], p.shape[-1]))


def fold_edge_padding(g, pad):
    """Transpose of np.pad(..., mode='edge') for the last two axes (gpu.py:56-67)."""
    L = _lib.load()
    nz, nx = g.shape[-2] - 2 * pad, g.shape[-1] - 2 * pad
    if nz < 1 or nx < 1:
        raise ValueError('padding larger than the array')
    batch = int(np.prod(g.shape[:-2])) if g.dim() > 2 else 1
    return _device_op(g, L.ss_fold_edge_padding_f32, L.ss_fold_edge_padding_f64, (*g.shape[:-2], nz, nx),
                      (batch, nz, nx, pad))


# A call on B background rows (5 solves each) keeps at most B*5 / SOLVES_PER_SLOT
# solves in flight (at least one), so that its scratch grows with the call
# like the reference's per-row checkpoint storage does.
SOLVES_PER_SLOT = 10


def _slot_bytes(pad):
    """(workspace with one solve in flight, bytes per further solve) for the OpenFWI grid: per-step history,
    trace, gradient rows."""
    L = _lib.load()
    g = engine.geometry(NZ, NX, NT, pad, SRC)
    one = L.ss_workspace_bytes_slots(g, _lib.MODE_IMAGES, 1)
    two = L.ss_workspace_bytes_slots(g, _lib.MODE_IMAGES, 2)
    if one == 0 or two == 0:
        _lib.check(_lib.ERR_UNSUPPORTED, 'ss_workspace_bytes_slots')
    return one, two - one


def max_solves_in_flight(batch):
    """Solves a call on `batch` background rows keeps in flight (Sim.images / Sim.gradient)."""
    return max(1, (int(batch) * len(SRC)) // SOLVES_PER_SLOT)


def imaging_memory_bytes(batch, pad=40, checkpoint_interval=40, bytes_per_value=4):
    """Device storage of one Sim.images / Sim.gradient call on ``batch`` background rows (gpu.py:70-73).

    Linear in ``batch`` like the reference's model, so that a caller's
    ``budget // imaging_memory_bytes(rows)`` (2_process.py:166-171) bounds the
    real use: per row, the gathers, outputs and velocity copies on the device,
    plus 1/SOLVES_PER_SLOT of one solve's scratch per solve, because the call
    keeps at most rows*5/SOLVES_PER_SLOT solves (their per-step histories) in
    flight.  A single row still needs one solve's scratch, hence the floor.
    ``checkpoint_interval`` does not apply: the adjoint reads a full history.
    """
    one_slot, per_slot = _slot_bytes(pad)
    scale = bytes_per_value / 4.0
    row = len(SRC) * (NT * NX + 2 * NZ * NX) * bytes_per_value + NZ * NX * bytes_per_value
    linear = batch * (row + len(SRC) * per_slot * scale / SOLVES_PER_SLOT)
    return int(math.ceil(max(linear, batch * row + one_slot * scale)))


class Sim:
    """Batched FD simulator and exact discrete adjoint (reference: gpu.py:76-210)."""

    def __init__(self, wavelet=None, pad=40, R=1e-5, checkpoint_interval=40,
                 device=None, dtype=torch.float32):
        if pad < 2 or checkpoint_interval < 1:                                 # gpu.py:79-80
            raise ValueError('pad must be >= 2 and checkpoint_interval must be positive')
        if dtype != torch.float32:
            raise ValueError('the B200 kernels compute in float32; dtype must be torch.float32')
        self.pad = pad
        self.R = R
        self.checkpoint_interval = checkpoint_interval
        self.device = DEV if device is None else resolve_device(str(device))
        self.dtype = dtype
        self.wav = np.asarray(RICKER if wavelet is None else wavelet)
        if self.wav.shape != (NT,) or not np.isfinite(self.wav).all() or not np.any(self.wav):   # gpu.py:92-93
            raise ValueError(f'wavelet must contain {NT} finite samples and nonzero energy')
        self.geometry = engine.geometry(NZ, NX, NT, pad, SRC, 1, DX, DT, R)
        self._engine = None
        self._w = None

    # -- plumbing -----------------------------------------------------------
    @property
    def engine(self):
        if self._engine is None:
            _lib.require_cuda(self.device)
            self._engine = engine.Engine(self.geometry, self.device)
        return self._engine

    def _wavelet(self):
        if self._w is None:
            self._w = engine.scaled_wavelet(self.wav, self.engine.device)
        return self._w

    @staticmethod
    def _velocity(v):
        v = np.asarray(v, np.float64)
        t = torch.from_numpy(v)           # the checks on all host threads
        if v.ndim != 3 or v.shape[1:] != (NZ, NX) or not bool(torch.isfinite(t).all()) or bool((t <= 0).any()):
            raise ValueError(f'velocities must be finite positive (B, {NZ}, {NX}) arrays')   # gpu.py:103-104
        return v

    def _to_dev(self, a):
        dev = self.engine.device
        if isinstance(a, torch.Tensor):
            return a.to(dev).to(torch.float32).contiguous()
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev).to(torch.float32).contiguous()

    def _mute(self, v_mute, B):
        if v_mute is None:
            return None
        v_mute = np.asarray(v_mute)
        if not np.isfinite(v_mute).all() or np.any(v_mute <= 0):              # gpu.py:144-145
            raise ValueError('mute velocities must be finite and positive')
        return self._to_dev(np.broadcast_to(np.asarray(v_mute, np.float32), (B,)).copy())

    def _observed(self, obs, B):
        observed = self._to_dev(obs)
        if tuple(observed.shape) != (B, 5, NT, NX):                            # gpu.py:156-157
            raise ValueError(f'observations must be finite with shape {(B, 5, NT, NX)}')
        return observed

    @contextlib.contextmanager
    def _in_flight(self, B):
        """Cap the solves in flight of one call on B rows (imaging_memory_bytes' storage model)."""
        eng = self.engine
        eng.max_slots = max_solves_in_flight(B)
        try:
            yield
        finally:
            eng.max_slots = None

    def _finish(self, B):
        try:
            self.engine.status()
        except ValueError:
            raise ValueError(f'observations must be finite with shape {(B, 5, NT, NX)}') from None

    # -- reference API -------------------------------------------------------
    def forward(self, v, store=False):
        """Return gathers, optional wavefield checkpoints, and squared Courant numbers (gpu.py:117-136).

        Checkpoints hold the states (p0, p1) before every checkpoint_interval-th
        step, as device tensors, like the reference's.
        """
        v = self._velocity(v)
        vd = self._to_dev(v)
        res = self.engine.forward(vd, self._wavelet(), self.checkpoint_interval if store else None)
        checkpoints = None
        if store:
            out, ck = res
            checkpoints = {k * self.checkpoint_interval: (ck[:, :, k, 0], ck[:, :, k, 1]) for k in range(ck.shape[2])}
        else:
            out = res
        c2 = self.engine.c2_field(vd)[:, None]
        return out, checkpoints, c2

    @torch.no_grad()
    def gathers(self, v, chunk=20):
        """Chunked forward returning host arrays (gpu.py:138-140)."""
        return np.concatenate([self.forward(v[i:i + chunk])[0].cpu().numpy() for i in range(0, len(v), chunk)])

    def mute_weights(self, v_mute, t_mute=0.12):
        """Cosine direct-wave mute weights (B,5,NT,NX) on the device (gpu.py:142-150)."""
        v_mute = np.atleast_1d(np.asarray(v_mute))
        return self.engine.mute_weights(self._mute(v_mute, len(v_mute)), t_mute)

    def _gradient(self, v_bg, obs, v_mute=None, t_mute=0.12):
        """Per-shot gradient and illumination as device tensors (gpu.py:152-188)."""
        v = self._velocity(v_bg)
        B = len(v)
        with self._in_flight(B):
            grad, illum = self.engine.gradient(self._to_dev(v), self._wavelet(), self._observed(obs, B),
                                               self._mute(v_mute, B), t_mute)
            self._finish(B)
        return grad, illum

    @torch.no_grad()
    def gradient(self, v_bg, obs, v_mute=None, t_mute=0.12):
        """Per-shot derivative of .5*sum(weight*(sim-obs)**2), with fixed mute weights (gpu.py:190-194)."""
        grad, illum = self._gradient(v_bg, obs, v_mute, t_mute)
        return grad.cpu().numpy(), illum.cpu().numpy()

    @torch.no_grad()
    def images(self, v_bg, obs, v_mute=None, t_mute=0.12, eps=1e-4, laplacian=True):
        """Illumination-normalised negative gradients and source illumination (gpu.py:196-210).

        The direct-wave cosine mute has a 30 ms ramp starting at offset/v_mute
        + t_mute; its weights are fixed during differentiation.
        """
        if eps <= 0:
            raise ValueError('illumination regularization eps must be positive')
        v = self._velocity(v_bg)
        B = len(v)
        with self._in_flight(B):
            return self._images(v, obs, v_mute, t_mute, eps, laplacian)

    def _images(self, v, obs, v_mute, t_mute, eps, laplacian):
        B = len(v)
        host = not (isinstance(obs, torch.Tensor) and obs.is_cuda)
        if host:   # host observations: copies overlapped with imaging, chunk by chunk
            o = obs if isinstance(obs, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(obs))
            if o.dtype not in (torch.float32, torch.float64):   # float64 rows convert chunk by chunk
                o = o.to(torch.float32)
            if tuple(o.shape) != (B, 5, NT, NX):                                   # gpu.py:156-157
                raise ValueError(f'observations must be finite with shape {(B, 5, NT, NX)}')
            try:   # float64 model rows are converted and copied chunk by chunk
                img, illum = self.engine.images_from_host(torch.from_numpy(v), self._wavelet(), o,
                                                          self._mute(v_mute, B), t_mute, eps, laplacian)
            except ValueError:
                raise ValueError(f'observations must be finite with shape {(B, 5, NT, NX)}') from None
            return img.numpy(), illum.numpy()
        img, illum = self.engine.images(self._to_dev(v), self._wavelet(), self._observed(obs, B),
                                        self._mute(v_mute, B), t_mute, eps, laplacian)
        self._finish(B)
        return img.cpu().numpy(), illum.cpu().numpy()


def calibrate(models, gathers, eps=1e-3):
    """One effective source wavelet pooled over training models with known velocity (gpu.py:213-221).

    Forward modelling of the known models runs on the GPU; the pooled
    frequency-domain Wiener filter (cross-spectrum over power spectrum, summed
    over models, shots and receivers, regularised by eps x its peak) is the
    reference's host-side step.
    """
    synthetic = Sim(RICKER).gathers(np.asarray(models, np.float64)).astype(np.float64)
    spec_s = np.fft.rfft(synthetic, axis=2)
    spec_o = np.fft.rfft(np.asarray(gathers, np.float64), axis=2)
    cross = np.einsum('nsfr,nsfr->f', np.conj(spec_s), spec_o)
    power = np.einsum('nsfr,nsfr->f', np.conj(spec_s), spec_s).real
    shaping = cross / (power + eps * power.max())
    return np.fft.irfft(np.fft.rfft(RICKER) * shaping, n=NT)
