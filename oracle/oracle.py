"""CPU oracle for the ShotSweep physics hot path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker (or as the timed
CPU port of the reference).  The product path in ``shotsweep_b200`` never
imports it and has no CPU fallback.

What it is: a parameterised restatement, in PyTorch CPU eager ops, of the
reference simulator ``openfwi/physics/gpu.py`` (ShotSweep): 4th-order-space /
2nd-order-time constant-density acoustic finite differences with a damped
absorbing layer, v^2-scaled Ricker injection, surface receivers, and the
checkpointed exact discrete adjoint that yields per-shot gradients,
illumination and RTM images.  The reference hard-wires a 70x70 grid, 1000
steps and 5 shots (openfwi/physics/constants.py:4-5, gpu.py:59,95-96,103,126);
this restatement takes them as parameters so that odd sizes can be checked.
Every function cites the reference lines it follows.  Run in float64 it is the
parity oracle; run in float32 with all host threads it is the CPU port whose
speed stands in for the reference's own CPU path.

Parity pin: ``tests/golden/make_golden.py`` runs the reference itself (float64,
CPU) on seeded inputs and stores its outputs under ``tests/golden``;
``tests/test_oracle.py`` checks this module against those fixtures at the
reference's own geometry.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import torch

# openfwi/physics/constants.py:4-7
DX = 10.0
DT = 1e-3
NX = NZ = 70
NT = 1000
F0 = 15.0
SRC_COLS = (0, 17, 34, 52, 69)
VMAX_DAMPING = 4500.0      # gpu.py:88 (the 4500 in the damping constant)
AMP_REF = 2000.0           # gpu.py:108,168 (source strength normalisation)


@dataclasses.dataclass(frozen=True)
class Geometry:
    """Acquisition and grid; defaults are the OpenFWI layout of the reference."""
    nz: int = NZ
    nx: int = NX
    nt: int = NT
    dx: float = DX
    dt: float = DT
    shot_cols: tuple = SRC_COLS
    src_row: int = 1          # sources and receivers 10 m deep (constants.py:6; gpu.py:114,134)

    @property
    def n_shots(self):
        return len(self.shot_cols)


def shot_columns(nx, n_shots):
    """Surface source columns: round(linspace(0, nx-1, ns)); gives (0,17,34,52,69) at 70/5 (gpu.py:14)."""
    return tuple(int(c) for c in np.round(np.linspace(0, nx - 1, n_shots)))


def ricker(nt=NT, dt=DT, f0=F0):
    """Ricker wavelet delayed by 1.2/f0 (gpu.py:15-17)."""
    t = np.arange(nt) * dt
    a = (np.pi * f0 * (t - 1.2 / f0)) ** 2
    return (1 - 2 * a) * np.exp(-a)


def damping_profile(n, pad):
    """Normalised distance into the absorbing layer along one axis (gpu.py:85-87)."""
    i = np.arange(n)
    return np.clip(np.maximum(pad - i, i - (n - 1 - pad)), 0, None) / pad


def damping(nzp, nxp, pad, dx=DX, dt=DT, R=1e-5):
    """A = 1/(1+a), B = 1-a with a = 3*4500/(2*pad*dx)*ln(1/R)*(dz^2+dx^2)*dt/2 (gpu.py:85-90)."""
    dz = damping_profile(nzp, pad)
    dxp = damping_profile(nxp, pad)
    a = 3 * VMAX_DAMPING / (2 * pad * dx) * np.log(1 / R) * (dz[:, None] ** 2 + dxp[None, :] ** 2) * dt / 2
    return 1 / (1 + a), 1 - a


def lap(p):
    """4th-order 5-point-per-axis Laplacian times dx^2, zero on a 2-cell border (gpu.py:33-37)."""
    out = torch.zeros_like(p)
    c = p[..., 2:-2, 2:-2]
    z = -p[..., :-4, 2:-2] + 16 * p[..., 1:-3, 2:-2] - 30 * c + 16 * p[..., 3:-1, 2:-2] - p[..., 4:, 2:-2]
    x = -p[..., 2:-2, :-4] + 16 * p[..., 2:-2, 1:-3] - 30 * c + 16 * p[..., 2:-2, 3:-1] - p[..., 2:-2, 4:]
    out[..., 2:-2, 2:-2] = (z + x) / 12
    return out


def lap_adjoint(p):
    """Exact transpose of ``lap`` including its zero border, in scatter form (gpu.py:40-53)."""
    out = torch.zeros_like(p)
    q = p[..., 2:-2, 2:-2] / 12
    for dz, w in ((-2, -1), (-1, 16), (1, 16), (2, -1)):
        out[..., 2 + dz:out.shape[-2] - 2 + dz, 2:-2] += w * q
    for dxs, w in ((-2, -1), (-1, 16), (1, 16), (2, -1)):
        out[..., 2:-2, 2 + dxs:out.shape[-1] - 2 + dxs] += w * q
    out[..., 2:-2, 2:-2] -= 60 * q
    return out


def fold_edge_padding(g, pad, nz=NZ, nx=NX):
    """Transpose of np.pad(mode='edge') on the last two axes (gpu.py:56-67)."""
    p = pad
    out = g[..., p:p + nz, p:p + nx].clone()
    out[..., 0, :] += g[..., :p, p:p + nx].sum(-2)
    out[..., -1, :] += g[..., p + nz:, p:p + nx].sum(-2)
    out[..., :, 0] += g[..., p:p + nz, :p].sum(-1)
    out[..., :, -1] += g[..., p:p + nz, p + nx:].sum(-1)
    for zi, zs in ((0, slice(None, p)), (-1, slice(p + nz, None))):
        for xi, xs in ((0, slice(None, p)), (-1, slice(p + nx, None))):
            out[..., zi, xi] += g[..., zs, xs].sum((-2, -1))
    return out


def imaging_memory_bytes(batch, pad=40, checkpoint_interval=40, bytes_per_value=4, geom=Geometry()):
    """Storage model of the checkpointed imaging path (gpu.py:70-73)."""
    fields = 2 * math.ceil(geom.nt / checkpoint_interval) + checkpoint_interval + 24
    return int(batch * geom.n_shots * bytes_per_value *
               ((geom.nz + 2 * pad) * (geom.nx + 2 * pad) * fields + 3 * geom.nt * geom.nx))


class OracleSim:
    """Restatement of ``gpu.Sim`` (gpu.py:76-210) on the CPU for any ``Geometry``."""

    def __init__(self, wavelet=None, pad=40, R=1e-5, checkpoint_interval=40,
                 dtype=torch.float64, geom=Geometry()):
        if pad < 2 or checkpoint_interval < 1:                         # gpu.py:79-80
            raise ValueError('pad must be >= 2 and checkpoint_interval must be positive')
        self.g = geom
        self.pad = pad
        self.checkpoint_interval = checkpoint_interval
        self.dtype = dtype
        self.nzp, self.nxp = geom.nz + 2 * pad, geom.nx + 2 * pad
        A, B = damping(self.nzp, self.nxp, pad, geom.dx, geom.dt, R)
        self.A, self.B = self._t(A), self._t(B)
        wav = np.asarray(ricker(geom.nt, geom.dt) if wavelet is None else wavelet)
        if wav.shape != (geom.nt,) or not np.isfinite(wav).all() or not np.any(wav):  # gpu.py:92-93
            raise ValueError(f'wavelet must contain {geom.nt} finite samples and nonzero energy')
        self.wav = wav
        self.w = self._t(wav * 1e3)                                      # gpu.py:94
        self.si = torch.arange(geom.n_shots)
        self.sx = torch.tensor(geom.shot_cols) + pad                     # gpu.py:96
        self.row = pad + geom.src_row

    def _t(self, value):
        return torch.as_tensor(value, dtype=self.dtype)

    def _setup(self, v):
        """c2 = edge-padded v^2 (dt/dx)^2 and v^2-scaled source strength (gpu.py:101-109)."""
        g = self.g
        v = np.asarray(v, np.float64)
        if v.ndim != 3 or v.shape[1:] != (g.nz, g.nx) or not np.isfinite(v).all() or np.any(v <= 0):
            raise ValueError(f'velocities must be finite positive (B, {g.nz}, {g.nx}) arrays')
        p = self.pad
        vp = np.pad(v, ((0, 0), (p, p), (p, p)), mode='edge')
        c2 = self._t(vp ** 2 * (g.dt / g.dx) ** 2)[:, None]
        amp = self._t((v[:, g.src_row, list(g.shot_cols)] / AMP_REF) ** 2)
        return c2, amp

    def _step(self, p0, p1, c2, amp, it):
        """One leapfrog step with damping, then source injection (gpu.py:111-115)."""
        L = lap(p1)
        p2 = (2 * p1 - self.B * p0 + c2 * L) * self.A
        p2[:, self.si, self.row, self.sx] += self.w[it] * amp
        return p2, L

    def forward(self, v, store=False):
        """Gathers (B,S,nt,nx), optional checkpoints {it: (p0,p1)}, c2 (gpu.py:117-136)."""
        g, p = self.g, self.pad
        c2, amp = self._setup(v)
        p0 = torch.zeros(len(v), g.n_shots, self.nzp, self.nxp, dtype=self.dtype)
        p1 = torch.zeros_like(p0)
        out = torch.zeros(len(v), g.n_shots, g.nt, g.nx, dtype=self.dtype)
        checkpoints = {} if store else None
        for it in range(g.nt):
            if store and it % self.checkpoint_interval == 0:
                checkpoints[it] = (p0.clone(), p1.clone())
            p2, _ = self._step(p0, p1, c2, amp, it)
            out[:, :, it] = p2[:, :, self.row, p:p + g.nx]
            p0, p1 = p1, p2
        return out, checkpoints, c2

    @torch.no_grad()
    def gathers(self, v, chunk=20):
        """Chunked forward returning host arrays (gpu.py:138-140)."""
        return np.concatenate([self.forward(v[i:i + chunk])[0].numpy() for i in range(0, len(v), chunk)])

    def mute_weights(self, v_mute, t_mute=0.12):
        """Cosine direct-wave mute with a 30 ms ramp from offset/v_mute + t_mute (gpu.py:142-150)."""
        g = self.g
        v_mute = np.asarray(v_mute)
        if not np.isfinite(v_mute).all() or np.any(v_mute <= 0):
            raise ValueError('mute velocities must be finite and positive')
        src_x = np.asarray(g.shot_cols) * g.dx
        h = self._t(np.abs(np.arange(g.nx)[None, :] * g.dx - src_x[:, None]))
        t = torch.arange(g.nt, dtype=self.dtype)[:, None] * g.dt
        t0 = h[None] / self._t(v_mute)[:, None, None] + t_mute
        ramp = torch.clamp((t[None, None] - t0[:, :, None, :]) / 0.03, 0, 1)
        return 0.5 - 0.5 * torch.cos(np.pi * ramp)

    def _gradient(self, v_bg, obs, v_mute=None, t_mute=0.12):
        """Checkpointed exact discrete adjoint (gpu.py:152-188)."""
        g, p = self.g, self.pad
        sim, checkpoints, c2 = self.forward(v_bg, store=True)
        observed = self._t(np.asarray(obs))
        if observed.shape != sim.shape or not torch.isfinite(observed).all():
            raise ValueError(f'observations must be finite with shape {tuple(sim.shape)}')
        res = sim - observed
        if v_mute is not None:
            res *= self.mute_weights(v_mute, t_mute)
        _, amp = self._setup(v_bg)
        shape = (len(v_bg), g.n_shots, self.nzp, self.nxp)
        m1 = torch.zeros(shape, dtype=self.dtype)
        m2 = torch.zeros_like(m1)
        grad_acc = torch.zeros_like(m1)
        source_grad = torch.zeros(len(v_bg), g.n_shots, dtype=self.dtype)
        illum = torch.zeros(len(v_bg), g.n_shots, g.nz, g.nx, dtype=self.dtype)
        source_derivative = 2 * self._t(np.asarray(v_bg)[:, g.src_row, list(g.shot_cols)]) / AMP_REF ** 2
        AB = self.A * self.B
        for start in reversed(list(checkpoints)):
            p0, p1 = checkpoints.pop(start)
            end = min(start + self.checkpoint_interval, g.nt)
            laplacians = []
            for it in range(start, end):                                  # segment recompute
                p2, L = self._step(p0, p1, c2, amp, it)
                laplacians.append(L)
                p0, p1 = p1, p2
            for it in range(end - 1, start - 1, -1):                      # adjoint sweep
                L = laplacians.pop()
                mu = 2 * self.A * m1 + lap_adjoint(c2 * self.A * m1) - AB * m2
                mu[:, :, self.row, p:p + g.nx] += res[:, :, it]
                grad_acc += self.A * mu * L
                source_grad += mu[:, self.si, self.row, self.sx] * self.w[it] * source_derivative
                illum += L[..., p:p + g.nz, p:p + g.nx] ** 2
                m2, m1 = m1, mu
        vp = self._t(np.pad(np.asarray(v_bg, np.float64), ((0, 0), (p, p), (p, p)), mode='edge'))[:, None]
        grad = fold_edge_padding(grad_acc * 2 * vp * (g.dt / g.dx) ** 2, p, g.nz, g.nx)
        grad[:, self.si, g.src_row, torch.tensor(g.shot_cols)] += source_grad
        return grad, illum

    @torch.no_grad()
    def gradient(self, v_bg, obs, v_mute=None, t_mute=0.12):
        """Per-shot d/dv of 0.5*sum(w*(sim-obs)^2) with fixed mute weights (gpu.py:190-194)."""
        grad, illum = self._gradient(v_bg, obs, v_mute, t_mute)
        return grad.numpy(), illum.numpy()

    @torch.no_grad()
    def images(self, v_bg, obs, v_mute=None, t_mute=0.12, eps=1e-4, laplacian=True):
        """Illumination-normalised negative gradients, optionally Laplacian filtered (gpu.py:196-210)."""
        if eps <= 0:
            raise ValueError('illumination regularization eps must be positive')
        grad, illum = self._gradient(v_bg, obs, v_mute, t_mute)
        return image_epilogue(grad, illum, eps, laplacian).numpy(), illum.numpy()


def image_epilogue(grad, illum, eps=1e-4, laplacian=True):
    """den = illum + eps*max(illum); img = -grad/den; img = -lap(replicate-pad(img)) (gpu.py:206-209)."""
    denominator = illum + eps * illum.amax(dim=(-2, -1), keepdim=True)
    img = -grad / denominator.clamp_min(torch.finfo(grad.dtype).tiny)
    if laplacian:
        shape = img.shape
        flat = img.reshape(-1, 1, *shape[-2:])
        padded = torch.nn.functional.pad(flat, (2, 2, 2, 2), mode='replicate').reshape(*shape[:-2], shape[-2] + 4, shape[-1] + 4)
        img = -lap(padded)[..., 2:-2, 2:-2]
    return img


def backgrounds(v_surface, trend, rhos=(0.6, 1.0, 1.4), nx=NX):
    """Laterally constant slow/medium/fast backgrounds clip(v_s + rho*trend) (openfwi/physics/background.py:97-99)."""
    return np.stack([np.tile(np.clip(v_surface + r * trend, 1500.0, 4500.0)[:, None], (1, nx)) for r in rhos])


def depth_trend(models):
    """Mean over models of mean_x v(z) - mean_x v(0) (openfwi/physics/background.py:91-94)."""
    m = np.asarray(models, np.float64)
    return (m.mean(2) - m[:, :1, :].mean(2)).mean(0)


def calibrate(models, gathers, eps=1e-3, dtype=torch.float32, geom=Geometry()):
    """Pooled frequency-domain Wiener estimate of the effective source wavelet (gpu.py:213-221).

    The reference simulates the known models with the Ricker in its default
    float32 (``Sim(RICKER)``, gpu.py:215), then shapes the Ricker by the
    cross-spectrum of synthetics and observations over their power spectrum,
    both summed over models, shots and receivers, regularised by eps x the
    power spectrum's peak."""
    sims = OracleSim(ricker(geom.nt, geom.dt), dtype=dtype, geom=geom).gathers(np.asarray(models, np.float64))
    sf = np.fft.rfft(sims, axis=2)
    of = np.fft.rfft(np.asarray(gathers, np.float64), axis=2)
    num = (np.conj(sf) * of).sum(axis=(0, 1, 3))
    den = (np.abs(sf) ** 2).sum(axis=(0, 1, 3))
    return np.fft.irfft(np.fft.rfft(ricker(geom.nt, geom.dt)) * num / (den + eps * den.max()), n=geom.nt)
