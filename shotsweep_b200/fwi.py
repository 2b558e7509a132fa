"""L-BFGS full-waveform inversion of many models at once on the GPU.

The iteration of the reference's FWI (archive/toy/slopes/fwi.py:130-164), with
the library's simulator for the data (the reference's gpu.Sim physics, all
shots, no mute) and its exact adjoint for the gradient of J = 0.5 sum (F(v) - d)^2:

    g <- precondition(gradient)            mute of the top rows, Gaussian smoothing (sigma 2 cells)
    d <- two-loop L-BFGS direction         memory 6; first step capped at 50 m/s; steepest descent
                                           (max 50 m/s) when g.d >= 0
    Armijo backtracking on v + step d      clipped to 1400-4600 m/s; c = 1e-4; at most 6 halvings;
                                           a model whose search fails stops, as the reference does
    (s, y) pushed when s.y > 1e-12

Every model runs its own L-BFGS (its own history, step and stopping), batched
in the kernels; only per-model scalars (misfits, g.d, steps) visit the host.

``run_bands`` is the reference's multiscale loop (fwi.py:144-163): per frequency
band (default a Gaussian low-pass at 8 Hz, then the full band) the gathers and
the Ricker are low-passed, each model's source wavelet is estimated by a Wiener
filter between its simulated and observed gathers (fwi.py:85-90), and L-BFGS
runs with a fresh history, each model with its own wavelet.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib

LO, HI = 1400.0, 4600.0
BANDS, BAND_ITERS = (8.0, None), (10, 25)     # fwi.py:138


def lowpass(x, fc, dt=1e-3):
    """Gaussian low-pass exp(-0.5 (f/fc)^4) along the time axis (fwi.py:78-83), float64 FFTs.

    x: gathers [..., nt, nx] on the device (returned float32) or a wavelet [nt] as a NumPy array
    (returned float64).  fc None: x unchanged."""
    if fc is None:
        return x
    if isinstance(x, torch.Tensor):
        n = x.shape[-2]
        f = torch.fft.rfftfreq(n, dt, dtype=torch.float64, device=x.device)
        h = torch.exp(-0.5 * (f / fc) ** 4)
        return torch.fft.irfft(torch.fft.rfft(x.double(), dim=-2) * h[:, None], n=n, dim=-2).float()
    x = np.asarray(x, np.float64)
    f = np.fft.rfftfreq(len(x), dt)
    return np.fft.irfft(np.fft.rfft(x) * np.exp(-0.5 * (f / fc) ** 4), n=len(x))


def estimate_wavelets(sim, obs, ricker, eps=1e-3):
    """Each model's effective source (fwi.py:85-90): the Ricker shaped by the Wiener filter
    sum conj(S) O / (sum |S|^2 + eps max) over the model's shots and receivers.

    sim, obs: [B, S, nt, nx] on the device; ricker: [nt] (the wavelet `sim` was made with, unscaled).
    Returns [B, nt] float64 on the device, unscaled."""
    nt = sim.shape[2]
    sf = torch.fft.rfft(sim.double(), dim=2)
    of = torch.fft.rfft(obs.double(), dim=2)
    num = (sf.conj() * of).sum(dim=(1, 3))
    den = (sf.real ** 2 + sf.imag ** 2).sum(dim=(1, 3))
    shaping = num / (den + eps * den.max(dim=1, keepdim=True).values)
    r = torch.fft.rfft(torch.as_tensor(np.asarray(ricker, np.float64), device=sim.device))
    return torch.fft.irfft(r[None] * shaping, n=nt, dim=1)


def scaled(w):
    """Injected samples: wavelet x 1e3 in float64, then float32 (gpu.py:94)."""
    if isinstance(w, torch.Tensor):
        return (w.double() * 1e3).float().contiguous()
    return torch.as_tensor(np.asarray(w, np.float64) * 1e3, dtype=torch.float32)


class BatchFWI:
    """wavelet: scaled source samples [nt] for every model, or [B, nt] (one per model)."""

    def __init__(self, eng, wavelet, obs, mem=6, smooth=2.0, cap=50.0, c=1e-4, halvings=6):
        self.eng, self.w, self.obs = eng, wavelet, obs.contiguous()
        self.dev = eng.device
        self.B = obs.shape[0]
        self.n = eng.g.nz * eng.g.nx
        self.mem, self.smooth, self.cap, self.c, self.halvings = mem, smooth, cap, c, halvings
        f32 = dict(dtype=torch.float32, device=self.dev)
        i32 = dict(dtype=torch.int32, device=self.dev)
        B, n = self.B, self.n
        self.v = torch.empty(B, n, **f32)
        self.vt = torch.empty(B, n, **f32)
        self.g = torch.empty(B, n, **f32)
        self.gn = torch.empty(B, n, **f32)
        self.d = torch.empty(B, n, **f32)
        self.S = torch.zeros(B, mem, n, **f32)
        self.Y = torch.zeros(B, mem, n, **f32)
        self.count = torch.zeros(B, **i32)
        self.next = torch.zeros(B, **i32)
        self.J = torch.empty(B, dtype=torch.float64, device=self.dev)
        self.Jt = torch.empty_like(self.J)
        self.gd = torch.empty_like(self.J)
        self.L = _lib.load()
        self.per = int(np.prod(obs.shape[1:]))

    def _s(self):
        return _lib.stream_handle(self.dev)

    def misfit(self, vel, out):
        sim = self.eng.forward(vel.view(self.B, self.eng.g.nz, self.eng.g.nx), self.w)
        _lib.check(self.L.ss_fwi_misfit(_lib.ptr(sim), _lib.ptr(self.obs), self.B, self.per, _lib.ptr(out), self._s()),
                   'ss_fwi_misfit')
        return out

    def gradient(self, vel, out):
        grad, _ = self.eng.gradient(vel.view(self.B, self.eng.g.nz, self.eng.g.nx), self.w, self.obs)
        _lib.check(self.L.ss_fwi_precondition(_lib.ptr(grad), self.B, self.eng.g.n_shots, self.eng.g.nz, self.eng.g.nx,
                                              self.smooth, _lib.ptr(out), self._s()), 'ss_fwi_precondition')
        return out

    def run(self, v0, iters=50, callback=None):
        """Invert from v0 [B, nz, nx]; returns (v, per-iteration [(seconds, J per model)])."""
        B = self.B
        t0 = time.perf_counter()
        self.v.copy_(v0.reshape(B, -1))
        self.count.zero_()
        self.next.zero_()
        self.misfit(self.v, self.J)
        self.gradient(self.v, self.g)
        active = np.ones(B, bool)
        torch.cuda.synchronize(self.dev)
        history = [(time.perf_counter() - t0, self.J.cpu().numpy().copy())]
        act_d = torch.ones(B, dtype=torch.int32, device=self.dev)
        for it in range(iters):
            if not active.any():
                history.append((time.perf_counter() - t0, history[-1][1]))
                continue
            act_d.copy_(torch.from_numpy(active.astype(np.int32)))
            _lib.check(self.L.ss_lbfgs_direction(_lib.ptr(self.g), _lib.ptr(self.S), _lib.ptr(self.Y),
                                                 _lib.ptr(self.count), _lib.ptr(self.next), _lib.ptr(act_d), B, self.n,
                                                 self.mem, self.cap, _lib.ptr(self.d), _lib.ptr(self.gd), self._s()),
                       'ss_lbfgs_direction')
            J = self.J.cpu().numpy()
            gd = self.gd.cpu().numpy()
            step = np.ones(B, np.float32)
            ok = np.zeros(B, bool)
            self.vt.copy_(self.v)
            for _ in range(self.halvings):
                todo = active & ~ok
                if not todo.any():
                    break
                mask = torch.from_numpy(todo.astype(np.int32)).to(self.dev)     # referenced until the launch ran
                step_d = torch.from_numpy(step).to(self.dev)
                _lib.check(self.L.ss_fwi_trial(_lib.ptr(self.v), _lib.ptr(self.d), _lib.ptr(step_d), _lib.ptr(mask),
                                               B, self.n, LO, HI, _lib.ptr(self.vt), self._s()), 'ss_fwi_trial')
                Jt = self.misfit(self.vt, self.Jt).cpu().numpy()
                accept = todo & (Jt < J + self.c * step * gd)
                ok |= accept
                J = np.where(accept, Jt, J)
                step = np.where(todo & ~accept, step * 0.5, step).astype(np.float32)
            active &= ok
            self.gradient(self.vt, self.gn)
            acc = torch.from_numpy(ok.astype(np.int32)).to(self.dev)
            _lib.check(self.L.ss_lbfgs_push(_lib.ptr(self.v), _lib.ptr(self.vt), _lib.ptr(self.g), _lib.ptr(self.gn),
                                            _lib.ptr(self.S), _lib.ptr(self.Y), _lib.ptr(self.count),
                                            _lib.ptr(self.next), _lib.ptr(acc), B, self.n, self.mem, self._s()),
                       'ss_lbfgs_push')
            self.J.copy_(torch.from_numpy(J))
            torch.cuda.synchronize(self.dev)
            history.append((time.perf_counter() - t0, J.copy()))
            if callback:
                callback(it, J)
        self.eng.status()
        return self.v.view(B, self.eng.g.nz, self.eng.g.nx).clone(), history

    def run_bands(self, v0, ricker, bands=BANDS, iters=BAND_ITERS, eps=1e-3, callback=None):
        """Multiscale FWI from v0 [B, nz, nx] (fwi.py:144-163).

        ricker: the unscaled source wavelet [nt] that the bands are cut from.  Returns (v, history) with
        history entries (seconds since the start, J per model, band index); J is the misfit against the
        band's low-passed gathers, so only entries of one band compare."""
        obs_full, w_full = self.obs, self.w
        t0 = time.perf_counter()
        history, v = [], v0
        self.wavelets = []
        try:
            for k, (fc, nit) in enumerate(zip(bands, iters)):
                self.obs = lowpass(obs_full, fc).contiguous()
                ric = lowpass(ricker, fc)
                sim = self.eng.forward(v.reshape(self.B, self.eng.g.nz, self.eng.g.nx).contiguous(),
                                       scaled(ric).to(self.dev))
                self.w = scaled(estimate_wavelets(sim, self.obs, ric, eps))
                del sim
                self.wavelets.append(self.w)
                start = time.perf_counter() - t0          # the band's filtering and estimate included
                v, h = self.run(v, nit, callback=callback)
                history += [(start + t, J, k) for t, J in h]
        finally:
            self.obs, self.w = obs_full, w_full
        return v, history
