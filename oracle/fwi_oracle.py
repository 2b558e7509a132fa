"""TEST INFRASTRUCTURE ONLY - NumPy restatement of the reference's L-BFGS FWI iteration.

archive/toy/slopes/fwi.py:130-164 and slopes.py:20-26 with the oracle simulator
(oracle/oracle.py, float64) for data and gradients; used by tests/ to check
shotsweep_b200/csrc/fwi.cu and shotsweep_b200/fwi.py.  Nothing in the product
imports it.
"""
from __future__ import annotations

import numpy as np


def gauss1d(a, s, axis):
    """slopes.py:20-26."""
    if s <= 0:
        return a
    r = int(3 * s) + 1
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / s) ** 2)
    k /= k.sum()
    a = np.moveaxis(a, axis, -1)
    pad = np.pad(a, [(0, 0)] * (a.ndim - 1) + [(r, r)], mode='edge')
    out = np.zeros_like(a)
    for i, w in enumerate(k):
        out += w * pad[..., i:i + a.shape[-1]]
    return np.moveaxis(out, -1, axis)


def precondition(g, smooth=2.0):
    """fwi.py:142-143 for g [nz, nx]."""
    mute = np.clip((np.arange(g.shape[0]) - 1) / 3.0, 0, 1)[:, None]
    return gauss1d(gauss1d(g * mute, smooth, 0), smooth, 1) * mute


def lbfgs_direction(g, S_hist, Y_hist):
    """fwi.py:130-136."""
    q = g.copy()
    al = []
    for s_, y_ in reversed(list(zip(S_hist, Y_hist))):
        rho = 1.0 / (y_ * s_).sum()
        a_ = rho * (s_ * q).sum()
        q -= a_ * y_
        al.append((rho, a_, s_, y_))
    if S_hist:
        q *= (S_hist[-1] * Y_hist[-1]).sum() / (Y_hist[-1] * Y_hist[-1]).sum()
    for rho, a_, s_, y_ in reversed(al):
        b_ = rho * (y_ * q).sum()
        q += s_ * (a_ - b_)
    return -q


def direction(g, S_hist, Y_hist, cap=50.0):
    """fwi.py:148-151: (d, g.d, history kept)."""
    d = lbfgs_direction(g, S_hist, Y_hist)
    if not S_hist:
        d = d / (np.abs(d).max() + 1e-30) * cap
    keep = True
    if (d * g).sum() >= 0:
        d = -g / (np.abs(g).max() + 1e-30) * cap
        keep = False
    return d, float((d * g).sum()), keep


def fwi(sim, obs, v0, iters, smooth=2.0, mem=6, cap=50.0, c=1e-4, halvings=6, lo=1400.0, hi=4600.0):
    """fwi.py:146-164 for one model with an OracleSim: (v, [J per iteration])."""
    v = np.asarray(v0, np.float64).copy()

    def J_of(vel):
        r = sim.gathers(vel[None])[0] - obs
        return 0.5 * float((r * r).sum())

    def grad(vel):
        g, _ = sim.gradient(vel[None], obs[None])
        return precondition(g[0].sum(0).astype(np.float64), smooth)

    Sh, Yh = [], []
    J, g = J_of(v), grad(v)
    history = [J]
    for _ in range(iters):
        d, gd, keep = direction(g, Sh, Yh, cap)
        if not keep:
            Sh, Yh = [], []
        step, ok = 1.0, False
        for _ in range(halvings):
            vt = np.clip(v + step * d, lo, hi)
            Jt = J_of(vt)
            if Jt < J + c * step * gd:
                ok = True
                break
            step *= 0.5
        if not ok:
            break
        gn = grad(vt)
        sk, yk = vt - v, gn - g
        if (sk * yk).sum() > 1e-12:
            Sh.append(sk)
            Yh.append(yk)
            Sh, Yh = Sh[-mem:], Yh[-mem:]
        v, J, g = vt, Jt, gn
        history.append(J)
    return v, history


def lowpass(x, fc, axis=1, dt=1e-3):
    """fwi.py:78-83: Gaussian low-pass exp(-0.5 (f/fc)^4) along `axis`; fc None leaves x unchanged."""
    if fc is None:
        return x
    n = x.shape[axis]
    f = np.fft.rfftfreq(n, dt)
    h = np.exp(-0.5 * (f / fc) ** 4)
    shape = [1] * x.ndim
    shape[axis] = len(f)
    return np.fft.irfft(np.fft.rfft(x, axis=axis) * h.reshape(shape), n=n, axis=axis)


def estimate_source(sim, obs, ricker, eps=1e-3):
    """fwi.py:85-90 for one model's gathers [shots, nt, nx]: the Ricker shaped by the pooled Wiener filter."""
    sf = np.fft.rfft(sim, axis=1)
    of = np.fft.rfft(obs, axis=1)
    num = (np.conj(sf) * of).sum(axis=(0, 2))
    den = (np.abs(sf) ** 2).sum(axis=(0, 2))
    shaping = num / (den + eps * den.max())
    return np.fft.irfft(np.fft.rfft(ricker) * shaping, n=len(ricker))


def fwi_bands(make_sim, obs, v0, ricker, bands=(8.0, None), iters=(10, 25), **kw):
    """fwi.py:144-163 for one model: per band, low-passed gathers and Ricker, a Wiener-estimated wavelet,
    then the L-BFGS loop with a fresh history.  make_sim(wavelet) -> OracleSim injecting that (unscaled)
    wavelet.  Returns (v, [(band, wavelet, [J per iteration])])."""
    v = np.asarray(v0, np.float64).copy()
    out = []
    for k, (fc, nit) in enumerate(zip(bands, iters)):
        obs_b = lowpass(np.asarray(obs, np.float64), fc)
        ric = lowpass(np.asarray(ricker, np.float64)[None, :, None], fc)[0, :, 0]
        wav = estimate_source(make_sim(ric).gathers(v[None])[0].astype(np.float64), obs_b, ric)
        v, hist = fwi(make_sim(wav), obs_b, v, nit, **kw)
        out.append((k, wav, hist))
    return v, out
