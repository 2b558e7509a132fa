"""Learned proposal + FWI: train on simulator gathers, propose, accept by forward misfit, refine by L-BFGS.

    res = run(n_train=20000, n_test=256, steps=6000, iters=50)                 # one full band
    res = run(..., iters=(10, 25), bands=(8.0, None))                           # the reference's two bands

1. Training data: `n_train` seeded models from the synthetic families (an equal mix of
   layered, curved, faulted and textured), their gathers simulated by the library's
   forward kernel and kept on the device in the stored float16 form sign(g) log1p(|g|)
   (3_train.py:157); the normalisation scale is the largest stored magnitude (3_train.py:513).
2. Training: ``proposal.ProposalNet`` with AdamW (lr 5e-4 with cosine decay, weight decay
   1e-4), L1 loss on (v - 3000) / 1500, batches drawn from a seeded permutation; one training
   step is one CUDA-graph replay.
3. Held-out models (`n_test`, other seeds): the network's velocity proposal, and the medium
   background (surface velocity from the first-arrival picker + 1.0 x the training depth trend,
   background.py:97-99; the training models' mean surface velocity where the picker refuses).
4. Acceptance by forward misfit: each model starts FWI from the proposal if its data misfit is
   below the background's, otherwise from the background (the fallback is plain FWI).
5. ``fwi.BatchFWI.run_bands`` from both starts: L-BFGS for `iters` iterations in the full band
   (an int), or the reference's multiscale schedule (fwi.py:138-163: `bands` such as an 8 Hz
   low-pass then the full band, `iters` per band, each model with its own Wiener-estimated wavelet
   per band).  Plain FWI runs the schedule as given.  With several bands the learned method runs
   it only for the models whose proposal was refused (the fallback is plain FWI, from the
   background, every band); an accepted proposal already holds the long wavelengths that the
   low band exists to recover, so its model goes straight to the full band, with as many
   iterations as the whole schedule.  The fallback group runs first, so its time counts in full.
   The time-to-misfit is the wall time the learned start (inference and acceptance included)
   needs to reach plain FWI's final full-band total misfit over all held-out models, against
   plain FWI's own wall time; only full-band misfits are compared.  `time_ratio_inclusive` adds
   the data simulation and the training to the learned side.
"""
from __future__ import annotations

import math
import time

import numpy as np
import torch

from . import background as BG
from . import engine, gpu, synth, train_inputs as TI
from .fwi import BatchFWI
from .proposal import OUT, ProposalNet


def simulate_stored(eng, models, w, chunk=1000):
    """Stored float16 gathers [n, 5, 1000, 70] (device) of models [n, 70, 70]."""
    out = torch.empty(len(models), eng.g.n_shots, eng.g.nt, eng.g.nx, dtype=torch.float16, device=eng.device)
    for a in range(0, len(models), chunk):
        g = eng.forward(torch.tensor(models[a:a + chunk], dtype=torch.float32, device=eng.device), w)
        out[a:a + len(g)] = TI.stored_gathers(g)
    eng.status()
    return out


def train(net, stored, targets, scale, steps, lr=5e-4, seed=0, log_every=500, log=None):
    """`steps` AdamW steps on batches of net.B samples; returns the loss of every `log_every`-th step."""
    n = stored.shape[0]
    rng = np.random.default_rng([seed, 5])
    perm = torch.tensor(np.concatenate([rng.permutation(n) for _ in range(math.ceil(steps * net.B / n) + 1)]),
                        dtype=torch.int32, device=net.dev)
    net.ids.copy_(perm[:net.B])
    net.train_step(stored, scale, targets)          # warm-up outside capture (attributes, tensor maps)
    torch.cuda.synchronize(net.dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        net.train_step(stored, scale, targets)
    losses = []
    for s in range(1, steps):
        net.ids.copy_(perm[s * net.B:(s + 1) * net.B])
        net.lr.fill_(lr * 0.5 * (1 + math.cos(math.pi * s / steps)))
        graph.replay()
        if s % log_every == 0 or s == steps - 1:
            losses.append((s, net.loss_sum.item() / (net.B * OUT * OUT)))
            if log:
                log(s, losses[-1][1])
    net.check()
    del graph
    return losses


def predict(net, stored, scale):
    """Velocities [n, 70, 70] (float32, device) proposed for every stored sample."""
    n = stored.shape[0]
    out = torch.empty(n, OUT, OUT, dtype=torch.float32, device=net.dev)
    for a in range(0, n, net.B):
        ids = torch.arange(a, a + net.B, dtype=torch.int32, device=net.dev).clamp_max(n - 1)
        net.ids.copy_(ids)
        net.load_batch(stored, scale)
        pred = net.forward()
        k = min(net.B, n - a)
        out[a:a + k] = pred[:k] * 1500.0 + 3000.0
    return out


def medium_backgrounds(gathers, trend, fallback_vs, device):
    """Medium (rho = 1.0) backgrounds from picked surface velocities; the fallback where the picker refuses."""
    est = BG.surface_estimates(gathers)
    vs = np.array([e.velocity if e.status == 0 else fallback_vs for e in est])
    return BG.backgrounds(vs, trend, rhos=(1.0,), device=device)[:, 0], vs, np.array([e.status for e in est])


def norm_mae(v, truth):
    """Mean absolute error of velocities normalised to [-1, 1] (the reference's metric, fwi.py norm/metrics)."""
    a = (np.clip(v, 1500, 4500) - 1500) / 3000 * 2 - 1
    b = (np.clip(truth, 1500, 4500) - 1500) / 3000 * 2 - 1
    return float(np.abs(a - b).mean())


def learned_multiscale(eng, w, obs, prop, bg, use, bands, iters, propose_s):
    """The learned side of a multiscale run: refused proposals fall back to plain FWI over every band
    (run first), accepted ones go straight to the full band for sum(iters) iterations.  Returns the
    final models and the curve [(seconds since the proposal started, total full-band misfit)]."""
    acc, rej = np.flatnonzero(use), np.flatnonzero(~use)
    dev = obs.device
    v = torch.empty_like(bg)
    t_rej, j_rej = 0.0, 0.0
    if len(rej):
        ri = torch.tensor(rej, device=dev)
        v_r, h_r = BatchFWI(eng, w, obs[ri].contiguous()).run_bands(bg[ri].contiguous(), gpu.RICKER, bands, iters)
        v[ri] = v_r
        t_rej = h_r[-1][0]
        j_rej = float(h_r[-1][1].sum())
    curve = [(propose_s + t_rej, float('inf'))]
    if len(acc):
        ai = torch.tensor(acc, device=dev)
        v_a, h_a = BatchFWI(eng, w, obs[ai].contiguous()).run_bands(prop[ai].contiguous(), gpu.RICKER,
                                                                   (bands[-1],), (int(sum(iters)),))
        v[ai] = v_a
        curve = [(propose_s + t_rej + h[0], j_rej + float(h[1].sum())) for h in h_a]
    else:
        curve = [(propose_s + t_rej, j_rej)]
    return v, curve


def run(n_train=20000, n_test=256, steps=6000, batch=64, iters=50, bands=None, seed=0, train_tag=101,
        test_tag=202, log=print):
    dev = torch.device('cuda', torch.cuda.current_device())
    sim = gpu.Sim(device=dev)
    eng = sim.engine
    w = engine.scaled_wavelet(gpu.RICKER, dev)
    res = {}
    t0 = time.perf_counter()
    train_models = synth.population(n_train, tag=train_tag)
    test_models = synth.population(n_test, tag=test_tag)
    stored = simulate_stored(eng, train_models, w)
    scale = float(stored.abs().max().item())
    targets = TI.targets(torch.tensor(train_models, device=dev)).contiguous()
    res['data_seconds'] = time.perf_counter() - t0
    net = ProposalNet(batch, device=dev, seed=seed)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    res['losses'] = train(net, stored, targets, scale, steps, seed=seed,
                          log=(lambda s, l: log(f'step {s}: L1 {l:.4f}')) if log else None)
    torch.cuda.synchronize(dev)
    res['train_seconds'] = time.perf_counter() - t1
    res['train_steps_per_s'] = steps / res['train_seconds']
    del stored
    # held-out models
    obs = eng.forward(torch.tensor(test_models, device=dev), w)
    trend = BG.depth_trend(train_models)
    fallback_vs = float(train_models[:, 0].mean())
    bg, vs, picked = medium_backgrounds(obs, trend, fallback_vs, dev)
    res['picker_refused'] = int((picked != 0).sum())
    fwi = BatchFWI(eng, w, obs)
    J_bg = fwi.misfit(bg.reshape(n_test, -1).contiguous(), torch.empty(n_test, dtype=torch.float64, device=dev)).cpu().numpy()
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    test_stored = TI.stored_gathers(obs)
    prop = predict(net, test_stored, scale)
    J_prop = fwi.misfit(prop.reshape(n_test, -1).contiguous(),
                        torch.empty(n_test, dtype=torch.float64, device=dev)).cpu().numpy()
    use = J_prop < J_bg
    start = torch.where(torch.tensor(use, device=dev)[:, None, None], prop, bg)
    torch.cuda.synchronize(dev)
    propose_s = time.perf_counter() - t2
    res.update(accepted=int(use.sum()), J_background=float(J_bg.sum()), J_proposal=float(J_prop.sum()),
               propose_seconds=propose_s,
               mae_background=norm_mae(bg.cpu().numpy(), test_models),
               mae_proposal=norm_mae(prop.cpu().numpy(), test_models))
    if isinstance(iters, int):             # one full band
        bands, iters = (None,), (iters,)
    if bands is None or len(bands) != len(iters):
        raise ValueError('give one iteration count per band')
    v_plain, h_plain = BatchFWI(eng, w, obs).run_bands(bg, gpu.RICKER, bands, iters)
    last = len(bands) - 1
    plain_total = [float(h[1].sum()) for h in h_plain if h[2] == last]
    target = plain_total[-1]
    t_plain = h_plain[-1][0]
    if len(bands) == 1:
        v_learn, h_learn = BatchFWI(eng, w, obs).run_bands(start, gpu.RICKER, bands, iters)
        curve = [(propose_s + h[0], float(h[1].sum())) for h in h_learn]
    else:
        v_learn, curve = learned_multiscale(eng, w, obs, prop, bg, use, bands, iters, propose_s)
    learn_total = [j for _, j in curve]
    reach = next((t for t, j in curve if j <= target), None)
    res.update(plain_final_misfit=target, learned_final_misfit=learn_total[-1], plain_seconds=t_plain,
               learned_seconds=curve[-1][0], learned_time_to_plain_misfit=reach,
               time_ratio=None if reach is None else reach / t_plain,
               time_ratio_inclusive=None if reach is None else
               (res['data_seconds'] + res['train_seconds'] + reach) / t_plain,
               plain_misfit_curve=plain_total, learned_misfit_curve=learn_total,
               mae_plain_fwi=norm_mae(v_plain.cpu().numpy(), test_models),
               mae_learned_fwi=norm_mae(v_learn.cpu().numpy(), test_models))
    return res
