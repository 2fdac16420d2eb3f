"""Fitting interaction parameters to a structural target with the window adjoint.

One iteration: every replica runs a differentiated window through the
torch.autograd Function of oercel_b200.autograd (dpd_window_adjoint: chemistry
frozen, noise replayed, checkpoints every `ckpt` steps), the per-replica losses
are summed, backward gives the gradient of the shared parameters (summed over
ranks with torch.distributed when `distributed`: one all-reduce of a few
floats, shard.reduce_gradients), and torch.optim.Adam moves them.  The
replicas then continue from the end of their window.  The reference fits
nothing (it has no reverse mode); its closest analogue is a sweep of
independent runs (cel/pc/sweep.py:146-166).
"""
from __future__ import annotations

import numpy as np

from . import _capi
from .params import TYPE_ALIASES, TYPE_NAMES

MAXT = 8


def param_index(key):
    """gradient slot of a parameter key: a_X_Y, gamma or k_bond"""
    if key == "gamma":
        return MAXT * MAXT
    if key == "k_bond":
        return MAXT * MAXT + 1
    if key.startswith("a_"):
        x, y = key[2:].split("_")
        t = [TYPE_NAMES.index(v) if v in TYPE_NAMES else TYPE_ALIASES[v] for v in (x, y)]
        i, j = min(t), max(t)
        return i * MAXT + j
    raise KeyError(key)


def get_value(p, key):
    if key in ("gamma", "k_bond"):
        return float(p[key])
    i = param_index(key)
    return float(p.a[i // MAXT][i % MAXT])


def shared_inputs(engine, keys, values):
    """the window's inputs with `keys` set to `values` (a float64 tensor) in
    every replica: per-replica repulsions (nrep, 8, 8) (the other entries kept
    from each replica's own parameters), gamma and k_bond, or None where no
    key touches them"""
    import torch
    nrep = engine.nrep
    base = torch.tensor(np.array([np.array(p.a, dtype=np.float64) for p in engine.params]))
    a = None
    gamma = k_bond = None
    for k, key in enumerate(keys):
        if key == "gamma":
            gamma = values[k]
        elif key == "k_bond":
            k_bond = values[k]
        else:
            idx = param_index(key)
            m = torch.zeros(nrep, MAXT, MAXT, dtype=torch.float64)
            m[:, idx // MAXT, idx % MAXT] = 1.0
            a = (base if a is None else a) * (1.0 - m) + values[k] * m
    return a, gamma, k_bond


def fit(engine, keys, target, *, iters=20, window=200, ckpt=20, spec=None, lr=1.0, distributed=False, log=None):
    """torch.optim.Adam on `keys` (a_X_Y, gamma, k_bond; shared by every replica
    of the engine) through the autograd Function; returns the history: per
    iteration the summed loss (over replicas and ranks), the gradient and the
    values the window ran with"""
    import torch

    from . import autograd as AG
    from .shard import reduce_gradients
    spec = spec or engine.rdf_spec()
    values = torch.tensor([get_value(engine.params[0], k) for k in keys], dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([values], lr=lr)
    cfg = AG.WindowConfig(engine, window, spec, target, ckpt=ckpt)
    hist = []
    for it in range(iters):
        used = values.detach().tolist()
        opt.zero_grad()
        loss = AG.window_loss(cfg, *shared_inputs(engine, keys, values)).sum()
        loss.backward()
        tot = float(loss.detach())
        if distributed:
            buf = torch.cat([values.grad, torch.tensor([tot], dtype=torch.float64)])
            reduce_gradients(buf)
            values.grad.copy_(buf[:-1])
            tot = float(buf[-1])
        g = values.grad.tolist()
        opt.step()
        hist.append(dict(iter=it, loss=tot, grad=g, values=used))
        if log:
            log(hist[-1])
    return hist


NGRAD = _capi.NGRAD
