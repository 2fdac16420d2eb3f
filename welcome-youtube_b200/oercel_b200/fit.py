"""Fitting interaction parameters to a structural target with the window adjoint.

One iteration: every replica runs a differentiated window (dpd_window_adjoint:
chemistry frozen, noise replayed, checkpoints every `ckpt` steps), the
per-replica gradients of the smoothed pair-distribution loss are summed into
one shared update (and over ranks with torch.distributed, one all-reduce of a
few dozen floats), and Adam moves the chosen parameters.  The replicas then
continue from the end of their window.
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


def set_value(p, key, v):
    if key in ("gamma", "k_bond"):
        p.set(key, repr(float(v)))
    else:
        p.set(key, repr(float(v)))


class Adam:
    def __init__(self, n, lr, b1=0.9, b2=0.999, eps=1e-12):
        self.m, self.v, self.t = np.zeros(n), np.zeros(n), 0
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps

    def step(self, g):
        self.t += 1
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        return -self.lr * mh / (np.sqrt(vh) + self.eps)


def fit(engine, keys, target, *, iters=20, window=200, ckpt=20, spec=None, lr=1.0, reduce=None, log=None):
    """Adam on `keys` (shared by every replica of the engine); returns the history"""
    spec = spec or engine.rdf_spec()
    opt = Adam(len(keys), lr)
    idx = [param_index(k) for k in keys]
    hist = []
    for it in range(iters):
        loss, grad, _ = engine.window_adjoint(window, ckpt, spec, target)
        g = grad[:, idx].sum(axis=0)
        tot = float(loss.sum())
        if reduce is not None:
            g, tot = reduce(g, tot)
        step = opt.step(g)
        vals = []
        for r, p in enumerate(engine.params):
            for k, d in zip(keys, step):
                set_value(p, k, get_value(p, k) + d)
            engine.set_params(r, p)
        vals = [get_value(engine.params[0], k) for k in keys]
        hist.append(dict(iter=it, loss=tot, grad=g.tolist(), values=vals))
        if log:
            log(hist[-1])
    return hist


def torch_reduce():
    """sum gradient and loss over ranks (NCCL or gloo): the one exchange of a batched fit"""
    import torch
    import torch.distributed as dist

    def red(g, loss):
        if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
            return g, loss
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor(np.append(g, loss), dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        out = t.cpu().numpy()
        return out[:-1], float(out[-1])

    return red


NGRAD = _capi.NGRAD
