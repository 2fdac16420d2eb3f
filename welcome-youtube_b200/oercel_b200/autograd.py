"""torch.autograd front end of the differentiated window.

The reference has no reverse mode: it fits nothing and runs replicas as
separate processes (cel/pc/sweep.py:146-166).  Here a window of Groot-Warren
steps (cel/engine/oercel.c:2303-2334) with the chemistry held fixed is a
differentiable function

    loss_r = WindowLoss(a, gamma, k_bond, x0, vh0, vt0)

of the repulsions a_ij, the friction gamma, the bond constant k_bond and,
optionally, the start state, for every replica r of an Engine.  Its value is
the smoothed pair-distribution loss of dpd_window_loss; its gradient is the
window adjoint (dpd_window_adjoint / dpd_window_adjoint_state: the pair noise
replayed from its key, checkpoints every `ckpt` steps, each segment recomputed
in reverse).  Because the adjoint needs the forward pass anyway, the forward
of this Function runs the adjoint at once when any input requires a gradient
and keeps the result for backward; with no gradient wanted it runs the plain
window.  Inputs:

  a       (k, k) repulsions shared by every replica, or (nrep, k, k) per
          replica; k = 4 (W, H, T, P) or 8 (every type).  Read as symmetric
          from the upper triangle (i <= j); the lower triangle is ignored and
          gets zero gradient.  None keeps the engine's repulsions.
  gamma, k_bond   scalars shared by every replica or (nrep,) tensors; None
          keeps the engine's values.
  x0, vh0, vt0    optional start state, (N_total, 2) in gid order packed by
          replica (replica r's gid g at row sum(n_beads[:r]) + g): positions,
          stored half-step velocities, predicted velocities.  Given, the
          engine is set to this state (types and links kept) at the step
          `cfg.step0` before the window, so the call is a pure function of its
          inputs.  None starts from the engine's current state.

The start forces are recomputed from the start state and the parameters of the
call, so loss and gradient belong to the same function.  After the call the
engine stands at the end of the window (a fit continues from there).
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from . import _capi
from .params import MAXT


class WindowConfig:
    """The non-differentiable part of a window: the engine, its length, the
    loss specification (Engine.rdf_spec), the target g(r) (nbin values, or
    nrep x nbin), the checkpoint interval and the start step (noise key of the
    start forces; None = the engine's step at the first call)."""

    def __init__(self, engine, nsteps, spec, target, ckpt=20, step0=None):
        self.engine = engine
        self.nsteps = int(nsteps)
        self.spec = spec
        self.target = np.asarray(target, np.float64)
        self.ckpt = int(ckpt)
        self.step0 = step0
        self._topology = None

    def topology(self):
        """per replica: types, prev and next in gid order (fixed inside windows)"""
        if self._topology is None:
            eng = self.engine
            topo = []
            for r in range(eng.nrep):
                s = eng.state(r)
                g = s["gid"].astype(np.int64)
                n = len(g)
                t = np.empty(n, np.uint8)
                t[g] = s["type"]
                pv = np.full(n, -1, np.int32)
                nx = np.full(n, -1, np.int32)
                pv[g] = np.where(s["prev"] >= 0, g[np.maximum(s["prev"], 0)], -1)
                nx[g] = np.where(s["next"] >= 0, g[np.maximum(s["next"], 0)], -1)
                topo.append((t, pv, nx))
            self._topology = topo
        return self._topology


def _per_replica(v, nrep, name):
    """a scalar or (nrep,) tensor as a list of nrep floats"""
    t = v.detach().to("cpu", torch.float64)
    if t.dim() == 0:
        return [float(t)] * nrep
    if t.shape != (nrep,):
        raise ValueError(f"{name} must be a scalar or have shape ({nrep},)")
    return [float(x) for x in t]


def _repulsions(a, nrep):
    """(k, k) or (nrep, k, k) -> per replica the k x k upper triangle as floats"""
    t = a.detach().to("cpu", torch.float64)
    if t.dim() == 2:
        t = t.expand(nrep, *t.shape)
    if t.dim() != 3 or t.shape[0] != nrep or t.shape[1] != t.shape[2] or t.shape[1] not in (4, 8):
        raise ValueError(f"a must be (k, k) or ({nrep}, k, k) with k = 4 or 8")
    return t.numpy()


def _apply_params(cfg, a, gamma, k_bond):
    eng = cfg.engine
    nrep = eng.nrep
    am = _repulsions(a, nrep) if a is not None else None
    gl = _per_replica(gamma, nrep, "gamma") if gamma is not None else None
    kl = _per_replica(k_bond, nrep, "k_bond") if k_bond is not None else None
    if am is None and gl is None and kl is None:
        return
    for r in range(nrep):
        p = copy.deepcopy(eng.params[r])
        if am is not None:
            k = am.shape[1]
            for i in range(k):
                for j in range(i, k):
                    p.a[i][j] = p.a[j][i] = float(am[r, i, j])
        if gl is not None:
            p.set("gamma", repr(gl[r]))
        if kl is not None:
            p.set("k_bond", repr(kl[r]))
        eng.set_params(r, p)


def _apply_state(cfg, x0, vh0, vt0):
    eng = cfg.engine
    if cfg.step0 is None:
        cfg.step0 = eng.step_no
    if x0 is None and vh0 is None and vt0 is None:
        return
    if x0 is None or vh0 is None or vt0 is None:
        raise ValueError("x0, vh0 and vt0 go together")
    topo = cfg.topology()
    X, VH, VT = (np.ascontiguousarray(v.detach().to("cpu", torch.float32).numpy()) for v in (x0, vh0, vt0))
    N = int(sum(eng.n_beads))
    for v in (X, VH, VT):
        if v.shape != (N, 2):
            raise ValueError(f"start state arrays must be ({N}, 2)")
    b0 = 0
    for r, n in enumerate(eng.n_beads):
        sl = slice(b0, b0 + n)
        t, pv, nx = topo[r]
        eng.set_state(r, X[sl, 0].copy(), X[sl, 1].copy(), VH[sl, 0].copy(), VH[sl, 1].copy(), t, None, pv, nx)
        eng.set_dynamics(r, vtx=VT[sl, 0].copy(), vty=VT[sl, 1].copy())
        b0 += n
    eng.build_cells()


class WindowLoss(torch.autograd.Function):
    """loss per replica of one differentiated window (see the module docstring)"""

    @staticmethod
    def forward(ctx, a, gamma, k_bond, x0, vh0, vt0, cfg):
        eng = cfg.engine
        _apply_params(cfg, a, gamma, k_bond)
        _apply_state(cfg, x0, vh0, vt0)
        if x0 is not None:
            eng.set_step(cfg.step0)
        eng.forces(eng.step_no)  # the start forces of this state and these parameters
        need = ctx.needs_input_grad if getattr(cfg, "grad_enabled", True) else (False,) * 7
        want_state = any(need[3:6])
        dev = next((v.device for v in (a, gamma, k_bond, x0) if isinstance(v, torch.Tensor)), torch.device("cpu"))
        if any(need[:6]):
            if want_state:
                loss, grad, _, xb, vhb, vtb = eng.window_adjoint_state(cfg.nsteps, cfg.ckpt, cfg.spec, cfg.target)
                ctx.state_grads = [torch.from_numpy(v.astype(np.float64)) for v in (xb, vhb, vtb)]
            else:
                loss, grad, _ = eng.window_adjoint(cfg.nsteps, cfg.ckpt, cfg.spec, cfg.target)
                ctx.state_grads = None
            ctx.grad = torch.from_numpy(grad)
        else:
            loss, _ = eng.window_loss(cfg.nsteps, cfg.spec, cfg.target)
        ctx.shapes = [None if v is None else (v.shape, v.dtype, v.device) for v in (a, gamma, k_bond)]
        ctx.n_beads = list(eng.n_beads)
        return torch.as_tensor(loss, dtype=torch.float64, device=dev)

    @staticmethod
    def backward(ctx, gl):
        gl = gl.detach().to("cpu", torch.float64)
        G = ctx.grad  # nrep x (64 + 2)
        nrep = G.shape[0]
        need = ctx.needs_input_grad
        out = [None] * 7
        sa, sg, sk = ctx.shapes
        if need[0]:
            A = G[:, : MAXT * MAXT].reshape(nrep, MAXT, MAXT) * gl[:, None, None]
            shape, dtype, device = sa
            k = shape[-1]
            A = A[:, :k, :k]
            out[0] = (A.sum(0) if len(shape) == 2 else A).to(dtype=dtype, device=device)
        for slot, idx, s in ((1, MAXT * MAXT, sg), (2, MAXT * MAXT + 1, sk)):
            if need[slot]:
                g = G[:, idx] * gl
                shape, dtype, device = s
                out[slot] = (g.sum() if len(shape) == 0 else g).reshape(shape).to(dtype=dtype, device=device)
        if getattr(ctx, "state_grads", None) is not None:
            rows = torch.repeat_interleave(gl, torch.tensor(ctx.n_beads))[:, None]
            for k in range(3):
                if need[3 + k]:
                    out[3 + k] = ctx.state_grads[k] * rows
        return tuple(out)


def window_loss(cfg: WindowConfig, a=None, gamma=None, k_bond=None, x0=None, vh0=None, vt0=None):
    """loss per replica (a float64 tensor of nrep values) of one differentiated
    window; see the module docstring for the arguments.  Under torch.no_grad
    the plain window runs (no adjoint)."""
    cfg.grad_enabled = torch.is_grad_enabled()
    return WindowLoss.apply(a, gamma, k_bond, x0, vh0, vt0, cfg)


def engine_values(engine, replica=0):
    """the engine's current (a (8, 8), gamma, k_bond) of one replica as float64 tensors"""
    p = engine.params[replica]
    return (torch.tensor(np.array(p.a, dtype=np.float64)), torch.tensor(float(p.gamma), dtype=torch.float64),
            torch.tensor(float(p.k_bond), dtype=torch.float64))


NGRAD = _capi.NGRAD
