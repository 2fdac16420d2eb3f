"""The torch.autograd front end of the differentiated window against torch
autograd of a naive all-pairs FP64 model unrolled through the same window.

The model restates one window on the host: Groot-Warren steps
(cel/engine/oercel.c:2303-2334) from a start state (x0, vh0, vt0), the start
forces F(x0, vt0), all-pairs DPD + bond forces (the O(N^2) pattern of
cel/engine/tests/forcetest.c:91-101) with the pair noise replayed from the
oracle's table at every step's key, and the smoothed T-T pair distribution
loss averaged over the window's last steps.  torch.autograd.grad of that loss
must equal the window adjoint's gradient to 1e-3 relative for the start
positions, both start velocities, every a_ij, gamma and k_bond."""
import numpy as np
import pytest

import oracle as O
import oercel_b200 as ob
from gpu_util import naive_chain_and_stir_forces, oracle_params, params

pytestmark = pytest.mark.gpu

MAXT = 8


def pair_forces_all(torch, x, v, asym, gamma, kb, types, theta, bi, bj, L, kT, dt, r0):
    n = x.shape[0]
    d = x[:, None, :] - x[None, :, :]
    d = d - L * torch.round(d / L)
    r2 = (d * d).sum(-1)
    eye = torch.eye(n, dtype=torch.bool)
    mask = (r2 < 1.0) & (r2 > 1e-24) & ~eye
    r = torch.sqrt(torch.where(mask, r2, torch.ones_like(r2)))
    w = 1.0 - r
    dv = v[:, None, :] - v[None, :, :]
    rv = (d * dv).sum(-1) / r
    s = torch.sqrt(2.0 * gamma * kT / dt)
    A = asym[types][:, types] - gamma * w * rv + s * theta
    fm = torch.where(mask, w * A / r, torch.zeros_like(r))
    F = (fm[..., None] * d).sum(1)
    db = x[bj] - x[bi]
    db = db - L * torch.round(db / L)
    rb = torch.sqrt((db * db).sum(-1))
    fb = kb * (1.0 - r0 / rb)[:, None] * db
    return F.index_add(0, bi, fb).index_add(0, bj, -fb)


def smoothed_pairs(torch, x, sel, L, nbin, rmax, sigma):
    """sum over unordered pairs of the selected beads of the Gaussian kernel on
    the bins within 4 sigma (the bins the device kernel visits)"""
    xs = x[sel]
    d = xs[:, None, :] - xs[None, :, :]
    d = d - L * torch.round(d / L)
    iu = torch.triu_indices(len(sel), len(sel), 1)
    dd = d[iu[0], iu[1]]
    r = torch.sqrt((dd * dd).sum(-1))
    dr = rmax / nbin
    rc = rmax + 4.0 * sigma
    keep = (r < rc) & (r > 0)
    r = r[keep]
    b = torch.arange(nbin, dtype=x.dtype)
    rb = (b + 0.5) * dr
    rd = r.detach()
    lo = torch.floor((rd - 4.0 * sigma) / dr).clamp(min=0)
    hi = torch.floor((rd + 4.0 * sigma) / dr).clamp(max=nbin - 1)
    inside = (b[None, :] >= lo[:, None]) & (b[None, :] <= hi[:, None])
    kn = dr / (sigma * np.sqrt(2.0 * np.pi))
    k = kn * torch.exp(-((r[:, None] - rb[None, :]) ** 2) / (2.0 * sigma * sigma))
    return torch.where(inside, k, torch.zeros_like(k)).sum(0)


def unrolled_window_loss(torch, p, step0, nsteps, x0, vh0, vt0, P, gamma, kb, types, bi, bj, spec, target,
                         prv=None, nxt=None):
    """prv, nxt (gid order): the chains, for the angle terms and stirring when p has them"""
    op = oracle_params(p)
    L = float(np.float32(p.L))
    dt = float(np.float32(p.dt))
    lam = float(p["lambda"])
    cvt, dt2 = (0.5 + lam) * dt, dt * dt
    asym = torch.triu(P) + torch.triu(P, 1).T
    gid = np.arange(x0.shape[0], dtype=np.uint32)
    sel = torch.as_tensor(np.nonzero(types.numpy() == spec.ta)[0])
    npairs = len(sel) * (len(sel) - 1) / 2

    def forces(x, v, step):
        th = torch.as_tensor(O.theta_matrix(op, step, gid))
        kT = p.kT
        if p.kT_amp != 0:  # the temperature cycle of the noise, t = step dt
            kT = p.kT + p.kT_amp * np.sin(2.0 * np.pi * step * p.dt / p.kT_period)
        F = pair_forces_all(torch, x, v, asym, gamma, kb, types, th, bi, bj, L, kT, dt, p.r0)
        if p.k_angle != 0 or p.stir_A != 0:
            F = F + naive_chain_and_stir_forces(torch, x, prv, nxt, p.k_angle, L, p.stir_A, p.stir_n)
        return F

    x, vh, vt = x0, vh0, vt0
    f = forces(x, vt, step0)
    hist = torch.zeros(spec.nbin, dtype=torch.float64)
    first = nsteps - spec.last_steps + 1
    for k in range(1, nsteps + 1):
        xn = x + dt * vh + dt2 * f
        xn = xn - L * torch.floor(xn.detach() / L)
        vt = vh + cvt * f
        vh = vh + dt * f
        x = xn
        f = forces(x, vt, step0 + k)
        if k >= first:
            hist = hist + smoothed_pairs(torch, x, sel, L, spec.nbin, spec.rmax, spec.sigma)
    dr = spec.rmax / spec.nbin
    rb = (torch.arange(spec.nbin, dtype=torch.float64) + 0.5) * dr
    g = hist / spec.last_steps * (L * L) / (npairs * 2.0 * np.pi * rb * dr)
    return ((g - torch.as_tensor(target)) ** 2).sum() / spec.nbin


def by_gid(s):
    g = s["gid"].astype(np.int64)
    n = len(g)
    out = {}
    for k in ("x", "y", "vhx", "vhy", "vtx", "vty"):
        v = np.empty(n, np.float32)
        v[g] = s[k]
        out[k] = v
    t = np.empty(n, np.uint8)
    t[g] = s["type"]
    nx = np.full(n, -1, np.int64)
    nx[g] = np.where(s["next"] >= 0, g[np.maximum(s["next"], 0)], -1)
    out["type"], out["next"] = t, nx
    return out


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


EXTRA = dict(k_angle=10.0, stir_A=0.5, stir_n=2, kT_amp=0.3, kT_period=2.0)


@pytest.mark.parametrize("nsteps,seed,extra", [(12, 31, {}), (20, 32, {}), (12, 34, EXTRA)])
def test_window_gradient_matches_unrolled_torch_autograd(cuda_ok, nsteps, seed, extra):
    """extra: the angle terms of the chains, stirring and the temperature cycle as well"""
    import torch
    from oercel_b200 import autograd as AG
    p = params(L=8.0, seed=seed, noise="philox", f_lip=0.3, c_N=0.1, **extra)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(30)
    step0 = e.step_no
    s = by_gid(e.state())
    spec = ob.Engine.rdf_spec(ta=2, tb=2, nbin=32, rmax=2.0, sigma=0.1, last_steps=5)
    target = np.linspace(0.5, 1.5, 32)
    dt = torch.float64
    x0 = torch.tensor(np.c_[s["x"], s["y"]], dtype=dt, requires_grad=True)
    vh0 = torch.tensor(np.c_[s["vhx"], s["vhy"]], dtype=dt, requires_grad=True)
    vt0 = torch.tensor(np.c_[s["vtx"], s["vty"]], dtype=dt, requires_grad=True)
    P = torch.tensor(np.array(p.a, dtype=np.float64), dtype=dt, requires_grad=True)
    gam = torch.tensor(p.gamma, dtype=dt, requires_grad=True)
    kb = torch.tensor(p.k_bond, dtype=dt, requires_grad=True)
    # the device window through the autograd Function
    cfg = AG.WindowConfig(e, nsteps, spec, target, ckpt=5, step0=step0)
    loss = AG.window_loss(cfg, P, gam, kb, x0, vh0, vt0)
    got = torch.autograd.grad(loss.sum(), [x0, vh0, vt0, P, gam, kb])
    # the host model
    types = torch.as_tensor(s["type"].astype(np.int64))
    bi = torch.as_tensor(np.nonzero(s["next"] >= 0)[0])
    bj = torch.as_tensor(s["next"][s["next"] >= 0])
    nxt = s["next"]
    prv = np.full(len(nxt), -1, np.int64)
    prv[nxt[nxt >= 0]] = np.nonzero(nxt >= 0)[0]
    lm = unrolled_window_loss(torch, p, step0, nsteps, x0, vh0, vt0, P, gam, kb, types, bi, bj, spec, target, prv,
                              nxt)
    want = torch.autograd.grad(lm, [x0, vh0, vt0, P, gam, kb])
    assert float(loss.detach()[0]) == pytest.approx(float(lm.detach()), rel=1e-4)
    names = ["x0", "vh0", "vt0"]
    for k in range(3):
        assert rel(got[k].numpy(), want[k].numpy()) < 1e-3, names[k]
    gP, wP = got[3].numpy(), want[3].numpy()
    assert np.all(np.tril(gP, -1) == 0.0)
    for i in range(4):
        for j in range(i, 4):
            if abs(wP[i, j]) > 1e-3 * np.abs(wP).max():
                assert gP[i, j] == pytest.approx(wP[i, j], rel=1e-3), (i, j)
            else:
                assert abs(gP[i, j] - wP[i, j]) < 1e-6 * np.abs(wP).max(), (i, j)
    assert float(got[4]) == pytest.approx(float(want[4]), rel=1e-3)
    assert float(got[5]) == pytest.approx(float(want[5]), rel=1e-3)


def test_window_loss_is_a_pure_function_of_its_inputs(cuda_ok):
    """Given the start state, two calls give the same loss and gradient, and the
    4 x 4 form of a gives the top-left block of the 8 x 8 gradient; under
    no_grad the plain window runs and gives the same loss."""
    import torch
    from oercel_b200 import autograd as AG
    p = params(L=10.0, seed=33, noise="philox", f_lip=0.3, c_N=0.1)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(20)
    step0 = e.step_no
    s = by_gid(e.state())
    spec = ob.Engine.rdf_spec(nbin=32, rmax=2.0, sigma=0.1, last_steps=4)
    target = np.linspace(0.5, 1.5, 32)
    cfg = AG.WindowConfig(e, 10, spec, target, ckpt=5, step0=step0)
    st = [torch.tensor(np.c_[s[a], s[b]], dtype=torch.float64) for a, b in (("x", "y"), ("vhx", "vhy"),
                                                                            ("vtx", "vty"))]
    a8 = torch.tensor(np.array(p.a, dtype=np.float64), requires_grad=True)
    l1 = AG.window_loss(cfg, a8, None, None, *st)
    g1, = torch.autograd.grad(l1.sum(), [a8])
    a4 = torch.tensor(np.array(p.a, dtype=np.float64)[:4, :4], requires_grad=True)
    l2 = AG.window_loss(cfg, a4, None, None, *st)
    g2, = torch.autograd.grad(l2.sum(), [a4])
    assert float(l1) == float(l2)
    assert np.array_equal(g1.numpy()[:4, :4], g2.numpy())
    with torch.no_grad():
        l3 = AG.window_loss(cfg, a8, None, None, *st)
    assert float(l3) == float(l1)


def test_torch_adam_fits_through_the_window(cuda_ok):
    """a torch.optim.Adam on a_W_T through the Function, on the pattern of the
    differentiated fit (target g_TT made at a_W_T = 75, start at 60)"""
    import torch
    from oercel_b200 import autograd as AG
    truth = params(L=20.0, seed=8, noise="philox", f_lip=0.3, c_N=0.05)
    e = ob.Engine(truth)
    e.load_soup(0)
    e.prime()
    e.step(200)
    spec = ob.Engine.rdf_spec(nbin=32, rmax=2.0, sigma=0.1, last_steps=20, horizon=10)
    _, target = e.window_loss(60, spec, np.zeros(32))
    a = torch.tensor(np.array(truth.a, dtype=np.float64))
    a[0, 2] = 60.0
    awt = torch.tensor(60.0, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([awt], lr=2.0)
    cfg = AG.WindowConfig(e, 60, spec, target[0], ckpt=20)
    mask = torch.zeros(8, 8, dtype=torch.float64)
    mask[0, 2] = 1.0
    hist = []
    for _ in range(6):
        used = float(awt)
        opt.zero_grad()
        loss = AG.window_loss(cfg, a * (1 - mask) + awt * mask).sum()
        loss.backward()
        opt.step()
        hist.append((float(loss), float(awt)))
        assert e.params[0].a[0][2] == used and e.params[0].a[2][0] == used  # the engine ran the value of the call
    assert hist[-1][1] > 60.0
    assert all(np.isfinite(h[0]) for h in hist)
