"""Reverse mode: the force VJP against torch autograd of a naive all-pairs model,
and the window adjoint (checkpoints + recomputation, replayed noise) against
central finite differences of the same window."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import oercel_b200 as ob
from gpu_util import engine_with, naive_chain_and_stir_forces, oracle_params, params

pytestmark = pytest.mark.gpu

MAXT = 8


def naive_forces(torch, x, v, P, gamma, kb, types, theta, nxt, L, kT, dt, r0):
    """all-pairs DPD + bond forces in float64 (the template of cel/engine/tests/forcetest.c:91-101)"""
    n = x.shape[0]
    a = torch.triu(P) + torch.triu(P, 1).T
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
    A = a[types][:, types] - gamma * w * rv + s * theta
    fm = torch.where(mask, w * A / r, torch.zeros_like(r))
    F = (fm[..., None] * d).sum(1)
    i = np.nonzero(nxt >= 0)[0]
    j = nxt[i]
    db = x[j] - x[i]
    db = db - L * torch.round(db / L)
    rb = torch.sqrt((db * db).sum(-1))
    fb = kb * (1.0 - r0 / rb)[:, None] * db
    F = F.index_add(0, torch.as_tensor(i), fb)
    F = F.index_add(0, torch.as_tensor(j), -fb)
    return F


def _theta_table(p, s, step):
    """the pair noise theta of every pair of the state at `step`, from the oracle"""
    op = oracle_params(p)
    n = len(s["x"])
    th = np.zeros((n, n))
    for a_ in range(n):
        for b_ in range(a_ + 1, n):
            th[a_, b_] = th[b_, a_] = O.lib().ora_theta(C.byref(op), step, int(s["gid"][a_]), int(s["gid"][b_]))
    return th


def test_force_vjp_with_angles_stirring_and_temperature_cycle(cuda_ok):
    """every term together: pairs with the noise at kT(t), bonds, angle terms and
    stirring, against torch autograd of the all-pairs model"""
    import torch
    p = params(L=8.0, seed=23, noise="philox", f_lip=0.3, c_N=0.1, k_angle=10.0, stir_A=0.5, stir_n=2, kT_amp=0.3,
               kT_period=0.5)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(5)
    step = e.step_no
    s = e.state()
    n = len(s["x"])
    rng = np.random.default_rng(0)
    gx, gy = rng.normal(size=(2, n)).astype(np.float32)
    xbx, xby, vbx, vby, grad = e.force_vjp(0, step, gx, gy)
    th = _theta_table(p, s, step)
    dt = torch.float64
    x = torch.tensor(np.c_[s["x"], s["y"]], dtype=dt, requires_grad=True)
    v = torch.tensor(np.c_[s["vtx"], s["vty"]], dtype=dt, requires_grad=True)
    P = torch.tensor(np.array(p.a, dtype=np.float64), dtype=dt, requires_grad=True)
    gam = torch.tensor(p.gamma, dtype=dt, requires_grad=True)
    kb = torch.tensor(p.k_bond, dtype=dt, requires_grad=True)
    L = float(np.float32(p.L))
    kT = p.kT + p.kT_amp * np.sin(2.0 * np.pi * step * p.dt / p.kT_period)  # t = step dt
    F = naive_forces(torch, x, v, P, gam, kb, torch.as_tensor(s["type"].astype(np.int64)), torch.tensor(th), s["next"],
                     L, kT, p.dt, p.r0)
    F = F + naive_chain_and_stir_forces(torch, x, s["prev"], s["next"], p.k_angle, L, p.stir_A, p.stir_n)
    assert np.abs(F.detach().numpy() - np.c_[s["fx"], s["fy"]]).max() < 1e-5 * np.abs(F.detach().numpy()).max()
    lam = (F * torch.tensor(np.c_[gx, gy], dtype=dt)).sum()
    gxv, gvv, gP, gg, gk = torch.autograd.grad(lam, [x, v, P, gam, kb])

    def rel(a, b):
        return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-30)

    assert rel(np.c_[xbx, xby], gxv.numpy()) < 1e-3
    assert rel(np.c_[vbx, vby], gvv.numpy()) < 1e-3
    gP = gP.numpy()
    up = np.array([[gP[i, j] if i <= j else 0.0 for j in range(MAXT)] for i in range(MAXT)])
    assert rel(grad[:64].reshape(MAXT, MAXT), up) < 1e-3
    assert grad[64] == pytest.approx(gg.item(), rel=1e-3)
    assert grad[65] == pytest.approx(gk.item(), rel=1e-3)


def test_force_vjp_terms_one_at_a_time(cuda_ok):
    """each term's own share of the VJP, the VJP with the term on less the VJP
    with it off on the same configuration, against torch autograd of that term
    alone: the angle terms, stirring, and the temperature cycle's noise"""
    import torch
    kv = dict(L=8.0, seed=25, noise="philox", f_lip=0.4, c_N=0.1)
    on = dict(k_angle=30.0, stir_A=2.0, stir_n=2, kT_amp=0.5, kT_period=0.5)
    full = params(**kv, **on)
    e = ob.Engine(full)
    e.load_soup(0)
    e.prime()
    e.step(5)
    step = e.step_no
    s = e.state()
    n = len(s["x"])
    rng = np.random.default_rng(4)
    gx, gy = rng.normal(size=(2, n)).astype(np.float32)

    def vjp(**off):
        e.set_params(0, params(**kv, **{**on, **off}))
        xbx, xby, vbx, vby, grad = e.force_vjp(0, step, gx, gy)
        return np.c_[xbx, xby].astype(np.float64), np.c_[vbx, vby].astype(np.float64), grad

    x_all, v_all, g_all = vjp()
    dt = torch.float64
    L = float(np.float32(full.L))
    g = torch.tensor(np.c_[gx, gy], dtype=dt)

    def share(F, x):
        return torch.autograd.grad((F * g).sum(), x)[0].numpy()

    def rel(a, b):
        return np.abs(a - b).max() / np.abs(b).max()

    x = torch.tensor(np.c_[s["x"], s["y"]], dtype=dt, requires_grad=True)
    want = share(naive_chain_and_stir_forces(torch, x, s["prev"], s["next"], on["k_angle"], L, 0.0, 1), x)
    assert np.abs(want).max() > 0
    assert rel(x_all - vjp(k_angle=0.0)[0], want) < 1e-4
    x = torch.tensor(np.c_[s["x"], s["y"]], dtype=dt, requires_grad=True)
    want = share(naive_chain_and_stir_forces(torch, x, s["prev"], s["next"], 0.0, L, on["stir_A"], on["stir_n"]), x)
    assert rel(x_all - vjp(stir_A=0.0)[0], want) < 1e-4
    # the noise at kT(t) less the noise at kT: through the positions and gamma
    th = _theta_table(full, s, step)
    x = torch.tensor(np.c_[s["x"], s["y"]], dtype=dt, requires_grad=True)
    v = torch.tensor(np.c_[s["vtx"], s["vty"]], dtype=dt, requires_grad=True)
    gam = torch.tensor(full.gamma, dtype=dt, requires_grad=True)
    P = torch.tensor(np.array(full.a, dtype=np.float64), dtype=dt)
    kb = torch.tensor(full.k_bond, dtype=dt)
    kTt = full.kT + on["kT_amp"] * np.sin(2.0 * np.pi * step * full.dt / on["kT_period"])
    args = (torch.as_tensor(s["type"].astype(np.int64)), torch.tensor(th), s["next"], L)
    F = naive_forces(torch, x, v, P, gam, kb, *args, kTt, full.dt, full.r0) - \
        naive_forces(torch, x, v, P, gam, kb, *args, full.kT, full.dt, full.r0)
    wx, wv, wg = torch.autograd.grad((F * g).sum(), [x, v, gam], allow_unused=True)
    x_off, v_off, g_off = vjp(kT_amp=0.0)
    assert rel(x_all - x_off, wx.numpy()) < 1e-3
    # the noise term does not depend on the velocities: their share is zero (torch's to rounding)
    assert wv is None or np.abs(wv.numpy()).max() <= 1e-12 * np.abs(wx.numpy()).max()
    assert np.abs(v_all - v_off).max() <= 1e-6 * np.abs(v_all).max()
    assert g_all[64] - g_off[64] == pytest.approx(wg.item(), rel=1e-3)


def naive_template_forces(torch, x, prv, nxt, tmpl, kb, L):
    """bonded forces of branched lipids from their template (mol_forces,
    oercel.c:1221-1257): each molecule is the chain of next links from a bead
    without prev; bonds kb (r - r0) toward each other, angles K (1 - cos) or
    K (cos - c0)^2 of (x_j - x_i, x_k - x_j); float64"""
    starts = np.nonzero((prv < 0) & (nxt >= 0))[0]
    mols = []
    for s0 in starts:
        m = [s0]
        while nxt[m[-1]] >= 0 and len(m) < tmpl.mlen:
            m.append(nxt[m[-1]])
        assert len(m) == tmpl.mlen
        mols.append(m)
    M = torch.as_tensor(np.array(mols))
    U = x.new_zeros(())

    def vec(i, j):
        d = x[M[:, j]] - x[M[:, i]]
        return d - L * torch.round(d / L)
    for q in range(tmpl.nb):
        r = vec(tmpl.bi[q], tmpl.bj[q]).norm(dim=-1)
        U = U + 0.5 * kb * ((r - tmpl.br0[q]) ** 2).sum()
    for q in range(tmpl.na):
        a, c = vec(tmpl.ai[q], tmpl.aj[q]), vec(tmpl.aj[q], tmpl.ak[q])
        cos = (a * c).sum(-1) / (a.norm(dim=-1) * c.norm(dim=-1))
        K, c0 = float(tmpl.aK[q]), float(tmpl.ac0[q])
        U = U + (K * (1.0 - cos) if tmpl.akind[q] == 0 else K * (cos - c0) ** 2).sum()
    return -torch.autograd.grad(U, x, create_graph=True)[0]


def test_force_vjp_of_branched_lipids(cuda_ok):
    """the template bonds and both kinds of angle term of pi lipids, against torch autograd"""
    import torch
    p = params(L=8.0, seed=24, noise="philox", f_lip=0.4, c_N=0.05, lip_arch="pi", lip_nT=2, lip_tie=1, r0_head=0.7,
               k_bond=300, k_angle=15, k_head=20, cos_head=-0.2)
    tmpl = p.template()
    assert any(tmpl.akind[q] == 1 for q in range(tmpl.na))
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(5)
    step = e.step_no
    s = e.state()
    n = len(s["x"])
    rng = np.random.default_rng(3)
    gx, gy = rng.normal(size=(2, n)).astype(np.float32)
    xbx, xby, vbx, vby, grad = e.force_vjp(0, step, gx, gy)
    th = _theta_table(p, s, step)
    dt = torch.float64
    x = torch.tensor(np.c_[s["x"], s["y"]], dtype=dt, requires_grad=True)
    v = torch.tensor(np.c_[s["vtx"], s["vty"]], dtype=dt, requires_grad=True)
    P = torch.tensor(np.array(p.a, dtype=np.float64), dtype=dt, requires_grad=True)
    gam = torch.tensor(p.gamma, dtype=dt, requires_grad=True)
    kb = torch.tensor(p.k_bond, dtype=dt, requires_grad=True)
    L = float(np.float32(p.L))
    none = -np.ones(n, dtype=np.int64)  # no linear bonds: the template's terms instead
    F = naive_forces(torch, x, v, P, gam, kb, torch.as_tensor(s["type"].astype(np.int64)), torch.tensor(th), none, L,
                     p.kT, p.dt, p.r0)
    F = F + naive_template_forces(torch, x, s["prev"], s["next"], tmpl, kb, L)
    assert np.abs(F.detach().numpy() - np.c_[s["fx"], s["fy"]]).max() < 1e-5 * np.abs(F.detach().numpy()).max()
    lam = (F * torch.tensor(np.c_[gx, gy], dtype=dt)).sum()
    gxv, gvv, gP, gg, gk = torch.autograd.grad(lam, [x, v, P, gam, kb])

    def rel(a, b):
        return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-30)

    assert rel(np.c_[xbx, xby], gxv.numpy()) < 1e-3
    assert rel(np.c_[vbx, vby], gvv.numpy()) < 1e-3
    assert grad[64] == pytest.approx(gg.item(), rel=1e-3)
    assert grad[65] == pytest.approx(gk.item(), rel=1e-3)


def test_force_vjp_matches_torch_autograd(cuda_ok):
    import torch
    p = params(L=8.0, seed=21, noise="philox", f_lip=0.3, c_N=0.1)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(5)
    step = e.step_no
    s = e.state()
    n = len(s["x"])
    rng = np.random.default_rng(0)
    gx, gy = rng.normal(size=(2, n)).astype(np.float32)
    xbx, xby, vbx, vby, grad = e.force_vjp(0, step, gx, gy)
    op = oracle_params(p)
    th = np.zeros((n, n))
    for a_ in range(n):
        for b_ in range(a_ + 1, n):
            th[a_, b_] = th[b_, a_] = O.lib().ora_theta(C.byref(op), step, int(s["gid"][a_]), int(s["gid"][b_]))
    dt = torch.float64
    x = torch.tensor(np.c_[s["x"], s["y"]], dtype=dt, requires_grad=True)
    v = torch.tensor(np.c_[s["vtx"], s["vty"]], dtype=dt, requires_grad=True)
    P = torch.tensor(np.array(p.a, dtype=np.float64), dtype=dt, requires_grad=True)
    gam = torch.tensor(p.gamma, dtype=dt, requires_grad=True)
    kb = torch.tensor(p.k_bond, dtype=dt, requires_grad=True)
    F = naive_forces(torch, x, v, P, gam, kb, torch.as_tensor(s["type"].astype(np.int64)), torch.tensor(th), s["next"],
                     float(np.float32(p.L)), p.kT, p.dt, p.r0)
    # the GPU forces themselves agree with the model
    assert np.abs(F.detach().numpy() - np.c_[s["fx"], s["fy"]]).max() < 1e-5 * np.abs(F.detach().numpy()).max()
    lam = (F * torch.tensor(np.c_[gx, gy], dtype=dt)).sum()
    gxv, gvv, gP, gg, gk = torch.autograd.grad(lam, [x, v, P, gam, kb])

    def rel(a, b):
        return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-30)

    assert rel(np.c_[xbx, xby], gxv.numpy()) < 1e-3
    assert rel(np.c_[vbx, vby], gvv.numpy()) < 1e-3
    gP = gP.numpy()
    up = np.array([[gP[i, j] if i <= j else 0.0 for j in range(MAXT)] for i in range(MAXT)])
    assert rel(grad[:64].reshape(MAXT, MAXT), up) < 1e-3
    assert grad[64] == pytest.approx(gg.item(), rel=1e-3)
    assert grad[65] == pytest.approx(gk.item(), rel=1e-3)


def _window_engine(p, s0, step0):
    e = engine_with(p, s0["x"], s0["y"], s0["vhx"], s0["vhy"], s0["type"], s0["prev"], s0["next"], gid=s0["gid"])
    e.build_cells()
    e.forces(step0)
    return e


def test_window_adjoint_matches_finite_differences(cuda_ok):
    base = params(L=12.0, seed=5, noise="philox", f_lip=0.3, c_N=0.1)
    e = ob.Engine(base)
    e.load_soup(0)
    e.prime()
    e.step(40)
    s0, step0 = e.state(), e.step_no
    spec = ob.Engine.rdf_spec(ta=2, tb=2, nbin=32, rmax=2.0, sigma=0.1, last_steps=5)
    target = np.linspace(0.5, 1.5, 32)
    # 6 steps (a checkpoint at 5): over longer windows of this dense box the FP32
    # trajectories of nearby parameter values part enough that central
    # differences scatter by about 3e-3 across step sizes (12 steps), which
    # would hide a 1e-3 error of the adjoint; at 6 steps they agree to 1e-4
    nsteps, ckpt = 6, 5
    e = _window_engine(base, s0, step0)
    loss, grad, rdf = e.window_adjoint(nsteps, ckpt, spec, target)
    assert loss[0] > 0 and np.all(np.isfinite(grad))
    # the adjoint run leaves the engine at the end of the window, like the plain window
    e2 = _window_engine(base, s0, step0)
    loss2, rdf2 = e2.window_loss(nsteps, spec, target)
    assert loss2[0] == loss[0] and np.array_equal(rdf, rdf2)
    assert np.array_equal(e.state()["x"], e2.state()["x"])

    def loss_at(**kv):
        pp = params(L=12.0, seed=5, noise="philox", f_lip=0.3, c_N=0.1, **kv)
        return _window_engine(pp, s0, step0).window_loss(nsteps, spec, target)[0][0]

    # central differences with steps of 4 % of each value: the loss is smooth on
    # that scale, and the step keeps the FP32 rounding of the two runs small
    # against their difference
    checks = [("a_W_T", 75.0, 0 * 8 + 2), ("a_H_T", 50.0, 1 * 8 + 2), ("gamma", 4.5, 64), ("k_bond", 100.0, 65)]
    for key, val, idx in checks:
        h = 0.04 * val
        fd = (loss_at(**{key: val + h}) - loss_at(**{key: val - h})) / (2 * h)
        assert grad[0][idx] == pytest.approx(fd, rel=1e-3, abs=1e-5 * np.abs(grad[0]).max()), key


def test_window_adjoint_with_angles_stirring_and_temperature_cycle(cuda_ok):
    """the window adjoint through the angle, stirring and kT(t) terms against
    central differences.  These terms bend the loss more over the 4 % steps of
    the test above, so the differences are Richardson-extrapolated from steps of
    2 % and 1 %: (4 D(h/2) - D(h)) / 3.  gamma is left to the exact check against
    the unrolled torch model (test_gpu_autograd.py): it scales the noise
    amplitude too, and its differences scatter by a few 1e-3 on this box."""
    kv = dict(L=12.0, seed=7, noise="philox", f_lip=0.3, c_N=0.1, k_angle=10.0, stir_A=0.5, stir_n=2, kT_amp=0.3,
              kT_period=2.0)
    base = params(**kv)
    e = ob.Engine(base)
    e.load_soup(0)
    e.prime()
    e.step(40)
    s0, step0 = e.state(), e.step_no
    spec = ob.Engine.rdf_spec(ta=2, tb=2, nbin=32, rmax=2.0, sigma=0.1, last_steps=5)
    target = np.linspace(0.5, 1.5, 32)
    nsteps, ckpt = 6, 5
    loss, grad, rdf = _window_engine(base, s0, step0).window_adjoint(nsteps, ckpt, spec, target)
    assert loss[0] > 0 and np.all(np.isfinite(grad))

    def loss_at(**over):
        return _window_engine(params(**{**kv, **over}), s0, step0).window_loss(nsteps, spec, target)[0][0]

    def d(key, val, h):
        return (loss_at(**{key: val + h}) - loss_at(**{key: val - h})) / (2 * h)

    for key, val, idx in [("a_W_T", 75.0, 2), ("a_H_T", 50.0, 10), ("k_bond", 100.0, 65)]:
        h = 0.02 * val
        fd = (4.0 * d(key, val, h / 2) - d(key, val, h)) / 3.0
        assert grad[0][idx] == pytest.approx(fd, rel=1e-3, abs=1e-5 * np.abs(grad[0]).max()), key


def test_horizon_truncates_the_reverse_pass(cuda_ok):
    base = params(L=12.0, seed=6, noise="philox", f_lip=0.3, c_N=0.1)
    e = ob.Engine(base)
    e.load_soup(0)
    e.prime()
    e.step(30)
    s0, step0 = e.state(), e.step_no
    target = np.linspace(0.5, 1.5, 32)
    full = _window_engine(base, s0, step0).window_adjoint(
        16, 4, ob.Engine.rdf_spec(nbin=32, rmax=2.0, sigma=0.1, last_steps=4), target)
    longh = _window_engine(base, s0, step0).window_adjoint(
        16, 4, ob.Engine.rdf_spec(nbin=32, rmax=2.0, sigma=0.1, last_steps=4, horizon=100), target)
    short = _window_engine(base, s0, step0).window_adjoint(
        16, 4, ob.Engine.rdf_spec(nbin=32, rmax=2.0, sigma=0.1, last_steps=4, horizon=3), target)
    assert np.array_equal(full[1], longh[1])  # a horizon past the window start changes nothing
    assert full[0][0] == short[0][0] and np.all(np.isfinite(short[1]))
    assert not np.array_equal(full[1], short[1])


def test_fit_moves_repulsion_toward_target(cuda_ok):
    """configuration-4 pattern on a small box: target g_TT(r) made at a_W_T = 75, fit from 60"""
    from oercel_b200 import fit
    truth = params(L=20.0, seed=8, noise="philox", f_lip=0.3, c_N=0.05)
    e = ob.Engine(truth)
    e.load_soup(0)
    e.prime()
    e.step(200)
    spec = ob.Engine.rdf_spec(nbin=32, rmax=2.0, sigma=0.1, last_steps=20, horizon=10)
    _, target = e.window_loss(60, spec, np.zeros(32))
    start = params(L=20.0, seed=8, noise="philox", f_lip=0.3, c_N=0.05, a_W_T=60)
    e.set_params(0, start)
    hist = fit.fit(e, ["a_W_T"], target[0], iters=6, window=60, ckpt=20, spec=spec, lr=2.0)
    assert hist[-1]["values"][0] > 60.0
    assert all(np.isfinite(h["loss"]) for h in hist)


def test_batched_adjoint_rows_equal_solo_boxes(cuda_ok):
    """configuration 5 at reduced size: 4 of its 64 boxes (L = 128, lipid
    fraction U(0.1, 0.3)) in one engine; each replica's loss and gradient row
    equal those of the same box run alone"""
    from oercel_b200 import workloads
    ps = workloads.config5(n_replicas=4)
    spec = ob.Engine.rdf_spec(nbin=64, rmax=2.0, sigma=0.05, last_steps=10, horizon=10)
    target = np.ones(64)
    e = ob.Engine(ps)
    for r in range(len(ps)):
        e.load_soup(r)
    e.prime()
    e.step(50)
    loss, grad, _ = e.window_adjoint(40, 20, spec, target)
    for r, p in enumerate(ps):
        s = ob.Engine(p)
        s.load_soup(0)
        s.prime()
        s.step(50)
        l1, g1, _ = s.window_adjoint(40, 20, spec, target)
        assert loss[r] == pytest.approx(l1[0], rel=1e-9)
        assert np.allclose(grad[r], g1[0], rtol=1e-6, atol=1e-9 * np.abs(g1[0]).max())
        s.close()


def test_batched_fit_moves_the_shared_repulsion(cuda_ok):
    """configuration 5's pattern on 4 boxes: per-box targets g_TT(r) made at
    a_W_T = 75, one a_W_T shared by every box fitted from 60 with the summed
    gradient rows"""
    from oercel_b200 import fit, workloads
    truth = workloads.config5(n_replicas=4)
    e = ob.Engine(truth)
    for r in range(len(truth)):
        e.load_soup(r)
    e.prime()
    e.step(200)
    spec = ob.Engine.rdf_spec(nbin=32, rmax=2.0, sigma=0.1, last_steps=20, horizon=10)
    _, target = e.window_loss(60, spec, np.zeros(32))
    for r, p in enumerate(workloads.config5(n_replicas=4, a_wt=60.0)):
        e.set_params(r, p)
    hist = fit.fit(e, ["a_W_T"], target, iters=6, window=60, ckpt=20, spec=spec, lr=2.0)
    assert hist[-1]["values"][0] > 60.0
    assert all(np.isfinite(h["loss"]) for h in hist)


def test_fit_graph_equals_the_eager_fit(cuda_ok):
    """dpd_fit_graph (windows, losses, gradients and Adam steps all on the
    device, one captured iteration replayed) against the same fit driven from
    the host: window_adjoint per iteration, the replicas' gradients summed, the
    Adam step of torch.optim.Adam in numpy, set_params"""
    def boxes():  # each engine its own parameter objects
        return [params(L=12.0, seed=41, noise="philox", f_lip=0.3, c_N=0.1, a_W_T=60.0),
                params(L=10.0, seed=42, noise="philox", f_lip=0.2, c_N=0.1, a_W_T=60.0)]
    ns = [p.n_beads() for p in boxes()]
    a, b = ob.Engine(boxes(), n_beads=ns), ob.Engine(boxes(), n_beads=ns)
    for e in (a, b):
        for r in range(2):
            e.load_soup(r)
        e.prime()
        e.step(20)
    spec = ob.Engine.rdf_spec(ta=2, tb=2, nbin=32, rmax=2.0, sigma=0.1, last_steps=4)
    target = np.linspace(0.5, 1.5, 32)
    nsteps, ckpt, iters, lr = 10, 5, 3, 0.5
    loss_g, grad_g, vals_g = a.fit_graph(["a_W_T"], nsteps, ckpt, spec, target, iters, lr=lr)
    b1, b2, eps = 0.9, 0.999, 1e-8
    val, m, v = 60.0, 0.0, 0.0
    for it in range(iters):
        assert vals_g[it, 0] == pytest.approx(val, rel=1e-9)
        loss, grad, _ = b.window_adjoint(nsteps, ckpt, spec, target)
        g = float(grad[0][2] + grad[1][2])
        tol = 1e-9 if it == 0 else 1e-4  # (later windows start from values equal to rounding)
        assert loss_g[it] == pytest.approx(loss, rel=tol)
        assert grad_g[it, 0] == pytest.approx(g, rel=max(tol, 1e-9))
        t = it + 1
        m = m + (1 - b1) * (g - m)
        v = b2 * v + (1 - b2) * g * g
        val = val - lr / (1 - b1 ** t) * m / (np.sqrt(v) / np.sqrt(1 - b2 ** t) + eps)
        for r in range(2):
            p = b.params[r]
            p.a[0][2] = p.a[2][0] = val
            b.set_params(r, p)
    assert vals_g[iters, 0] == pytest.approx(val, rel=1e-6)
    assert a.params[0].a[0][2] == vals_g[iters, 0]
    assert a.step_no == b.step_no
    sa, sb = a.state(0), b.state(0)
    assert np.allclose(sa["x"], sb["x"], atol=1e-3)
