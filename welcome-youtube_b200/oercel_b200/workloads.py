"""The benchmark workloads, as parameter sets with synthetic seeded inputs.

  config1  L = 32, rho = 4 (4096 beads), W/H/T/P soup: 80 % W, 5 % P, H-T-T
           lipids; chemistry off; the reference CPU engine's own case
  config2  the same physics at L = 512 (1,048,576 beads) with the lipid
           chemistry every step (P -> T growth 1e-3, H-T break 1e-5, free
           T + free H bonding 1e-2), Philox seed 1
  config3  256 replicas, bead counts log-uniform in [2048, 65536] at rho = 4
           in square boxes, per-replica seed, every off-diagonal a_ij scaled
           by U(0.9, 1.1), chemistry rates scaled by U(0.5, 2)
Repulsions: 25 like-like, W-T = P-T = 75, H-T = 50, W-H = W-P = H-P = 25;
gamma = 4.5, sigma = 3 (kT = 1), dt = 0.02, k = 100, r0 = 0.5.  The
reference publishes no dataset for these runs; all inputs are seeded soups.
"""
from __future__ import annotations

import math

import numpy as np

from .params import Params

PHYSICS = dict(rho=4, dt=0.02, gamma=4.5, kT=1, k_bond=100, r0=0.5, k_angle=0, lip_nH=1, lip_nT=2, f_lip=0.15,
               f_Ka=0, f_Kb=0, c_N=0.05, warmup=0, a_W_H=25, a_W_T=75, a_H_T=50, a_W_P=25, a_H_P=25, a_P_T=75)
CHEMISTRY = dict(chem=1, chem_kind="lipid", n_chem=1, p_grow=1e-3, p_break=1e-5, p_bond=1e-2, r_grow=1.0, r_bond=0.6,
                 n_t_min=2)


def config1(seed=0, **kv):
    d = dict(PHYSICS, L=32, seed=seed, chem=0)
    d.update(kv)
    return Params(**d)


def config2(seed=1, **kv):
    d = dict(PHYSICS, L=512, seed=seed, **CHEMISTRY)
    d.update(kv)
    return Params(**d)


def config3(n_replicas=256, seed=2026, nmin=2048, nmax=65536, chem=True):
    """list of (Params, n_beads) for the batched ensemble"""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n_replicas):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        L = float(np.float32(math.sqrt(n / 4.0)))
        d = dict(PHYSICS, L=L, seed=1000 + b)
        if chem:
            d.update(CHEMISTRY)
            s = rng.uniform(0.5, 2.0)
            d.update(p_grow=CHEMISTRY["p_grow"] * s, p_break=CHEMISTRY["p_break"] * s, p_bond=CHEMISTRY["p_bond"] * s)
        else:
            d["chem"] = 0
        p = Params(**d)
        for i in range(8):
            for j in range(i + 1, 8):
                p.a[i][j] = p.a[j][i] = p.a[i][j] * rng.uniform(0.9, 1.1)
        out.append((p, p.n_beads()))
    return out


def config4(a_wt=75.0, seed=4):
    """the differentiated fit: L = 64 (16384 beads), chemistry frozen"""
    return Params(**dict(PHYSICS, L=64, seed=seed, chem=0, a_W_T=a_wt))


def config5(n_replicas=64, seed=2027, a_wt=75.0):
    """the batched adjoint: 64 boxes of L = 128 (65536 beads), lipid fraction U(0.1, 0.3)"""
    rng = np.random.default_rng(seed)
    return [Params(**dict(PHYSICS, L=128, seed=3000 + b, chem=0, a_W_T=a_wt, f_lip=float(rng.uniform(0.1, 0.3))))
            for b in range(n_replicas)]


# The reference's big-soup experiment (cel/pc/plan.txt item 1): a random soup of L = 512
# with the membrane physics of cel/engine/params/membranes.ini (tied H2T2 pi lipids, the
# demixing repulsions) and the plan's chemistry rates, a check every 10 steps.  Every key
# is a reference key.
CATALYST_PLAN = dict(L=512, dt=0.03, kT=1, gamma=4.5, warmup=3000, f_lip=0.20, f_Ka=0.01, f_Kb=0, c_N=0.10,
                     lip_arch="pi", lip_nT=1, lip_tie=1, r0_head=0.7, k_head=0, k_bond=300, r0=0.5, k_angle=15,
                     syn_nN=0, a_W_H=20, a_W_T=200, a_H_T=50, a_W_N=45, a_H_N=22, a_T_N=120, a_W_K=45, a_H_K=30,
                     a_T_K=200, chem=1, events=1, n_chem=10, p_syn_a=3e-5, p_syn_b=1e-4, p_rep_a=1e-5,
                     p_rep_b=1e-5, mu=0.02, p_ld=2e-6, p_kd=5e-6, p_nd=1e-6, feed="uniform", p_feed=1e-4,
                     feed_cap=0.12)


def catalyst_plan(seed=1, **kv):
    """the catalyst chemistry workload: 786,432 beads, about 7,900 catalysts"""
    return Params().update([(k, str(v)) for k, v in dict(CATALYST_PLAN, seed=seed, **kv).items()])


def catalyst_plan_ini(seed: int, steps: int, threads: int) -> str:
    """the reference engine's ini for catalyst_plan(seed)"""
    kv = dict(CATALYST_PLAN, seed=seed, steps=steps, threads=threads, snap_every=0, stats_every=steps,
              ckpt_every=0, log_every=0)
    return "".join(f"{k} = {v}\n" for k, v in kv.items())


def reference_ini(p: Params, steps: int, threads: int) -> str:
    """the reference engine's ini for the physics of p (type 3 is its N; its
    catalyst chemistry is switched off: the lipid rules do not exist there)"""
    a = p.a
    lines = [f"L = {p.L!r}", f"rho = {p.rho!r}", f"dt = {p.dt!r}", f"lambda = {p['lambda']!r}",
             f"gamma = {p.gamma!r}", f"kT = {p.kT!r}", f"k_bond = {p.k_bond!r}", f"r0 = {p.r0!r}", "k_angle = 0",
             f"lip_nH = {p.lip_nH}", f"lip_nT = {p.lip_nT}", f"f_lip = {p.f_lip!r}", "f_Ka = 0", "f_Kb = 0",
             f"c_N = {p.c_N!r}", "chem = 0", "events = 0", "warmup = 0", f"seed = {p.seed}", f"steps = {steps}",
             "snap_every = 0", f"stats_every = {steps}", "ckpt_every = 0", "log_every = 0", f"threads = {threads}",
             "nsub = 4"]
    names = ["W", "H", "T", "N"]
    for i in range(4):
        for j in range(i, 4):
            lines.append(f"a_{names[i]}_{names[j]} = {a[i][j]!r}")
    return "\n".join(lines) + "\n"
