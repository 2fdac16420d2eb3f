"""Helpers shared by the GPU tests: engines on prepared states and oracle views of them."""
import numpy as np

import oracle as O
import oercel_b200 as ob
from conftest import amat_config

# physics of the workloads (configuration 1 of the workload table)
BASE = dict(rho=4, dt=0.02, gamma=4.5, kT=1, k_bond=100, r0=0.5, k_angle=0, lip_nH=1, lip_nT=2, f_lip=0.15,
            f_Ka=0, f_Kb=0, c_N=0.05, chem=0, chem_kind="lipid", warmup=0, a_W_H=25, a_W_T=75, a_H_T=50, a_W_P=25,
            a_H_P=25, a_P_T=75)


def params(**kv):
    d = dict(BASE)
    d.update(kv)
    return ob.Params(**d)


def oracle_params(p: ob.Params, noise=None):
    a = np.array(p.a, dtype=np.float64)
    return O.params(float(np.float32(p.L)), a, dt=p.dt, lam=p["lambda"], gamma=p.gamma, kT=p.kT, k_bond=p.k_bond,
                    r0=p.r0, seed=p.seed, noise=(0 if p.noise == "philox" else 1) if noise is None else noise)


def links_from_next(nxt):
    nxt = np.asarray(nxt, np.int32)
    prev = np.full_like(nxt, -1)
    m = nxt >= 0
    prev[nxt[m]] = np.nonzero(m)[0]
    return prev, nxt


def engine_with(p, x, y, vx, vy, type_, prev=None, nxt=None, gid=None):
    e = ob.Engine(p, n_beads=len(x))
    e.set_state(0, np.asarray(x, np.float32), np.asarray(y, np.float32), np.asarray(vx, np.float32),
                np.asarray(vy, np.float32), np.asarray(type_, np.uint8), gid, prev, nxt)
    return e


def oracle_state(s):
    """engine state dict -> oracle state dict (float32 arrays, links)"""
    return dict(x=s["x"].copy(), y=s["y"].copy(), vtx=s["vtx"].copy(), vty=s["vty"].copy(), vhx=s["vhx"].copy(),
                vhy=s["vhy"].copy(), fx=s["fx"].copy(), fy=s["fy"].copy(), type=s["type"].copy(),
                gid=s["gid"].copy(), prev=s["prev"].copy(), next=s["next"].copy())


def rel_err(got, ref):
    """max |got - ref| over the largest |ref| (the force criterion of the tests)"""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30)


def by_gid(s, key):
    out = np.empty_like(s[key])
    out[s["gid"]] = s[key]
    return out


def links_by_gid(s):
    """(prev gid, next gid) per gid, -1 = none"""
    g = s["gid"].astype(np.int64)
    pv = np.where(s["prev"] >= 0, g[np.maximum(s["prev"], 0)], -1)
    nx = np.where(s["next"] >= 0, g[np.maximum(s["next"], 0)], -1)
    P = np.empty(len(g), np.int64)
    Nn = np.empty(len(g), np.int64)
    P[g] = pv
    Nn[g] = nx
    return P, Nn


def naive_chain_and_stir_forces(torch, x, prv, nxt, ka, L, stir_A, stir_n):
    """angle terms U = ka (1 - cos) of every chain triplet (oercel.c:1237-1256) and the
    stirring body force A sin(2 pi n y / L) less its mean (oercel.c:1183-1195), float64"""
    F = torch.zeros_like(x)
    j = np.nonzero((prv >= 0) & (nxt >= 0))[0]
    if ka != 0.0 and len(j):
        p_, n_ = prv[j], nxt[j]
        a = x[j] - x[p_]
        a = a - L * torch.round(a / L)
        c = x[n_] - x[j]
        c = c - L * torch.round(c / L)
        cos = (a * c).sum(-1) / (a.norm(dim=-1) * c.norm(dim=-1))
        U = (ka * (1.0 - cos)).sum()
        F = F - torch.autograd.grad(U, x, create_graph=True)[0]
    if stir_A != 0.0:
        f = stir_A * torch.sin(2.0 * np.pi * stir_n * x[:, 1] / L)
        F = F + torch.stack([f - f.mean(), torch.zeros_like(f)], -1)
    return F
