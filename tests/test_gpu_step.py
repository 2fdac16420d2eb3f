"""The fused production step against its phases, the reference's trajectory and
the reference's equilibrium statistics (through the C ABI)."""
import numpy as np
import pytest

import oercel_b200 as ob
from conftest import golden
from gpu_util import engine_with, params, rel_err

pytestmark = pytest.mark.gpu


def primed(L=16, seed=5, noise="mix13", **kv):
    p = params(L=L, seed=seed, noise=noise, **kv)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    return p, e


def clone(p, e):
    """a second engine holding the same state (slot order, vh, f, step)"""
    s = e.state()
    e2 = engine_with(p, s["x"], s["y"], s["vhx"], s["vhy"], s["type"], s["prev"], s["next"], gid=s["gid"])
    e2.set_dynamics(0, s["vhx"], s["vhy"], s["fx"], s["fy"])
    e2.resume()
    e2.set_step(e.step_no)
    return e2


def same_state(a, b, keys=("x", "y", "vhx", "vhy", "vtx", "vty", "fx", "fy", "type", "gid", "prev", "next")):
    for k in keys:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("noise", ["philox", "mix13"])
def test_fused_step_equals_phases(cuda_ok, noise):
    """one dpd_step (scan, place, stable fix-up, permute + integrate, forces + next keys)
    is bit-identical to dpd_integrate, dpd_build_cells, dpd_forces in turn"""
    p, a = primed(noise=noise)
    a.step(3)
    b = clone(p, a)
    s0 = a.step_no
    a.step(1)
    b.integrate()
    b.build_cells()
    b.forces(s0 + 1)
    sa, sb = a.state(), b.state()
    same_state(sa, sb, keys=("x", "y", "vhx", "vhy", "vtx", "vty", "fx", "fy", "type", "gid", "prev", "next"))
    assert np.array_equal(a.cells(), b.cells())


def test_sort_falls_back_when_a_bead_jumps_cells(cuda_ok):
    """a step in which one bead moves two cells gives the same stable sort (and
    the same state) as dpd_integrate, dpd_build_cells and dpd_forces in turn"""
    p, a = primed(noise="philox")
    a.step(3)
    b = clone(p, a)
    s0 = a.step_no
    for e in (a, b):
        vhx = e.state()["vhx"].copy()
        vhx[11] = 100.0  # dt 0.02: two cells in one step
        e.set_dynamics(0, vhx=vhx)
    a.step(1)
    b.integrate()
    b.build_cells()
    b.forces(s0 + 1)
    same_state(a.state(), b.state())
    assert np.array_equal(a.cells(), b.cells())
    a.step(2)


def test_graph_replay_equals_eager(cuda_ok, monkeypatch):
    """a CUDA-graph replay of the step gives the same bits as eager launches"""
    p, a = primed(noise="philox")
    monkeypatch.setenv("DPD_NO_GRAPH", "1")
    b = clone(p, a)
    b.step(200)
    monkeypatch.delenv("DPD_NO_GRAPH")
    a.step(200)  # 1024 beads: graphs of 64 steps
    same_state(a.state(), b.state())


def test_trajectory_tracks_reference(cuda_ok):
    """the reference's own soup, forces and noise (mix13), 20 steps: the kinetic
    temperature of every step agrees with the reference's FP64 run to 1e-3"""
    g = golden("traj_L16_seed5.npz")
    p, e = primed(L=16, seed=5, noise="mix13")
    T = []
    for _ in range(20):
        e.step(1)
        T.append(e.observables(0)["T"])
    assert rel_err(T, g["T"]) < 1e-3


def test_restart_continuation_is_bitwise(cuda_ok):
    """state read out and loaded into a new engine continues bit-identically
    (the reference's checkpoint/restart guarantee, validate.sh:80-105)"""
    p, a = primed(noise="philox")
    a.step(10)
    b = clone(p, a)
    a.step(25)
    b.step(25)
    same_state(a.state(), b.state())


def test_equilibrium_statistics_match_reference(cuda_ok):
    """configuration 1 for 10^4 steps: <T>, the conservative virial and the T-T
    pair histogram agree with the reference's FP64 run within the statistical
    error (criteria of cel/engine_gpu/tests/compare.py:103-127)"""
    g = golden("stats_config1.npz")
    p = params(L=32, seed=0, noise="philox")
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(int(g["equil"]))
    T, vir, hist = [], [], []
    every = int(g["every"])
    for _ in range((int(g["nsteps"]) - int(g["equil"])) // every):
        e.step(every)
        o = e.observables(0)
        T.append(o["T"])
        vir.append(o["virial"])
        hist.append(e.pair_hist(0, 2, 2, 2.0, 64))
        assert abs(o["px"]) < 1e-2 and abs(o["py"]) < 1e-2
    T, vir, hist = np.array(T), np.array(vir), np.array(hist)

    def blocks(v):
        b = np.array([c.mean(axis=0) for c in np.array_split(v, 20)])
        return v.mean(axis=0), b.std(axis=0, ddof=1) / np.sqrt(20)

    (Tm, Te), (Vm, Ve), (Hm, He) = blocks(T), blocks(vir), blocks(hist)
    assert abs(Tm - g["T"]) < max(4 * np.hypot(Te, g["T_err"]), 0.003)
    rho = 4.0
    P_gpu, P_ref = rho * Tm + Vm, rho * g["T"] + g["virial"]
    assert abs(P_gpu - P_ref) / P_ref < 0.01
    sig = np.hypot(He, g["tt_hist_err"])
    z = np.abs(Hm - g["tt_hist"]) / np.maximum(sig, 0.05 * np.maximum(g["tt_hist"], 1.0))
    assert z.max() < 5.0
