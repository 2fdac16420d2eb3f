"""The reference's catalyst chemistry on the GPU (chem_kind = catalyst).

Against the reference itself: one chemistry check from a sorted state with FP32
positions (tests/golden/catalyst_*.npz, made by the reference's own check) must
give the same types, links and serial generator state exactly, the same events,
and positions and velocities of the new chains within 2e-6 (the reference keeps
them in FP64, the engine in FP32).  Runs through the drop-in executable
are checked against the reference executable in test_gpu_cli.py.
"""
import numpy as np
import pytest

import oracle as O
import oercel_b200 as ob
from conftest import golden
from gpu_util import params

pytestmark = pytest.mark.gpu
# pi: two-headed lipids with one tail each, a rung and junction terms (the template's placement and relaxation)
CASES = ["catalyst_L16_seed12.npz", "catalyst_vent_L16_seed13.npz", "catalyst_pi_L16_seed14.npz"]


def ini_items(g):
    return [tuple(line.split(" = ", 1)) for line in bytes(g["ini"]).decode().strip().split("\n")]


def engine_for(name):
    g = golden(name)
    p = ob.Params().update(ini_items(g) + [("noise", "mix13")])
    nxt = g["nxt0"].astype(np.int32)
    prev = np.full_like(nxt, -1)
    prev[nxt[nxt >= 0]] = np.nonzero(nxt >= 0)[0]
    e = ob.Engine(p, n_beads=len(g["x0"]))
    e.set_state(0, g["x0"].astype(np.float32), g["y0"].astype(np.float32), g["vx0"].astype(np.float32),
                g["vy0"].astype(np.float32), g["type0"].astype(np.uint8), g["gid0"].astype(np.uint32), prev, nxt)
    e.set_dynamics(0, vtx=g["vtx0"], vty=g["vty0"])
    e.set_rng(0, g["rng0"])
    e.build_cells()
    return g, p, e


@pytest.mark.parametrize("name", CASES)
def test_catalyst_check_matches_reference(cuda_ok, name):
    g, p, e = engine_for(name)
    assert np.array_equal(e.state()["gid"], g["gid0"])  # the sort kept the reference's slot order
    assert np.array_equal(e.cells(), g["cstart"])
    e.chemistry(int(g["step"]))
    s = e.state()
    assert np.array_equal(e.rng(0), g["rng1"])
    assert np.array_equal(s["type"], g["type1"])
    assert np.array_equal(s["next"], g["nxt1"])
    L = float(np.float32(p.L))
    for k in ("x", "y"):
        d = s[k].astype(np.float64) - g[f"{k}1"]
        d -= L * np.round(d / L)
        assert np.abs(d).max() < 2e-6, k
    for k, r in (("vhx", "vx1"), ("vhy", "vy1"), ("vtx", "vtx1"), ("vty", "vty1")):
        assert np.abs(s[k] - g[r]).max() < 1e-6, k
    ref = sorted((int(r["kind"]) + 3, int(r["i"]), int(r["variant"])) for r in g["events"])
    got = sorted((ev[1], ev[2], ev[3] if ev[3] < 2**31 else ev[3] - 2**32) for ev in e.events())
    assert got == ref


def test_catalyst_steps_are_deterministic_across_graphs(cuda_ok, monkeypatch):
    """steps with a catalyst check every 3 steps: graph replays and eager
    launches give the same bits, and the net force stays zero"""
    g = golden(CASES[0])
    p = ob.Params().update(ini_items(g) + [("noise", "philox"), ("n_chem", "3")])
    runs = []
    for eager in (False, True):
        if eager:
            monkeypatch.setenv("DPD_NO_GRAPH", "1")
        e = ob.Engine(p)
        e.load_soup(0)
        e.prime()
        e.step(40)
        ev = [tuple(None if isinstance(v, float) and v != v else v for v in r) for r in e.events()]  # feed: NaN x, y
        runs.append((e.state(), sorted(ev, key=repr), e.rng(0)))
    a, b = runs
    for k in ("x", "y", "vhx", "fx", "type", "gid", "prev", "next"):
        assert np.array_equal(a[0][k], b[0][k]), k
    assert a[1] == b[1] and np.array_equal(a[2], b[2])
    assert {ev[1] for ev in a[1]} & {3, 4}  # syntheses and replications happened
    assert abs(a[0]["fx"].astype(np.float64).sum()) < 1e-9


CAT = dict(chem=1, chem_kind="catalyst", f_Ka=0.03, f_Kb=0.02, c_N=0.25, p_syn_a=0.5, p_syn_b=0.6, p_rep_a=0.4,
           p_rep_b=0.4, mu=0.3, p_ld=0.05, p_kd=0.05, p_nd=0.03, p_feed=0.05, feed_cap=0.27, warmup=0,
           noise="philox")


def oracle_blocks(p):
    """the oracle's parameter blocks for an engine's Params"""
    L = float(np.float32(p.L))
    op = O.params(L, np.array(p.a, dtype=np.float64), dt=p.dt, k_bond=p.k_bond, r0=p.r0, seed=p.seed,
                  k_angle=p.k_angle)
    feed = {"none": 0, "0": 0, "uniform": 1, "vent": 2}[p.feed]
    vent = {"disk": 0, "vstrip": 1, "hstrip": 2}[p.vent_shape]
    c = O.cat(r_cat=p.r_cat, syn_tries=int(p.syn_tries), syn_relax=int(p.syn_relax), syn_nN=int(p.syn_nN),
              nH=int(p.lip_nH), nT=int(p.lip_nT), feed_mode=feed, vent_kind=vent, p_syn_a=p.p_syn_a,
              p_syn_b=p.p_syn_b, p_rep_a=p.p_rep_a, p_rep_b=p.p_rep_b, mu=p.mu, p_ld=p.p_ld, p_kd=p.p_kd,
              p_nd=p.p_nd, p_feed=p.p_feed, feed_cap=p.feed_cap,
              vent_x=0.5 * L if p.vent_x < 0 else p.vent_x, vent_y=0.5 * L if p.vent_y < 0 else p.vent_y,
              vent_r=p.vent_r, vent_w=p.vent_w)
    return op, c


# low rates: nearly every catalyst is decided from the counts found before the walk
LOW = dict(p_syn_a=0.01, p_syn_b=0.03, p_rep_a=0.01, p_rep_b=0.01, mu=0.2, p_ld=0.002, p_kd=0.002, p_nd=0.002,
           p_feed=0.01)


@pytest.mark.parametrize("L, feed, rates", [(40, "uniform", {}), (40, "vent", {}), (100, "uniform", LOW)])
def test_catalyst_check_matches_the_oracle_on_a_large_box(cuda_ok, L, feed, rates):
    """a box evolved by the engine (L = 40: 4800 beads, about 240 catalysts, high
    rates; L = 100: 30000 beads, about 1500 catalysts in two windows of the
    walk, low rates): one check on the GPU against the oracle's serial
    restatement on the same sorted state, cell index and generator state"""
    p = ob.Params(L=L, seed=7, n_chem=10, feed=feed, **dict(CAT, **rates))
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(19)  # includes the engine's own check at step 10
    assert {ev[1] for ev in e.events()} & {3, 4}  # read (and cleared) before the compared check
    s, cs, rng = e.state(), e.cells(), e.rng(0)
    op, oc = oracle_blocks(p)
    st = {k: s[k].copy() for k in ("x", "y", "vhx", "vhy", "vtx", "vty", "type", "gid", "prev", "next")}
    orng = rng.copy()
    _, oev = O.catalyst_chemistry(op, oc, st, cs.astype(np.int32), 20, orng)
    e.chemistry(20)
    g = e.state()
    assert np.array_equal(e.rng(0), orng)
    assert np.array_equal(g["type"], st["type"]) and np.array_equal(g["next"], st["next"])
    assert np.array_equal(g["prev"], st["prev"])
    for k in ("x", "y", "vhx", "vhy", "vtx", "vty"):
        assert np.abs(g[k].astype(np.float64) - st[k]).max() <= 1e-5, k
    got = sorted((ev[1], ev[2], ev[3] if ev[3] < 2**31 else ev[3] - 2**32) for ev in e.events())
    ref = sorted((ev[1], ev[2], ev[3]) for ev in oev)
    assert got == ref
    assert {k for k, _, _ in ref} >= {3, 4, 6, 7, 8, 9}  # syn, rep, decays and feed all happened
    assert len([k for k, _, _ in ref if k in (3, 4, 5)]) < (100 if rates else 1000)


def test_mixed_chemistries_in_one_batch_equal_solo_runs(cuda_ok):
    """a catalyst replica (check every 3 steps) and a lipid-chemistry replica
    in one engine give bit for bit the runs of each alone"""
    p_cat = ob.Params(L=16, seed=7, n_chem=3, **CAT)
    p_lip = params(L=16, seed=9, chem=1, chem_kind="lipid", n_chem=1, p_grow=0.05, p_bond=0.3, p_break=0.02)

    def run(plist):
        e = ob.Engine(plist)
        for r in range(len(plist)):
            e.load_soup(r)
        e.prime()
        e.step(30)
        ev = [tuple(None if isinstance(v, float) and v != v else v for v in x) for x in e.events()]
        return e, ev

    both, ev_both = run([p_cat, p_lip])
    for r, p in enumerate([p_cat, p_lip]):
        solo, ev_solo = run([p])
        a, b = both.state(r), solo.state(0)
        for k in a:
            assert np.array_equal(a[k], b[k]), (r, k)
        assert np.array_equal(both.rng(r), solo.rng(0))
        mine = sorted((x[:6] for x in ev_both if x[6] == r), key=repr)
        assert mine == sorted((x[:6] for x in ev_solo), key=repr) and mine, r


def test_catalyst_replicas_of_uneven_size_equal_solo_runs(cuda_ok):
    """three catalyst replicas of different sizes and settings in one engine
    (their draw streams, lists and scratch at different offsets) give bit for
    bit the runs of each alone"""
    plist = [ob.Params(L=16, seed=7, n_chem=3, **CAT),
             ob.Params(L=24, seed=8, n_chem=2, **dict(CAT, p_syn_a=0.2, p_rep_a=0.1)),
             ob.Params(L=18, seed=9, n_chem=3, feed="vent", **CAT)]

    def run(ps):
        e = ob.Engine(ps)
        for r in range(len(ps)):
            e.load_soup(r)
        e.prime()
        e.step(24)
        ev = [tuple(None if isinstance(v, float) and v != v else v for v in x) for x in e.events()]
        return e, ev

    both, ev_both = run(plist)
    for r, p in enumerate(plist):
        solo, ev_solo = run([p])
        a, b = both.state(r), solo.state(0)
        for k in a:
            assert np.array_equal(a[k], b[k]), (r, k)
        assert np.array_equal(both.rng(r), solo.rng(0))
        mine = sorted((x[:6] for x in ev_both if x[6] == r), key=repr)
        assert mine == sorted((x[:6] for x in ev_solo), key=repr) and mine, r


def test_catalyst_check_with_the_shuffle_scratch_in_global_memory(cuda_ok):
    """a 480 x 480 box with about 11,500 catalysts: more than the shuffle keeps
    in shared memory; one check against the oracle"""
    p = ob.Params(L=480, seed=3, n_chem=10, **dict(CAT, **LOW))
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(9)
    s, cs, rng = e.state(), e.cells(), e.rng(0)
    assert int(np.isin(s["type"], (4, 5)).sum()) > 11264
    op, oc = oracle_blocks(p)
    st = {k: s[k].copy() for k in ("x", "y", "vhx", "vhy", "vtx", "vty", "type", "gid", "prev", "next")}
    orng = rng.copy()
    _, oev = O.catalyst_chemistry(op, oc, st, cs.astype(np.int32), 10, orng, evcap=1 << 18)
    e.chemistry(10)
    g = e.state()
    assert np.array_equal(e.rng(0), orng)
    assert np.array_equal(g["type"], st["type"]) and np.array_equal(g["next"], st["next"])
    got = sorted((ev[1], ev[2], ev[3] if ev[3] < 2**31 else ev[3] - 2**32) for ev in e.events())
    assert got == sorted((ev[1], ev[2], ev[3]) for ev in oev)
