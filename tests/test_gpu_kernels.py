"""Parity of each CUDA phase with the oracle and the reference (through the C ABI).

Criteria: cell assignment, cell starts, the sort permutation, link topology and
the FP32 integrator are bit-exact; forces are within 1e-5 relative to the
largest force (max |F_gpu - F_ref| <= 1e-5 max |F_ref|), FP32 against FP64.
"""
import numpy as np
import pytest

import oercel_b200 as ob
import oracle as O
from conftest import golden
from gpu_util import (engine_with, links_from_next, oracle_params, oracle_state, params, rel_err)

pytestmark = pytest.mark.gpu
FORCE_TOL = 1e-5

CASES = [("step_L12p5_seed99.npz", 12.5, 99, 12345), ("step_L9_seed7.npz", 9.0, 7, 3)]


def fixture_engine(name, L, seed, noise="mix13", use_vt=True, **kv):
    g = golden(name)
    p = params(L=L, seed=seed, noise=noise, **kv)
    prev, nxt = links_from_next(g["nxt0"])
    v = (g["vtx0"], g["vty0"]) if use_vt else (g["vx0"], g["vy0"])
    e = engine_with(p, g["x0"], g["y0"], v[0], v[1], g["type0"], prev, nxt)
    return g, p, e


@pytest.mark.parametrize("name,L,seed,step", CASES)
def test_build_cells_matches_reference(cuda_ok, name, L, seed, step):
    g, p, e = fixture_engine(name, L, seed)
    e.build_cells()
    s = e.state()
    assert np.array_equal(e.cells(), g["cstart"])
    assert np.array_equal(s["gid"], g["gid"])
    # links follow the beads: next of slot d is the slot holding nxt0[gid[d]]
    nxt0 = g["nxt0"]
    slot = np.empty(len(s["gid"]), np.int64)
    slot[s["gid"]] = np.arange(len(slot))
    want = np.where(nxt0[s["gid"]] >= 0, slot[np.maximum(nxt0[s["gid"]], 0)], -1)
    assert np.array_equal(s["next"], want)
    assert np.array_equal(s["x"], g["x0"][s["gid"]].astype(np.float32))


@pytest.mark.parametrize("name,L,seed,step", CASES)
def test_pair_forces_match_reference(cuda_ok, name, L, seed, step):
    g, p, e = fixture_engine(name, L, seed, noise="mix13")
    e.build_cells()
    fx, fy = e.pair_forces(0, step)
    assert rel_err(fx, g[f"fx_{step}"]) < FORCE_TOL
    assert rel_err(fy, g[f"fy_{step}"]) < FORCE_TOL


@pytest.mark.parametrize("noise", ["philox", "mix13"])
def test_pair_forces_match_oracle(cuda_ok, noise):
    g, p, e = fixture_engine("step_L12p5_seed99.npz", 12.5, 99, noise=noise)
    e.build_cells()
    s = oracle_state(e.state())
    op = oracle_params(p)
    for step in (0, 1, 777):
        fx, fy = e.pair_forces(0, step)
        rx, ry = O.pair_forces(op, s, e.cells(), step, noise=True)
        assert rel_err(fx, rx) < FORCE_TOL and rel_err(fy, ry) < FORCE_TOL, step


def test_pair_forces_without_noise(cuda_ok):
    """sigma -> 0 (kT = 1e-20): conservative + dissipative forces only"""
    g, p, e = fixture_engine("step_L12p5_seed99.npz", 12.5, 99, noise="philox", kT=1e-20)
    e.build_cells()
    s = oracle_state(e.state())
    fx, fy = e.pair_forces(0, 5)
    rx, ry = O.pair_forces(oracle_params(p), s, e.cells(), 5, noise=False)
    assert rel_err(fx, rx) < FORCE_TOL and rel_err(fy, ry) < FORCE_TOL


@pytest.mark.parametrize("name,L,seed,step", CASES)
def test_bond_forces_match_reference(cuda_ok, name, L, seed, step):
    g, p, e = fixture_engine(name, L, seed)
    e.build_cells()
    bx, by, mb = e.bond_forces(0)
    assert rel_err(bx, g["bfx"]) < FORCE_TOL and rel_err(by, g["bfy"]) < FORCE_TOL
    assert mb == pytest.approx(float(g["maxbond"]), rel=1e-6)


def test_forces_deterministic_and_momentum_free(cuda_ok):
    g, p, e = fixture_engine("step_L12p5_seed99.npz", 12.5, 99, noise="philox")
    e.build_cells()
    e.forces(42)
    a = e.state()
    e.forces(42)
    b = e.state()
    assert np.array_equal(a["fx"], b["fx"]) and np.array_equal(a["fy"], b["fy"])
    # pair and bond terms cancel exactly in fixed point; what is left is the
    # final FP32 rounding of each bead's sum (<= 1/2 ulp each)
    ulp = np.spacing(np.abs(a["fx"]).astype(np.float32)).astype(np.float64)
    assert abs(a["fx"].astype(np.float64).sum()) <= 0.5 * ulp.sum()
    pair_plus_bond = e.pair_forces(0, 42)[0].astype(np.float64) + e.bond_forces(0)[0]
    assert np.abs(pair_plus_bond - a["fx"]).max() <= 4 * np.spacing(np.float32(np.abs(a["fx"]).max()))


def test_integrate_bit_exact_against_fp32_oracle(cuda_ok):
    g, p, e = fixture_engine("step_L12p5_seed99.npz", 12.5, 99)
    e.build_cells()
    rng = np.random.default_rng(3)
    n = len(g["x0"])
    vh = rng.normal(size=(2, n)).astype(np.float32)
    f = (80 * rng.normal(size=(2, n))).astype(np.float32)
    e.set_dynamics(0, vh[0], vh[1], f[0], f[1])
    before = e.state()
    e.integrate()
    after = e.state()
    st = dict(x=before["x"].copy(), y=before["y"].copy(), vhx=before["vhx"].copy(), vhy=before["vhy"].copy(),
              vtx=np.zeros(n, np.float32), vty=np.zeros(n, np.float32), fx=before["fx"], fy=before["fy"])
    assert O.integrate_f32(oracle_params(p), st) == 0
    for k in ("x", "y", "vhx", "vhy", "vtx", "vty"):
        assert np.array_equal(after[k], st[k]), k


@pytest.mark.parametrize("sort_mode", [0, 1, 2])
def test_sort_at_one_million_beads(cuda_ok, sort_mode):
    """size-independent properties at the 1M-bead size: the sort is the oracle's
    stable counting sort, bit for bit, and every bead lies in its cell; with
    the two-pass scan, the one-pass look-back scan (256 blocks, each waiting on
    its predecessors) and the block-local scan whose prefixes the placement
    adds"""
    import oercel_b200 as ob
    p = params(L=512, seed=1)
    s = ob.soup_for(p)
    e = engine_with(p, s["x"], s["y"], s["vx"], s["vy"], s["type"], s["prev"], s["next"])
    e.set_tuning(sort_mode=sort_mode)
    for _ in range(3):  # repeated launches: the look-back's epochs must keep the blocks' words apart
        e.build_cells()
    st = e.state()
    key, cs, src = O.sort(oracle_params(p), s["x"], s["y"])
    assert np.array_equal(e.cells(), cs)
    assert np.array_equal(st["gid"], src.astype(np.uint32))
    assert np.all(np.diff(key[src]) >= 0)


def test_scan_forms_give_the_same_steps(cuda_ok):
    """the production step with each form of the sort: bit-identical
    trajectories (with the lipid chemistry), through CUDA graphs of 4 steps"""
    import oercel_b200 as ob
    p = params(L=48, seed=12, noise="philox", chem=1, n_chem=1, p_grow=0.05, p_bond=0.2, p_break=0.01)
    runs = []
    for mode in (0, 1, 2):
        e = ob.Engine(p)
        e.set_tuning(sort_mode=mode, graph_steps=4)
        e.load_soup(0)
        e.prime()
        e.step(40)
        runs.append((e.state(), e.cells()))
    for r in runs[1:]:
        for k in ("x", "y", "vhx", "fx", "type", "gid", "prev", "next"):
            assert np.array_equal(runs[0][0][k], r[0][k]), k
        assert np.array_equal(runs[0][1], r[1])


def a_eff(a, warmup, warm_end, step):
    """the warm-up repulsion of the reference (cel/engine/oercel.c:1124-1129), rounded to FP32 like the engine's table"""
    a = np.asarray(a, np.float64)
    if warmup <= 0 or step >= warm_end:
        return a
    f = max(0.0, 1.0 - (warm_end - step) / warmup)
    return np.where(a > 25.0, 25.0 + (a - 25.0) * f, a).astype(np.float32).astype(np.float64)


def test_warmup_ramp_matches_oracle(cuda_ok):
    g, p, e = fixture_engine("step_L12p5_seed99.npz", 12.5, 99, noise="philox", warmup=100)
    e.build_cells()
    s = oracle_state(e.state())
    for step in (0, 1, 37, 99, 100, 5000):
        op = O.params(float(np.float32(p.L)), a_eff(p.a, 100, 100, step), dt=p.dt, lam=p["lambda"], gamma=p.gamma,
                      kT=p.kT, k_bond=p.k_bond, r0=p.r0, seed=p.seed, noise=0)
        fx, fy = e.pair_forces(0, step)
        rx, ry = O.pair_forces(op, s, e.cells(), step, noise=True)
        assert rel_err(fx, rx) < FORCE_TOL and rel_err(fy, ry) < FORCE_TOL, step
    # the ramp really changes the forces
    f0 = e.pair_forces(0, 0)[0]
    f1 = e.pair_forces(0, 100)[0]
    assert rel_err(f0, f1) > 1e-2


@pytest.mark.parametrize("force_kernel", [0, 1])   # cell tiles, per bead
def test_warmup_in_the_fused_step(cuda_ok, force_kernel):
    """the production step through the ramp: stored forces at step s use a_eff(s)"""
    import oercel_b200 as ob
    p = params(L=16.0, seed=4, noise="philox", warmup=30)
    e = ob.Engine(p)
    e.set_tuning(force_kernel=force_kernel)
    e.load_soup(0)
    e.prime()
    for n in (7, 13, 20):   # steps 7, 20 (inside the ramp) and 40 (after it)
        e.step(n)
        st = e.step_no
        s = oracle_state(e.state())
        op = O.params(float(np.float32(p.L)), a_eff(p.a, 30, 30, st), dt=p.dt, lam=p["lambda"], gamma=p.gamma,
                      kT=p.kT, k_bond=p.k_bond, r0=p.r0, seed=p.seed, noise=0)
        rx, ry = O.pair_forces(op, s, e.cells(), st, noise=True)
        rx, ry, _ = O.bond_forces(op, s, rx, ry)
        assert rel_err(s["fx"], rx) < FORCE_TOL and rel_err(s["fy"], ry) < FORCE_TOL, st


def extras_engine(force_kernel=0):
    """the state of tests/golden/extras_L12p5_seed21.npz with angle terms,
    stirring and the temperature cycle on (the reference's own forces there
    pin the oracle, tests/test_oracle.py)"""
    g = golden("extras_L12p5_seed21.npz")
    p = params(L=float(g["L"]), seed=int(g["seed"]), noise="mix13", k_angle=10, stir_A=1.5, stir_n=2, kT_amp=0.4,
               kT_period=37)
    prev, nxt = links_from_next(g["nxt0"])
    e = engine_with(p, g["x0"], g["y0"], g["vtx0"], g["vty0"], g["type0"], prev, nxt)
    e.set_tuning(force_kernel=force_kernel)
    e.build_cells()
    op = O.params(float(np.float32(p.L)), np.array(p.a, dtype=np.float64), dt=p.dt, lam=p["lambda"], gamma=p.gamma,
                  kT=p.kT, k_bond=p.k_bond, r0=p.r0, seed=p.seed, noise=1, k_angle=10, stir_A=1.5, stir_n=2,
                  kT_amp=0.4, kT_period=37)
    return g, p, e, op


def test_angle_terms_match_oracle(cuda_ok):
    g, p, e, op = extras_engine()
    s = oracle_state(e.state())
    bx, by, mb = e.bond_forces(0)
    rx, ry, rmb = O.bond_forces(op, s)
    assert rel_err(bx, rx) < FORCE_TOL and rel_err(by, ry) < FORCE_TOL
    assert abs(mb - rmb) < 1e-6
    assert abs(bx.astype(np.float64).sum()) < 1e-9  # the three shares of every angle term cancel exactly


def test_stirring_and_temperature_cycle_match_oracle(cuda_ok):
    g, p, e, op = extras_engine()
    s = oracle_state(e.state())
    step = int(g["step"])
    fx, fy = e.pair_forces(0, step)
    rx, ry = O.pair_forces(op, s, e.cells(), step, noise=True)
    O.stir_forces(op, s, rx)
    assert rel_err(fx, rx) < FORCE_TOL and rel_err(fy, ry) < FORCE_TOL
    assert fx.astype(np.float64).sum() == 0.0  # net stirring force exactly zero in fixed point


def test_extras_tile_and_bead_kernels_agree(cuda_ok):
    runs = []
    for fk in (0, 1):
        g, p, e, op = extras_engine(fk)
        e.forces(int(g["step"]))
        runs.append(e.state())
    assert np.array_equal(runs[0]["fx"], runs[1]["fx"]) and np.array_equal(runs[0]["fy"], runs[1]["fy"])


def test_stats_async_equals_stats(cuda_ok):
    """dpd_stats_async + dpd_stats_decode give the numbers of dpd_stats (two
    identical engines: a stats read restarts the running max bond)"""
    p = params(L=16, seed=5, chem=1, n_chem=1, p_grow=0.05, p_bond=0.3, p_break=0.02)
    rows = []
    for use_async in (False, True):
        e = ob.Engine(p)
        e.load_soup(0)
        e.prime()
        e.step(7)
        if use_async:
            raw = np.zeros(16, np.uint64)
            e.stats_async(0, raw)
            e.sync()
            rows.append(e.stats_decode(0, raw))
        else:
            rows.append(e.observables(0, virial=False))
    a, b = rows
    for k in ("T", "px", "py", "maxbond", "n_chains"):
        assert a[k] == b[k], k
    assert np.array_equal(a["counts"], b["counts"])


def test_set_state_checks_its_input(cuda_ok):
    """a type above 7, a link or gid out of range, a non-finite position: DPD_E_ARG,
    nothing out of range stored; finite positions outside [0, L) are wrapped in"""
    p = params(L=8, seed=3)
    e = ob.Engine(p)
    s = ob.make_soup(float(p.L), p.n_beads(), 3, nH=p.lip_nH, nT=p.lip_nT, f_lip=p.f_lip, c_N=p.c_N)
    base = dict(x=s["x"], y=s["y"], vx=s["vx"], vy=s["vy"], type=s["type"], prev=s["prev"], next=s["next"])
    for key, bad in (("type", 9), ("next", len(s["x"])), ("prev", -2), ("x", np.nan)):
        kv = {k: v.copy() for k, v in base.items()}
        kv[key][5] = bad
        with pytest.raises(ob.DpdError, match="set_state"):
            e.set_state(0, kv["x"], kv["y"], kv["vx"], kv["vy"], kv["type"], None, kv["prev"], kv["next"])
    with pytest.raises(ob.DpdError, match="set_state"):
        e.set_state(0, base["x"], base["y"], base["vx"], base["vy"], base["type"],
                     np.full(len(s["x"]), len(s["x"]) + 3, np.uint32), base["prev"], base["next"])
    kv = {k: v.copy() for k, v in base.items()}
    kv["x"][0], kv["y"][1] = np.float32(p.L), np.float32(-0.5)
    e.set_state(0, kv["x"], kv["y"], kv["vx"], kv["vy"], kv["type"], None, kv["prev"], kv["next"])
    st = e.state()
    assert np.all((st["x"] >= 0) & (st["x"] < p.L) & (st["y"] >= 0) & (st["y"] < p.L))
    assert st["x"][0] == 0.0 and st["y"][1] == np.float32(p.L) - np.float32(0.5)
    e.prime()
    e.step(5)


def test_stats_ring_rows_equal_stats_async(cuda_ok):
    """rows the steps write into a pinned ring (4-step graphs) equal the rows of
    dpd_stats_async after each eager step of the same run, word 6 the step; a
    pageable ring is refused"""
    import torch
    p = params(L=16, seed=4)
    a, b = ob.Engine(p), ob.Engine(p)
    for e in (a, b):
        e.load_soup(0)
        e.prime()
    ring = torch.zeros((8, 16), dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    with pytest.raises(ob.DpdError, match="pinned"):
        a.stats_ring(0, np.zeros((8, 16), np.uint64))
    a.stats_ring(0, ring)
    a.set_graph_steps(4)
    b.set_graph_steps(1)
    for _ in range(3):
        a.step(4)
        rows = {int(r[6]): r.copy() for r in ring}
        for _ in range(4):
            b.step(1)
            raw = np.zeros(16, np.uint64)
            b.stats_async(0, raw)
            b.sync()
            got = rows[b.step_no].copy()
            got[6] = 0
            assert np.array_equal(got, raw)
    a.stats_ring(0, None)
    a.step(4)
    assert max(int(r[6]) for r in ring) == 12  # no row after the ring was stopped


@pytest.mark.parametrize("rho,chem", [(4, 0), (7, 0), (4, 1)])
def test_stats_ring_of_one_replica_in_a_batch(cuda_ok, rho, chem):
    """the tile force kernel assembles the ring's row itself: replica 1 of a
    two-box engine gives the rows that dpd_stats_async gives for it; at rho 7 the
    14 x 14 tiles hold more beads than shared memory does and take the direct
    path; with the lipid chemistry every step the types and chains change under
    the rows"""
    import torch
    kv = dict(noise="philox", chem=1, n_chem=1, p_grow=0.05, p_bond=0.2, p_break=0.01, f_lip=0.3, c_N=0.1) \
        if chem else {}
    ps = [params(L=24, seed=6, rho=rho, **kv), params(L=20, seed=7, rho=rho, **kv)]
    ns = [p.n_beads() for p in ps]
    a, b = ob.Engine(ps, n_beads=ns), ob.Engine(ps, n_beads=ns)
    for e in (a, b):
        for r in range(2):
            e.load_soup(r)
        e.prime()
        e.set_tuning(force_kernel=0, tile_w=14, tile_h=14, tile_threads=256)
    ring = torch.zeros((8, 16), dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    a.stats_ring(1, ring)
    a.set_graph_steps(2)
    b.set_graph_steps(1)
    for _ in range(3):
        a.step(2)
        rows = {int(r[6]): r.copy() for r in ring}
        for _ in range(2):
            b.step(1)
            raw = np.zeros(16, np.uint64)
            b.stats_async(1, raw)
            b.sync()
            got = rows[b.step_no].copy()
            got[6] = 0
            assert np.array_equal(got, raw)
    a.stats_ring(1, None)


def test_events_async_equal_get_events(cuda_ok):
    """events read without a wait (dpd_events_async into pinned memory) are the
    events dpd_get_events returns for a twin run, every 5 steps (as sets: the
    order in which the device appends them may differ); a buffer too small
    keeps some of them and reports the full count"""
    import torch
    p = params(L=24, seed=11, noise="philox", chem=1, n_chem=1, p_grow=0.05, p_bond=0.2, p_break=0.01, f_lip=0.3,
               c_N=0.1)
    a, b = ob.Engine(p), ob.Engine(p)
    for e in (a, b):
        e.load_soup(0)
        e.prime()
    cap = 4096
    buf = torch.empty(cap * ob.Engine.EVENT_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True).numpy()
    buf = buf.view(ob.Engine.EVENT_DTYPE)
    cnt = torch.zeros(1, dtype=torch.int32, pin_memory=True).numpy()
    total = 0
    for _ in range(4):
        a.step(5)
        want = a.events()
        b.step_async(5)
        b.events_async(buf, cnt)
        b.sync()
        assert int(cnt[0]) == len(want)
        assert sorted(ob.Engine.event_tuples(buf, cnt[0])) == sorted(want)
        total += len(want)
    assert total > 0
    a.step(5)
    want = a.events()
    assert len(want) > 2
    b.step(5)
    b.events_async(buf[:2], cnt)
    b.sync()
    got = ob.Engine.event_tuples(buf[:2], cnt[0])
    assert int(cnt[0]) == len(want) and len(got) == 2 and set(got) <= set(want)
    with pytest.raises(ob.DpdError, match="pinned"):
        b.events_async(np.zeros(8, ob.Engine.EVENT_DTYPE), cnt)
