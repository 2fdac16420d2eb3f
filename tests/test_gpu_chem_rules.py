"""The three lipid-chemistry rules of the 1M-bead workload checked from outside
the oracle.  The reference has none of these reactions, so the device code and
the oracle's serial restatement are written from the same rule text; these
tests derive the expected outcome from the rules alone:

  * rates: over 1000 production steps of an L = 64 box, the events of each rule
    equal p x (the beads eligible for it, counted here in numpy from each
    step's state) within 4 binomial sigma;
  * scenes built by hand with expected outcomes written down: a P with one and
    with two T beads within r_grow, two free H at exactly equal distance from
    a free T (the lower gid wins, as the reference's distance-then-gid
    tie-break, cel/engine/oercel.c:1387-1396), a chain at max_chain, two
    requesters for one H (the lowest gid wins, the GPU port's ordered
    conflict resolution, cel/engine_gpu/oercel_gpu.cu:1746-1757).

Rules: an H-T bond breaks with p_break (drawn by the
H bead); a P with at least n_t_min T beads within r_grow becomes a T bonded to
its nearest growable chain end within r_grow (a lone H, or the tail T of a
chain headed by H shorter than max_chain) with p_grow; a free T bonds to its
nearest free H within r_bond with p_bond."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

import oercel_b200 as ob
from gpu_util import engine_with, params

pytestmark = pytest.mark.gpu

W, H, T, P = 0, 1, 2, 3


def by_gid(s):
    g = s["gid"].astype(np.int64)
    n = len(g)
    out = {}
    for k in ("x", "y"):
        v = np.empty(n, np.float64)
        v[g] = s[k]
        out[k] = v
    t = np.empty(n, np.int64)
    t[g] = s["type"]
    pv = np.full(n, -1, np.int64)
    nx = np.full(n, -1, np.int64)
    pv[g] = np.where(s["prev"] >= 0, g[np.maximum(s["prev"], 0)], -1)
    nx[g] = np.where(s["next"] >= 0, g[np.maximum(s["next"], 0)], -1)
    out["type"], out["prev"], out["next"] = t, pv, nx
    return out


def growable_ends(t, pv, nx, max_chain):
    """gids that a P may attach to: lone H beads, and the tail T of a chain
    headed by H with fewer than max_chain beads"""
    n = len(t)
    ok = np.zeros(n, bool)
    ok |= (t == H) & (pv < 0) & (nx < 0)
    for e in np.nonzero((t == T) & (nx < 0) & (pv >= 0))[0]:
        c, k = e, 1
        while pv[c] >= 0 and k <= max_chain:
            c = pv[c]
            k += 1
        ok[e] = t[c] == H and k < max_chain
    return ok


def test_event_rates_follow_the_rules(cuda_ok):
    rates = dict(p_break=1e-3, p_grow=2e-3, p_bond=1e-2)
    p = params(L=64.0, seed=41, noise="philox", chem=1, n_chem=1, **rates)
    s = ob.soup_for(p)
    prev, nxt = s["prev"].copy(), s["next"].copy()
    for h in np.nonzero(s["type"] == H)[0][::3]:  # every third lipid dissolved into free H and T
        c = h
        while c >= 0:
            n = nxt[c]
            prev[c] = nxt[c] = -1
            c = n
    e = engine_with(p, s["x"], s["y"], s["vx"], s["vy"], s["type"], prev, nxt)
    e.prime()
    L = float(np.float32(p.L))
    before = by_gid(e.state())
    exp = {0: [0.0, 0.0], 1: [0.0, 0.0], 2: [0.0, 0.0]}  # kind -> [mean, variance]
    seen = {0: 0, 1: 0, 2: 0}
    for _ in range(1000):
        e.step(1)
        after = by_gid(e.state())
        ev = e.events()
        t, pv, nx = before["type"].copy(), before["prev"].copy(), before["next"].copy()
        pos = np.c_[after["x"], after["y"]] % L

        def within(sel_from, sel_to, r):  # per bead of sel_from: beads of sel_to within r (none of them itself)
            if len(sel_to) == 0 or len(sel_from) == 0:
                return np.zeros(len(sel_from), np.int64)
            return cKDTree(pos[sel_to], boxsize=L).query_ball_point(pos[sel_from], r, return_length=True)

        # break: every H-T bond of the step's start
        n_ht = int(np.sum((t == H) & (nx >= 0) & (t[np.maximum(nx, 0)] == T)))
        exp[1][0] += rates["p_break"] * n_ht
        exp[1][1] += rates["p_break"] * (1 - rates["p_break"]) * n_ht
        for (_, k, g, pg, *_rest) in ev:
            if k == 1:
                assert t[g] == H and nx[g] == pg and t[pg] == T
                nx[g], pv[pg] = -1, -1
        # growth: P beads with >= n_t_min T within r_grow and a growable end within r_grow
        ends = growable_ends(t, pv, nx, p.max_chain)
        ps = np.nonzero(t == P)[0]
        ok = (within(ps, np.nonzero(t == T)[0], p.r_grow) >= p.n_t_min) & (within(ps, np.nonzero(ends)[0], p.r_grow) > 0)
        n_grow = int(ok.sum())
        exp[0][0] += rates["p_grow"] * n_grow
        exp[0][1] += rates["p_grow"] * (1 - rates["p_grow"]) * n_grow
        for (_, k, g, pg, *_rest) in ev:
            if k == 0:
                assert t[g] == P and ends[pg]
                t[g] = T
                pv[g], nx[pg] = pg, g
        # bonding: free T beads with a free H within r_bond
        free = (pv < 0) & (nx < 0)
        fts = np.nonzero((t == T) & free)[0]
        n_bond = int((within(fts, np.nonzero((t == H) & free)[0], p.r_bond) > 0).sum())
        exp[2][0] += rates["p_bond"] * n_bond
        exp[2][1] += rates["p_bond"] * (1 - rates["p_bond"]) * n_bond
        for (_, k, *_r) in ev:
            seen[k] += 1
        before = after
    for k, name in ((0, "grow"), (1, "break"), (2, "bond")):
        mean, var = exp[k]
        assert seen[k] >= 150, (name, seen[k])
        assert abs(seen[k] - mean) < 4.0 * np.sqrt(var) + 0.02 * mean, (name, seen[k], mean, np.sqrt(var))


def scene_engine(beads, L=8.0, gid=None, **kv):
    """an engine holding exactly these beads: (x, y, type, prev, next) rows
    (links are row indices), gids = row indices unless given"""
    rates = dict(p_break=0.0, p_grow=0.0, p_bond=0.0)
    rates.update(kv)
    p = params(L=L, seed=5, noise="philox", chem=1, n_chem=1, **rates)
    b = np.array(beads, dtype=np.float64)
    n = len(b)
    z = np.zeros(n, np.float32)
    e = engine_with(p, b[:, 0], b[:, 1], z, z, b[:, 2].astype(np.uint8), b[:, 3].astype(np.int32),
                    b[:, 4].astype(np.int32), gid=None if gid is None else np.asarray(gid, np.uint32))
    e.build_cells()
    return e


def links_of(e):
    s = by_gid(e.state())
    return s["type"], s["prev"], s["next"]


def test_growth_needs_two_tails_within_reach(cuda_ok):
    """P at (4, 4) next to a lone H (a growable end) at distance 0.5; with one
    T within r_grow nothing grows, with two it grows onto the H"""
    far = (7.0, 7.0, W, -1, -1)
    one_t = [(4.0, 4.0, P, -1, -1), (4.5, 4.0, H, -1, -1), (4.0, 4.5, T, -1, -1), (4.0, 2.5, T, -1, -1), far]
    e = scene_engine(one_t, p_grow=1.0)
    e.chemistry(1)
    t, pv, nx = links_of(e)
    assert t[0] == P and nx[1] == -1 and e.events() == []
    two_t = [(4.0, 4.0, P, -1, -1), (4.5, 4.0, H, -1, -1), (4.0, 4.5, T, -1, -1), (4.0, 3.25, T, -1, -1), far]
    e = scene_engine(two_t, p_grow=1.0)
    e.chemistry(1)
    t, pv, nx = links_of(e)
    assert t[0] == T and pv[0] == 1 and nx[1] == 0
    assert [(k, g, pg) for (_, k, g, pg, *_r) in e.events()] == [(0, 0, 1)]


def test_equal_distance_goes_to_the_lower_gid(cuda_ok):
    """a free T at (4, 4) and free H beads at (4.25, 4) and (4, 4.25), both 0.25
    away exactly; the H with the lower gid is taken, whichever of the two
    places and slots it has"""
    rows = [(4.0, 4.0, T, -1, -1), (4.25, 4.0, H, -1, -1), (4.0, 4.25, H, -1, -1), (7.0, 7.0, W, -1, -1)]
    for gid in ([0, 1, 2, 3], [0, 2, 1, 3]):
        e = scene_engine(rows, gid=gid, p_bond=1.0)
        e.chemistry(1)
        t, pv, nx = links_of(e)
        assert pv[0] == 1 and nx[1] == 0 and nx[2] == -1
        assert [(k, g, pg) for (_, k, g, pg, *_r) in e.events()] == [(2, 0, 1)]


def chain(x0, y, n_t, gid0):
    """an H followed by n_t T beads along x, 0.5 apart, gids gid0..gid0+n_t"""
    rows = []
    for k in range(n_t + 1):
        rows.append((x0 + 0.5 * k, y, H if k == 0 else T, gid0 + k - 1 if k > 0 else -1,
                     gid0 + k + 1 if k < n_t else -1))
    return rows


def test_no_growth_past_max_chain(cuda_ok):
    """a chain of max_chain beads does not grow; one bead shorter does"""
    for n_beads, grows in ((6, False), (5, True)):
        rows = chain(1.0, 4.0, n_beads - 1, 0)
        tail = rows[-1]
        tx = tail[0]
        ng = len(rows)
        rows += [(tx + 0.4, 4.3, P, -1, -1), (tx + 0.4, 3.6, T, -1, -1), (7.5, 7.5, W, -1, -1)]
        e = scene_engine(rows, L=10.0, p_grow=1.0, max_chain=6)
        e.chemistry(1)
        t, pv, nx = links_of(e)
        assert (t[ng] == T and pv[ng] == ng - 1 and nx[ng - 1] == ng) == grows


def test_two_requesters_for_one_head(cuda_ok):
    """two free T beads whose nearest free H is the same bead: the lower gid
    wins it, the other stays free this step"""
    for near_gid in (1, 2):  # the lower-gid T nearer, then farther
        a, b = (4.2, 4.0), (3.7, 4.0)
        if near_gid == 2:
            a, b = b, a
        rows = [(4.0, 4.0, H, -1, -1), (a[0], a[1], T, -1, -1), (b[0], b[1], T, -1, -1), (7.0, 7.0, W, -1, -1)]
        e = scene_engine(rows, p_bond=1.0)
        e.chemistry(1)
        t, pv, nx = links_of(e)
        assert nx[0] == 1 and pv[1] == 0 and pv[2] == -1 and nx[2] == -1
        assert [(k, g, pg) for (_, k, g, pg, *_r) in e.events()] == [(2, 1, 0)]
