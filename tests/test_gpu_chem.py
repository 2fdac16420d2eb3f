"""The chemistry pass on the GPU against the oracle's serial restatement
(bit-exact types, links and events) and the chain invariants it must keep.
Parity of these rules is unpinned by the reference, which has no such reactions;
the oracle is the serial statement of the rules in oracle/dpd_oracle.c."""
import numpy as np
import pytest

import oracle as O
import oercel_b200 as ob
from gpu_util import engine_with, links_by_gid, oracle_params, oracle_state, params

pytestmark = pytest.mark.gpu

RATES = dict(p_grow=0.3, p_break=0.2, p_bond=0.5)


def chem_engine(L=16, seed=3, max_chain=12, **rates):
    r = dict(RATES)
    r.update(rates)
    p = params(L=L, seed=seed, noise="philox", chem=1, n_chem=1, c_N=0.2, f_lip=0.3, max_chain=max_chain, **r)
    s = ob.soup_for(p)
    prev, nxt = s["prev"].copy(), s["next"].copy()
    # dissolve every third lipid into free H and free T beads
    for h in np.nonzero(s["type"] == 1)[0][::3]:
        c = h
        while c >= 0:
            n = nxt[c]
            prev[c] = nxt[c] = -1
            c = n
    e = engine_with(p, s["x"], s["y"], s["vx"], s["vy"], s["type"], prev, nxt)
    e.build_cells()
    return p, e


def oracle_chem(p):
    return O.chem(p_break=p.p_break, p_grow=p.p_grow, p_bond=p.p_bond, r_grow=p.r_grow, r_bond=p.r_bond,
                  n_t_min=p.n_t_min, max_chain=p.max_chain)


def check_chains(s, max_chain):
    """links are mutual, chains are linear and acyclic, H only at a chain head,
    no chain longer than max_chain"""
    prev, nxt, ty = s["prev"], s["next"], s["type"]
    n = len(prev)
    for d in range(n):
        if nxt[d] >= 0:
            assert prev[nxt[d]] == d
        if prev[d] >= 0:
            assert nxt[prev[d]] == d
            assert ty[d] != 1, "H bead in the middle of a chain"
    for h in np.nonzero((prev < 0) & (nxt >= 0))[0]:
        c, k = h, 0
        while c >= 0:
            c = nxt[c]
            k += 1
            assert k <= max_chain
    assert np.all(ty[(prev >= 0) | (nxt >= 0)] != 0) and np.all(ty[(prev >= 0) | (nxt >= 0)] != 3)


@pytest.mark.parametrize("seed", [3, 11])
def test_chemistry_matches_oracle(cuda_ok, seed):
    p, e = chem_engine(seed=seed)
    op, oc = oracle_params(p), oracle_chem(p)
    total, kinds = 0, set()
    for step in range(1, 9):
        s = e.state()
        st = oracle_state(s)
        n, ev = O.chemistry(op, oc, st, e.cells(), step)
        e.chemistry(step)
        t = e.state()
        assert np.array_equal(t["type"], st["type"]), step
        assert np.array_equal(t["prev"], st["prev"]) and np.array_equal(t["next"], st["next"]), step
        got = sorted((k, g, pg, x, y) for (_, k, g, pg, x, y, _) in e.events())
        want = sorted((k, g, pg, x, y) for (_, k, g, pg, x, y) in ev)
        assert got == want, step
        total += n
        kinds |= {k for (k, *_) in want}
        check_chains(t, p.max_chain)
    assert total > 50 and kinds == {0, 1, 2}


def test_chain_cap_holds(cuda_ok):
    p, e = chem_engine(seed=5, max_chain=4, p_grow=0.9)
    for step in range(1, 15):
        e.chemistry(step)
    e.events()
    check_chains(e.state(), 4)


def test_decisions_do_not_depend_on_slot_order(cuda_ok):
    """the same beads in another slot order react identically (keyed by gid)"""
    p, e = chem_engine(seed=7)
    s = e.state()
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(s["x"]))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    prev = np.where(s["prev"][perm] >= 0, inv[np.maximum(s["prev"][perm], 0)], -1).astype(np.int32)
    nxt = np.where(s["next"][perm] >= 0, inv[np.maximum(s["next"][perm], 0)], -1).astype(np.int32)
    e2 = engine_with(p, s["x"][perm], s["y"][perm], s["vhx"][perm], s["vhy"][perm], s["type"][perm], prev, nxt,
                     gid=s["gid"][perm])
    e2.build_cells()
    e.chemistry(4)
    e2.chemistry(4)
    a, b = e.state(), e2.state()
    pa, na = links_by_gid(a)
    pb, nb = links_by_gid(b)
    assert np.array_equal(pa, pb) and np.array_equal(na, nb)
    ta, tb = np.empty_like(a["type"]), np.empty_like(b["type"])
    ta[a["gid"]] = a["type"]
    tb[b["gid"]] = b["type"]
    assert np.array_equal(ta, tb)


def test_step_with_chemistry_equals_phases(cuda_ok):
    """dpd_step with chemistry due every step equals integrate, sort, chemistry, forces"""
    p = params(L=16, seed=9, noise="philox", chem=1, n_chem=1, c_N=0.2, f_lip=0.3, **RATES)
    a = ob.Engine(p)
    a.load_soup(0)
    a.prime()
    a.step(4)
    a.events()
    s = a.state()
    b = engine_with(p, s["x"], s["y"], s["vhx"], s["vhy"], s["type"], s["prev"], s["next"], gid=s["gid"])
    b.set_dynamics(0, s["vhx"], s["vhy"], s["fx"], s["fy"])
    b.resume()
    s0 = a.step_no
    a.step(1)
    b.integrate()
    b.build_cells()
    b.chemistry(s0 + 1)
    b.forces(s0 + 1)
    sa, sb = a.state(), b.state()
    for k in ("x", "y", "vhx", "vhy", "fx", "fy", "type", "gid", "prev", "next"):
        assert np.array_equal(sa[k], sb[k]), k
    ea = sorted(ev[1:6] for ev in a.events())
    eb = sorted(ev[1:6] for ev in b.events())
    assert ea == eb and len(ea) > 0
