"""Replicas of uneven size packed into one set of device arrays advance exactly
as each replica does alone (forces, positions, chemistry: bit-identical)."""
import numpy as np
import pytest

import oercel_b200 as ob
from gpu_util import params

pytestmark = pytest.mark.gpu


def replica_params():
    # uneven boxes, per-replica seeds, perturbed repulsions and chemistry rates
    return [
        params(L=10.0, seed=1, noise="philox"),
        params(L=float(np.float32(np.sqrt(3000 / 4))), seed=2, noise="philox", a_W_T=79.3, a_H_T=47.1),
        params(L=16.0, seed=3, noise="mix13", chem=1, n_chem=1, c_N=0.2, f_lip=0.3, p_grow=0.05, p_bond=0.2,
               p_break=0.01),
        params(L=9.0, seed=4, noise="philox", chem=1, n_chem=2, c_N=0.2, f_lip=0.3, p_grow=0.1, p_bond=0.3,
               p_break=0.02),
    ]


def test_batched_equals_single(cuda_ok):
    ps = replica_params()
    batched = ob.Engine(ps)
    singles = [ob.Engine(p) for p in ps]
    for r, p in enumerate(ps):
        batched.load_soup(r)
        singles[r].load_soup(0)
    batched.prime()
    for s in singles:
        s.prime()
    batched.step(37)
    for s in singles:
        s.step(37)
    ev_b = batched.events()
    for r, s in enumerate(singles):
        a, b = batched.state(r), s.state(0)
        for k in ("x", "y", "vhx", "vhy", "vtx", "vty", "fx", "fy", "type", "gid", "prev", "next"):
            assert np.array_equal(a[k], b[k]), (r, k)
        assert np.array_equal(batched.cells(r), s.cells(0))
        got = sorted(e[:6] for e in ev_b if e[6] == r)
        want = sorted(e[:6] for e in s.events())
        assert got == want, r
        oa, ob_ = batched.observables(r), s.observables(0)
        assert oa["T"] == ob_["T"] and oa["virial"] == ob_["virial"]
