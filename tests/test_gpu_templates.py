"""Branched lipids (pi, y, bola) on the GPU: the template's bonds and angle
terms (k_mol_forces, added by both force kernels' epilogue).

Against the reference: its bonded_forces with the template on states it
evolved (tests/golden/mol_*.npz), within 1e-5 of the largest force (FP32
against FP64), the running max bond within 1e-6, and the net bonded force
exactly zero (fixed point).  Against the oracle (pinned to the same fixtures)
on states the engine evolved itself; and the two force kernels bit for bit.
"""
import numpy as np
import pytest

import oracle as O
import oercel_b200 as ob
from conftest import golden

pytestmark = pytest.mark.gpu
CASES = ["mol_pi_L12_seed31.npz", "mol_y_L12_seed32.npz", "mol_bola_L12_seed33.npz"]


def params_of(g, **over):
    kv = [tuple(line.split(" = ", 1)) for line in bytes(g["ini"]).decode().strip().split("\n")]
    return ob.Params().update(kv + [(k, str(v)) for k, v in over.items()])


def template_of(g):
    return {k[2:]: g[k] for k in g.files if k.startswith("t_")}


@pytest.mark.parametrize("name", CASES)
def test_template_forces_match_reference(cuda_ok, name):
    g = golden(name)
    p = params_of(g)
    n = len(g["x"])
    nxt = g["nxt"].astype(np.int32)
    prev = np.full(n, -1, np.int32)
    prev[nxt[nxt >= 0]] = np.nonzero(nxt >= 0)[0]
    e = ob.Engine(p, n_beads=n)
    z = np.zeros(n, np.float32)
    e.set_state(0, g["x"].astype(np.float32), g["y"].astype(np.float32), z, z, g["type"], g["gid"], prev, nxt)
    fx, fy, mb = e.bond_forces(0)
    scale = np.abs(g["fx"]).max()
    assert np.abs(fx - g["fx"]).max() <= 1e-5 * scale and np.abs(fy - g["fy"]).max() <= 1e-5 * scale
    assert mb == pytest.approx(float(g["maxbond"]), rel=1e-6)
    assert fx.astype(np.float64).sum() == 0.0 and fy.astype(np.float64).sum() == 0.0


@pytest.mark.parametrize("name", CASES)
def test_template_forces_follow_the_oracle_on_evolved_states(cuda_ok, name):
    g = golden(name)
    p = params_of(g, L=16, seed=9, noise="philox")
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(40)
    s = e.state()
    fx, fy, mb = e.bond_forces(0)
    op = O.params(float(np.float32(p.L)), np.full((8, 8), 25.0), k_bond=p.k_bond, r0=p.r0)
    ox, oy, omb = O.mol_forces(op, O.mol(template_of(g)), dict(x=s["x"], y=s["y"], next=s["next"]))
    scale = np.abs(ox).max()
    assert np.abs(fx - ox).max() <= 1e-5 * scale and np.abs(fy - oy).max() <= 1e-5 * scale
    assert mb == pytest.approx(omb, rel=1e-6)


@pytest.mark.parametrize("name", CASES)
def test_force_kernels_agree_with_branched_lipids(cuda_ok, name):
    g = golden(name)
    p = params_of(g, L=16, seed=10, noise="philox")
    runs = []
    for fk in (0, 1):
        e = ob.Engine(p)
        e.set_tuning(force_kernel=fk)
        e.load_soup(0)
        e.prime()
        e.step(25)
        runs.append(e.state())
    for k in ("x", "y", "vhx", "vhy", "fx", "fy", "gid", "next"):
        assert np.array_equal(runs[0][k], runs[1][k]), k
