"""Cluster analysis on the GPU (dpd_type_clusters) against the oracle's
restatement of the reference's `snapcheck.py tclust` (oracle/analysis.py,
pinned to the tool's own output): on the reference snapshots of
tests/golden/tclust.npz and on states the engine evolved, every count exact
(beads, clusters, largest, sum of squared sizes, neighbour counts)."""
import numpy as np
import pytest

import analysis
import oercel_b200 as ob
from conftest import golden
from gpu_util import params
from oercel_b200 import cli

pytestmark = pytest.mark.gpu
KEYS = ("n", "clusters", "largest", "sum_sq", "nb_all", "nb_same")


def snapshots():
    g = golden("tclust.npz")
    k = 0
    while f"c{k}_snap" in g:
        yield bytes(g[f"c{k}_snap"])
        k += 1


@pytest.mark.parametrize("k, snap", list(enumerate(snapshots())))
def test_clusters_of_reference_snapshots(cuda_ok, tmp_path, k, snap):
    p = tmp_path / "s.bin"
    p.write_bytes(snap)
    s = cli.read_snapshot(str(p))
    n = s["N"]
    e = ob.Engine(ob.Params(L=s["L"], chem=0), n_beads=n)
    z = np.zeros(n, np.float32)
    e.set_state(0, s["x"], s["y"], z, z, s["type"])
    e.build_cells()
    got = e.type_clusters(0, 2, 1.0)
    ref = analysis.type_clusters(s["x"], s["y"], s["type"], s["L"])
    assert {k_: got[k_] for k_ in KEYS} == ref


@pytest.mark.parametrize("rcut", [1.0, 0.8])
def test_clusters_of_an_evolved_box(cuda_ok, rcut):
    """a 64 x 64 lipid soup after 300 steps (tails aggregating)"""
    p = params(L=64, seed=21, chem=0, noise="philox", a_W_T=90)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(300)
    st = e.state()
    got = e.type_clusters(0, 2, rcut)
    ref = analysis.type_clusters(st["x"], st["y"], st["type"], float(np.float32(p.L)), 2, rcut)
    assert {k_: got[k_] for k_ in KEYS} == ref
    assert got["n"] == int((st["type"] == 2).sum()) and got["clusters"] < got["n"]
