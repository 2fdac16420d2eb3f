"""Analysis on the GPU against the oracle's restatements (oracle/analysis.py,
pinned to the reference tools' own output): tail-bead clusters
(dpd_type_clusters, the reference's `snapcheck.py tclust`) on the reference
snapshots of tests/golden/tclust.npz and on states the engine evolved, every
count exact (beads, clusters, largest, sum of squared sizes, neighbour
counts); molecules and membrane aggregates (dpd_aggregates, the first stages
of the reference's cells.detect) on evolved boxes of linear and pi lipids,
every count and every bead's aggregate exact."""
import os
import subprocess
import sys

import numpy as np
import pytest

import analysis
import oercel_b200 as ob
from conftest import PKG, golden
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


@pytest.mark.parametrize("arch", ["linear", "pi"])
def test_aggregates_of_an_evolved_box(cuda_ok, arch):
    """molecules and membrane aggregates (the first stages of the reference's
    cell detection) on a 32 x 32 lipid box after 1500 steps, against the oracle
    (pinned to the reference's cells.detect): every count and the aggregate
    label of every bead"""
    kv = dict(L=32, seed=23, chem=0, noise="philox", f_lip=0.3, warmup=0)
    if arch == "linear":
        p = params(a_W_T=100, lip_nT=3, k_angle=10, **kv)
    else:
        p = params(lip_arch="pi", lip_nT=2, lip_tie=1, r0_head=0.7, k_bond=300, k_angle=15, a_W_T=150, **kv)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(1500)
    st = e.state()
    got = e.aggregates(0, 1.0, 12, labels=True)
    if arch == "linear":
        g, nx = st["gid"].astype(np.int64), st["next"]
        bonds = np.stack([g[nx >= 0], g[nx[nx >= 0]]], axis=1)
    else:
        bonds = cli.template_bonds(st, p.template())
    n = len(st["x"])
    x, y, t = np.empty(n, np.float32), np.empty(n, np.float32), np.empty(n, np.uint8)
    x[st["gid"]], y[st["gid"]], t[st["gid"]] = st["x"], st["y"], st["type"]
    ref = analysis.aggregates(x, y, t, bonds, float(np.float32(p.L)), 1.0, 12)
    for k in ("n_molecules", "n_aggregates", "n_membranes", "lipids_in_small_aggregates", "largest_aggregate"):
        assert got[k] == ref[k], k
    assert np.array_equal(got["labels"], ref["labels"])
    assert got["n_membranes"] >= 1


@pytest.mark.parametrize("k", range(6))
def test_rdf_counts_of_reference_snapshots(cuda_ok, tmp_path, k):
    """the pair-distance histogram (dpd_pair_hist, all beads and T beads, rmax 3,
    30 bins) equals the oracle's restatement of the reference's `snapcheck.py
    rdf` count for count on the reference snapshots (two with membranes)"""
    g = golden("aggregates.npz")
    p = tmp_path / "s.bin"
    p.write_bytes(bytes(g[f"c{k}_snap"]))
    s = cli.read_snapshot(str(p))
    n = s["N"]
    e = ob.Engine(ob.Params(L=s["L"], chem=0), n_beads=n)
    z = np.zeros(n, np.float32)
    e.set_state(0, s["x"], s["y"], z, z, s["type"])
    e.build_cells()
    for typ in (None, 2):
        got = e.pair_hist(0, -1 if typ is None else typ, -1 if typ is None else typ, 3.0, 30)
        ref, _ = analysis.rdf_counts(s["x"], s["y"], s["type"], s["L"], typ)
        assert np.array_equal(got.astype(np.int64), ref), typ



SNAPCHECK = os.path.join(PKG, "bin", "oercel_b200_snapcheck")


@pytest.mark.parametrize("k", range(6))
def test_snapcheck_drop_in_prints_what_the_reference_tool_prints(cuda_ok, tmp_path, k):
    """`oercel_b200_snapcheck rdf|tclust SNAP` (GPU) prints the reference tool's
    own output (tests/golden/rdf.npz, tclust.npz) byte for byte; g(r) of the
    tail beads too, through the module's rdf(typ=2)"""
    import io
    from oercel_b200 import snapcheck
    g, r = golden("aggregates.npz"), golden("rdf.npz")
    p = tmp_path / "snap.bin"
    p.write_bytes(bytes(g[f"c{k}_snap"]))
    out = subprocess.run([sys.executable, SNAPCHECK, "rdf", str(p)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout == bytes(r[f"c{k}_all"]).decode()
    buf = io.StringIO()
    snapcheck.rdf([str(p)], 2, out=buf)
    assert buf.getvalue() == bytes(r[f"c{k}_T"]).decode()
    t = golden("tclust.npz")
    if f"c{k}_line" in t.files:
        out = subprocess.run([sys.executable, SNAPCHECK, "tclust", str(p)], capture_output=True, text=True,
                             timeout=300)
        assert out.returncode == 0, out.stderr[-2000:]
        assert out.stdout.strip() == bytes(t[f"c{k}_line"]).decode()
