"""Cell detection on the GPU (oercel_b200.cells.detect, dpd_cells_detect)
against the reference's cells.detect (cel/tools/cells.py:331-611).

tests/golden/cells.npz holds the reference's every output on hand-built
snapshots (tests/golden/cell_scenes.py): vesicles free, across the box edge
and on the corner, a nested pair, a dry and an open vesicle, micelles, free
lipids; a membrane network that wraps the box and encloses lumens (one across
the edge) with a vesicle fused onto it; a 2 x 2 tiling; and, under other
configurations, a pixel size that is not a power of two (h = 0.3), another
stamp radius, thresholds and padding; and the edge cases: water only,
micelles only, a box under three contact cells wide, a lumen too small to
count, no beads at all; and four snapshots that the reference executable wrote
after 20,000 and 30,000 steps of membrane-forming runs (one membrane wraps the
box with eleven holes).  The GPU must give
the same summary, membrane list, label grid, per-bead maps and cells; every
cell field equal after the reference's rounding, except the centroid (FP64
sums in another order: 1e-9) and the shape fields computed through an
eigen-decomposition and a hull (one unit in the last rounded digit).

At larger boxes, where the reference takes minutes, the property the
reference's own self-test checks (cel/tools/selftest.py:172-182): a box tiled
k x k has k^2 times the cells, with the same areas.
"""
import json
import os
import sys

import numpy as np
import pytest

import oercel_b200 as ob
from conftest import GOLDEN, golden

sys.path.insert(0, GOLDEN)
import cell_scenes as cs  # noqa: E402
from oercel_b200 import cells, cli  # noqa: E402

pytestmark = pytest.mark.gpu
EXACT = ("id", "area", "r_eq", "n_lipids", "n_Ka", "n_Kb", "n_N", "n_W", "n_Z", "agg", "agg_lumens", "agg_lipids",
         "inner_heads", "outer_heads", "inner_frac", "wraps_membrane", "exposure", "wall")


def cases():
    g = golden("cells.npz")
    k = 0
    while f"c{k}_snap" in g.files:
        yield k
        k += 1


def js(g, key):
    return json.loads(bytes(g[key]).decode())


def same_cells(got, ref):
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        assert list(a) == list(b)
        for k in EXACT:
            assert a[k] == b[k], (k, a[k], b[k])
        assert abs(a["x"] - b["x"]) < 1e-9 and abs(a["y"] - b["y"]) < 1e-9
        for k, tol in (("aspect", 1.5e-3), ("solidity", 1.5e-3), ("extent", 1.5e-2)):
            assert abs(a[k] - b[k]) < tol, (k, a[k], b[k])


@pytest.mark.parametrize("k", list(cases()))
def test_detect_matches_the_reference(cuda_ok, tmp_path, k):
    g = golden("cells.npz")
    p = tmp_path / "snap.bin"
    p.write_bytes(bytes(g[f"c{k}_snap"]))
    r = cells.detect(cells.read_snapshot(str(p)), js(g, f"c{k}_cfg"))
    assert r["ng"] == int(g[f"c{k}_ng"]) and r["h"] == float(g[f"c{k}_h"])
    assert r["summary"] == js(g, f"c{k}_summary")
    assert r["aggregates"] == js(g, f"c{k}_aggregates")
    for key in ("mol", "bead_agg", "bead_cell"):
        assert np.array_equal(r[key], g[f"c{k}_{key}"]), key
    assert r["label"].dtype == g[f"c{k}_label"].dtype
    assert np.array_equal(r["label"], g[f"c{k}_label"])
    same_cells(r["cells"], js(g, f"c{k}_cells"))


@pytest.mark.parametrize("k", [4, 8])
def test_tiled_box_has_k2_times_the_cells(cuda_ok, k):
    sc = cs.vesicles(1)
    x, y, t, b = sc.arrays()
    base = cells.detect(cells.Snapshot(0, 0.0, sc.L, x.astype(np.float64), y.astype(np.float64), t, b))
    L, X, Y, T, B = cs.tile(sc.L, x, y, t, b, k)
    big = cells.detect(cells.Snapshot(0, 0.0, L, X, Y, T, B))
    assert len(base["cells"]) > 0
    assert len(big["cells"]) == k * k * len(base["cells"])
    assert sorted(c["area"] for c in big["cells"]) == sorted([c["area"] for c in base["cells"]] * (k * k))
    assert big["summary"]["n_membranes"] == k * k * base["summary"]["n_membranes"]
    assert big["label"].shape == (base["ng"] * k, base["ng"] * k)


LIPIDS = {"pi": dict(lip_arch="pi", lip_nT=2, lip_tie=1, f_lip=0.35, k_angle=15, a_W_T=200, seed=22),
          "linear": dict(lip_arch="linear", lip_nH=1, lip_nT=3, f_lip=0.3, k_angle=10, a_W_T=100, seed=21)}


@pytest.mark.parametrize("arch", list(LIPIDS))
def test_engine_detect_cells_equals_its_snapshot_file(cuda_ok, tmp_path, arch):
    """Engine.detect_cells on a box of lipids (tied pi: bonds from the template;
    linear: from the chain links) after 3000 steps gives what detect gives on the
    snapshot file the drop-in executable writes for it"""
    p = ob.Params(L=48, dt=0.03, gamma=4.5, warmup=200, f_Ka=0.0, f_Kb=0.0, c_N=0.05, chem=0, **LIPIDS[arch])
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(3000)
    got = e.detect_cells()
    path = str(tmp_path / "snap.bin")
    cli.write_snapshot(path, e.state(0), e.step_no, 0.0, float(p.L), p.template() if arch != "linear" else None)
    ref = cells.detect(cells.read_snapshot(path))
    assert got["summary"] == ref["summary"] and got["summary"]["n_membranes"] > 0
    assert got["aggregates"] == ref["aggregates"]
    for key in ("label", "bead_cell", "mol", "bead_agg"):
        assert np.array_equal(got[key], ref[key]), key
    assert got["cells"] == ref["cells"]
