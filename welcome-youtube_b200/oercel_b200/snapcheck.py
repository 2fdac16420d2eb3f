"""GPU drop-in for the reference's snapshot checks (cel/engine/tests/snapcheck.py):
`rdf SNAPFILE... [type]` and `tclust SNAPFILE...` computed by the engine's
analysis kernels (dpd_pair_hist, dpd_type_clusters) and printed as the
reference prints them (snapcheck.py:86-144).

    python -m oercel_b200.snapcheck rdf snap_0000001000.bin [snap_...bin ...] [type]
    python -m oercel_b200.snapcheck tclust snap_0000001000.bin [...]
"""
from __future__ import annotations

import sys

import numpy as np

from .cli import read_snapshot
from .engine import Engine
from .params import Params

RMAX, NBIN = 3.0, 30


def engine_for(snap) -> Engine:
    """an engine holding the snapshot's beads, sorted into cells"""
    n = snap["N"]
    e = Engine(Params(L=snap["L"], chem=0), n_beads=n)
    z = np.zeros(n, np.float32)
    e.set_state(0, snap["x"], snap["y"], z, z, snap["type"])
    e.build_cells()
    return e


def rdf(paths, typ=None, out=sys.stdout):
    """g(r) of all beads (or of type typ) averaged over the snapshots"""
    edges = np.linspace(0.0, RMAX, NBIN + 1)
    shell = np.pi * (edges[1:] ** 2 - edges[:-1] ** 2)
    gs = []
    for p in paths:
        s = read_snapshot(p)
        e = engine_for(s)
        t = -1 if typ is None else int(typ)
        h = e.pair_hist(0, t, t, RMAX, NBIN)
        e.close()
        n = s["N"] if typ is None else int((s["type"] == int(typ)).sum())
        gs.append(2 * h / (n * (n / s["L"] ** 2) * shell))
    g = np.mean(gs, axis=0)
    rc = 0.5 * (edges[1:] + edges[:-1])
    print(f"g(r) averaged over {len(paths)} snapshot(s)", file=out)
    for r_, g_ in zip(rc, g):
        print(f"{r_:.3f} {g_:.4f} " + "#" * int(40 * g_ / max(g.max(), 1e-9)), file=out)
    return rc, g


def tclust(path, rcut=1.0, out=sys.stdout):
    """tail-bead clusters within rcut and the T-neighbour fraction within 1.0"""
    s = read_snapshot(path)
    e = engine_for(s)
    c = e.type_clusters(0, 2, rcut)
    e.close()
    print(f"step={s['step']} nT={c['n']} clusters={c['clusters']} largest={c['largest']} mean size "
          f"(bead-weighted)={c['sum_sq'] / max(c['n'], 1):.1f}  T-neighbour fraction={c['fraction']:.3f}", file=out)
    return c


def main(argv=None):
    argv = sys.argv if argv is None else argv
    if len(argv) < 3 or argv[1] not in ("rdf", "tclust"):
        sys.stderr.write(__doc__)
        return 2
    if argv[1] == "rdf":
        paths = [a for a in argv[2:] if a.endswith(".bin")]
        rest = [a for a in argv[2:] if not a.endswith(".bin")]
        rdf(paths, rest[0] if rest else None)
    else:
        for p in argv[2:]:
            tclust(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
