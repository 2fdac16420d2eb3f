"""CPU restatement of the reference's snapshot analysis of tail-bead clusters
(TEST INFRASTRUCTURE ONLY: the checker of dpd_type_clusters, never part of
the product).

Follows `cmd_tclust` of cel/engine/tests/snapcheck.py:122-144: beads of one
type within rcut of each other (periodic box, distances <= rcut) form
clusters, the connected components of that contact graph; the neighbour
fraction counts, over the type's beads, the beads within 1.0 of the same
type against those of any type (self excluded).  Positions are the FP32
snapshot values taken in FP64 modulo L, as the reference reads them.  Pinned
against the reference tool's own output on reference snapshots
(tests/golden/tclust.npz, made by tests/golden/make_golden.py).
"""
import numpy as np


def type_clusters(x, y, types, L, t=2, rcut=1.0):
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree

    everyone = np.stack([np.asarray(x, np.float64), np.asarray(y, np.float64)], axis=1) % L
    mine = everyone[np.asarray(types) == t]
    n = len(mine)
    tree = cKDTree(mine, boxsize=L)
    pairs = tree.query_pairs(rcut, output_type="ndarray")
    graph = coo_matrix((np.ones(len(pairs)), (pairs[:, 0], pairs[:, 1])), shape=(n, n))
    nclust, label = connected_components(graph, directed=False)
    sizes = np.bincount(label, minlength=1) if n else np.zeros(0, np.int64)
    near_all = cKDTree(everyone, boxsize=L).query_ball_point(mine, 1.0, return_length=True) - 1
    near_same = tree.query_ball_point(mine, 1.0, return_length=True) - 1
    return dict(n=n, clusters=int(nclust) if n else 0, largest=int(sizes.max()) if n else 0,
                sum_sq=int((sizes.astype(np.int64) ** 2).sum()), nb_all=int(near_all.sum()),
                nb_same=int(near_same.sum()))
