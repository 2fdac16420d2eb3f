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


def aggregates(x, y, types, bonds, L, r_tail=1.0, min_lipids=12):
    """Molecules and membrane aggregates: the first stages of the reference's
    cell detection (cel/tools/cells.py: lipid_molecules 68-86, detect 345-366,
    summary 605-608).  Molecules are the components of the bonds between lipid
    beads (H = 1, T = 2); aggregates join molecules whose T beads lie within
    r_tail.  Returns the summary counts and, per bead, the smallest bead index
    of its aggregate (-1 for other beads)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    from scipy.spatial import cKDTree

    types = np.asarray(types)
    n = len(types)
    lipid = (types == 1) | (types == 2)
    bonds = np.asarray(bonds, np.int64).reshape(-1, 2)
    bonds = bonds[lipid[bonds[:, 0]] & lipid[bonds[:, 1]]] if len(bonds) else bonds
    tails = np.nonzero(types == 2)[0]
    contacts = np.zeros((0, 2), np.int64)
    if len(tails) > 1:
        pts = np.stack([np.asarray(x, np.float64)[tails], np.asarray(y, np.float64)[tails]], axis=1) % L
        pr = cKDTree(pts, boxsize=L).query_pairs(r_tail, output_type="ndarray")
        contacts = tails[pr] if len(pr) else contacts
    # molecules: components of the bond graph over the lipid beads
    mol_graph = coo_matrix((np.ones(len(bonds)), (bonds[:, 0], bonds[:, 1])), shape=(n, n))
    _, mol = connected_components(mol_graph, directed=False)
    mol_ids, mol = np.unique(np.where(lipid, mol, -1), return_inverse=True)
    mol = mol - (1 if mol_ids[0] == -1 else 0)
    mol[~lipid] = -1
    nmol = int(mol.max()) + 1 if lipid.any() else 0
    # aggregates: components of the molecules joined by tail contacts
    if nmol:
        e = mol[contacts] if len(contacts) else np.zeros((0, 2), np.int64)
        g = coo_matrix((np.ones(len(e)), (e[:, 0], e[:, 1])), shape=(nmol, nmol))
        nagg, agg_of_mol = connected_components(g, directed=False)
        size = np.bincount(agg_of_mol, minlength=nagg)
    else:
        nagg, agg_of_mol, size = 0, np.zeros(0, np.int64), np.zeros(0, np.int64)
    label = np.full(n, -1, np.int64)
    if nmol:
        agg = agg_of_mol[mol[lipid]]
        first = np.full(nagg, n, np.int64)
        np.minimum.at(first, agg, np.nonzero(lipid)[0])
        label[lipid] = first[agg]
    return dict(n_molecules=nmol, n_aggregates=int(nagg), n_membranes=int((size >= min_lipids).sum()),
                lipids_in_small_aggregates=int(size[size < min_lipids].sum()),
                largest_aggregate=int(size.max()) if nmol else 0, labels=label)


def rdf_counts(x, y, types, L, t=None, rmax=3.0, nbin=30):
    """Pair-distance counts of the reference's `snapcheck.py rdf`
    (cel/engine/tests/snapcheck.py:86-107): the beads (of type t, or all),
    positions in FP64 modulo L, the pairs within rmax of each other (periodic,
    distance <= rmax), their minimum-image distances binned over [0, rmax]
    into nbin bins.  Returns the counts and the number of beads."""
    from scipy.spatial import cKDTree

    pts = np.stack([np.asarray(x, np.float64), np.asarray(y, np.float64)], axis=1) % L
    if t is not None:
        pts = pts[np.asarray(types) == int(t)]
    pairs = cKDTree(pts, boxsize=L).query_pairs(rmax, output_type="ndarray")
    d = pts[pairs[:, 0]] - pts[pairs[:, 1]]
    d -= L * np.round(d / L)
    r = np.hypot(d[:, 0], d[:, 1])
    counts, _ = np.histogram(r, bins=nbin, range=(0.0, rmax))
    return counts, len(pts)


def rdf_lines(counts, n, L, rmax=3.0, nbin=30):
    """g(r) from the counts, printed as the reference tool prints it"""
    edges = np.linspace(0.0, rmax, nbin + 1)
    g = 2 * counts / (n * (n / L**2) * (np.pi * (edges[1:] ** 2 - edges[:-1] ** 2)))
    rc = 0.5 * (edges[1:] + edges[:-1])
    return [f"{r_:.3f} {g_:.4f} " + "#" * int(40 * g_ / max(g.max(), 1e-9)) for r_, g_ in zip(rc, g)]
