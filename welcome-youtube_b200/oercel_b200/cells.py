"""Cell detection in one snapshot on the GPU: the drop-in for the reference's
analysis call `cells.detect(snap, cfg)` (cel/tools/cells.py:331-611).

detect() takes the same snapshot object (any object with L, x, y, type and
bonds, as the reference's ocio.read_snapshot returns it; read_snapshot() here
reads the same file the same way) and the same configuration keys
(DEFAULTS, cells.py:37-56), and returns the same dict: 'cells' (one dict per
cell, the reference's keys and rounding), 'label' (ng x ng lumen grid, int16
below 32767 cells), 'bead_cell', 'h', 'ng', 'aggregates', 'summary', 'mol',
'bead_agg'.  Every stage runs in libdpd.so (dpd_cells_detect); this module
only converts arguments and results.
"""
from __future__ import annotations

import ctypes as C
import math
import struct
from dataclasses import dataclass

import numpy as np

from ._capi import CELL_COLS, DpdCellsCfg, check, load, ptr

DEFAULTS = dict(
    r_tail=1.0,
    h=0.25,
    r_stamp=0.75,
    min_membrane_lipids=12,
    min_lumen_area=16.0,
    min_aqueous_frac=0.30,
    rho=3.0,
    pad=2.5,
    leaflet_in=1.5,
    leaflet_max=6.0,
    min_exposure=0.8,
    wall_extra=4.0,
    inner_frac_range=(0.2, 0.62),
)
INT16_LABELS = 32767


@dataclass
class Snapshot:
    step: int
    time: float
    L: float
    x: np.ndarray       # float64, wrapped into [0, L)
    y: np.ndarray
    type: np.ndarray    # uint8
    bonds: np.ndarray   # int64 (nbonds, 2)
    path: str = ""

    @property
    def n(self):
        return len(self.type)


def _wrap(a, L):
    a = np.mod(a, L)
    a[a >= L] -= L
    return a


def read_snapshot(path) -> Snapshot:
    """a snapshot file (magic OCEL, version 1) with positions widened to FP64
    and wrapped into [0, L), as the reference's tools read it"""
    with open(path, "rb") as f:
        buf = f.read()
    if len(buf) < 40 or buf[:4] != b"OCEL":
        raise ValueError(f"{path}: not a snapshot")
    ver, n, nb = struct.unpack_from("<iii", buf, 4)
    step, time, L = struct.unpack_from("<qdd", buf, 16)
    if ver != 1 or len(buf) != 40 + 9 * n + 8 * nb:
        raise ValueError(f"{path}: unsupported version or size")
    o = 40
    x = np.frombuffer(buf, "<f4", n, o).astype(np.float64)
    o += 4 * n
    y = np.frombuffer(buf, "<f4", n, o).astype(np.float64)
    o += 4 * n
    t = np.frombuffer(buf, "u1", n, o).copy()
    o += n
    b = np.frombuffer(buf, "<i4", 2 * nb, o).reshape(nb, 2).astype(np.int64)
    return Snapshot(step=step, time=time, L=float(L), x=_wrap(x, L), y=_wrap(y, L), type=t, bonds=b, path=str(path))


def _cfg_struct(c: dict) -> DpdCellsCfg:
    s = DpdCellsCfg()
    check(load().dpd_cells_default(C.byref(s)))
    for k in ("r_tail", "h", "r_stamp", "min_lumen_area", "min_aqueous_frac", "rho", "pad", "leaflet_in",
              "leaflet_max", "min_exposure", "wall_extra"):
        setattr(s, k, float(c[k]))
    s.min_membrane_lipids = int(c["min_membrane_lipids"])
    s.inner_frac_lo, s.inner_frac_hi = (float(v) for v in c["inner_frac_range"])
    return s


def _cell_dict(j, r):
    area = float(r[2])
    inner, outer = int(r[12]), int(r[13])
    wall = float(r[19])
    return dict(
        id=j,
        x=float(r[0]), y=float(r[1]),
        area=round(area, 3),
        r_eq=round(float(np.sqrt(area / np.pi)), 3),
        n_lipids=int(r[3]),
        n_Ka=int(r[4]), n_Kb=int(r[5]),
        n_N=int(r[6]), n_W=int(r[7]), n_Z=int(r[8]),
        agg=int(r[9]),
        agg_lumens=int(r[10]),
        agg_lipids=int(r[11]),
        inner_heads=inner, outer_heads=outer,
        inner_frac=round(float(inner / max(inner + outer, 1)), 3),
        aspect=round(float(r[14]), 3), solidity=round(min(float(r[15]), 1.0), 3),
        extent=round(float(r[16]), 2),
        wraps_membrane=bool(r[17]),
        exposure=round(float(r[18]), 3), wall=round(wall, 2) if math.isfinite(wall) else None,
    )


def detect(snap, cfg=None):
    """Detect cells in a snapshot on the GPU; arguments and result as the
    reference's cells.detect"""
    c = dict(DEFAULTS)
    if cfg:
        c.update(cfg)
    lib = load()
    L = float(snap.L)
    x = np.ascontiguousarray(snap.x, np.float64)
    y = np.ascontiguousarray(snap.y, np.float64)
    t = np.ascontiguousarray(snap.type, np.uint8)
    b = np.ascontiguousarray(np.asarray(snap.bonds).reshape(-1, 2), np.int32)
    n = len(t)
    s = _cfg_struct(c)
    h = C.c_void_p()
    check(lib.dpd_cells_detect(C.byref(s), L, n, ptr(x), ptr(y), ptr(t), len(b), ptr(b), C.byref(h)))
    try:
        info = np.zeros(9, np.int64)
        hh = C.c_double()
        check(lib.dpd_cells_info(h, ptr(info), C.byref(hh)))
        ng, ncell, nagg = int(info[6]), int(info[7]), int(info[8])
        rows = np.zeros((ncell, CELL_COLS))
        aggs = np.zeros((nagg, 4), np.int64)
        label = np.empty((ng, ng), np.int16 if ncell < INT16_LABELS else np.int32)
        bead_cell = np.empty(n, np.int32)
        mol = np.empty(n, np.int32)
        bead_agg = np.empty(n, np.int32)
        check(lib.dpd_cells_fetch(h, ptr(rows), ptr(aggs), ptr(label), label.itemsize, ptr(bead_cell), ptr(mol),
                                  ptr(bead_agg)))
    finally:
        lib.dpd_cells_free(h)
    cells = [_cell_dict(j, r) for j, r in enumerate(rows)]
    summary = dict(n_molecules=int(info[0]), n_aggregates=int(info[1]), n_membranes=int(info[2]),
                   lipids_in_small_aggregates=int(info[3]), largest_aggregate=int(info[4]),
                   wrapping_membranes=int(info[5]))
    agg_info = [dict(agg=int(a), n_lipids=int(k), wraps=bool(w), n_holes=int(nh)) for a, k, w, nh in aggs]
    return dict(cells=cells, label=label, bead_cell=bead_cell, h=float(hh.value), ng=ng,
                aggregates=agg_info, summary=summary, mol=mol.astype(np.int64), bead_agg=bead_agg.astype(np.int64))
