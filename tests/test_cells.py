"""Host side of the GPU cell detection (oercel_b200.cells), no GPU: the
snapshot reader widens and wraps positions as the reference's tools do
(cel/tools/ocio.py), the configuration reaches the C struct, and a raw row of
dpd_cells_fetch becomes the reference's cell dict with its rounding
(cel/tools/cells.py:582-601)."""
import math
import struct

import numpy as np

from conftest import golden
from oercel_b200 import cells


def test_read_snapshot_widens_and_wraps(tmp_path):
    g = golden("cells.npz")
    raw = bytes(g["c0_snap"])
    p = tmp_path / "s.bin"
    p.write_bytes(raw)
    s = cells.read_snapshot(str(p))
    n = struct.unpack_from("<i", raw, 8)[0]
    assert s.n == n and s.L == 56.0 and s.x.dtype == np.float64 and s.bonds.dtype == np.int64
    assert np.array_equal(s.x, np.frombuffer(raw, "<f4", n, 40).astype(np.float64))
    assert np.all((s.x >= 0) & (s.x < s.L)) and np.all((s.y >= 0) & (s.y < s.L))
    # a position at or beyond L is wrapped, as the reference's reader wraps it
    b = bytearray(raw)
    struct.pack_into("<f", b, 40, 56.0)
    struct.pack_into("<f", b, 44, -1.5)
    p.write_bytes(bytes(b))
    s = cells.read_snapshot(str(p))
    assert s.x[0] == 0.0 and s.x[1] == 54.5


def test_configuration_struct():
    s = cells._cfg_struct(dict(cells.DEFAULTS, min_lumen_area=20.0, inner_frac_range=(0.1, 0.7)))
    assert (s.min_lumen_area, s.inner_frac_lo, s.inner_frac_hi, s.min_membrane_lipids) == (20.0, 0.1, 0.7, 12)
    assert (s.r_tail, s.h, s.r_stamp, s.rho, s.pad, s.wall_extra) == (1.0, 0.25, 0.75, 3.0, 2.5, 4.0)


def test_cell_row_to_dict():
    row = np.array([3.25, 7.5, 41.5, 120, 1, 2, 3, 137, 4, 5, 1, 122, 44, 78, 1.01149, 1.0004, 15.56789, 0, 1.0,
                    4.8149999])
    d = cells._cell_dict(2, row)
    assert list(d) == ["id", "x", "y", "area", "r_eq", "n_lipids", "n_Ka", "n_Kb", "n_N", "n_W", "n_Z", "agg",
                       "agg_lumens", "agg_lipids", "inner_heads", "outer_heads", "inner_frac", "aspect", "solidity",
                       "extent", "wraps_membrane", "exposure", "wall"]
    assert d["r_eq"] == round(math.sqrt(41.5 / math.pi), 3) and d["inner_frac"] == round(44 / 122, 3)
    assert d["solidity"] == 1.0 and d["aspect"] == 1.011 and d["extent"] == 15.57 and d["wall"] == 4.81
    row[19] = math.inf
    assert cells._cell_dict(0, row)["wall"] is None


def test_detect_refuses_unwrapped_positions_and_bad_bonds():
    """checked on the host before anything reaches the device"""
    import pytest
    from oercel_b200 import DpdError
    x = np.array([1.0, 2.0, 3.0])
    s = cells.Snapshot(0, 0.0, 8.0, x, np.array([1.0, 8.0, 2.0]), np.array([1, 2, 0], np.uint8),
                       np.array([[0, 1]], np.int64))
    with pytest.raises(DpdError, match="outside"):
        cells.detect(s)
    s.y = np.array([1.0, 2.0, 3.0])
    s.bonds = np.array([[0, 5]], np.int64)
    with pytest.raises(DpdError, match="bond index"):
        cells.detect(s)
