"""dpd_sort_cells_noalloc, the cell sort for callers that cannot allocate
device memory (code inside another framework's operator hook, where a
cudaMalloc and its device-wide synchronisation are not allowed).

Its scratch is one fixed device array of the library, shared by every call, so
the tests make calls in a row of different sizes (a later call must not see an
earlier one's leftovers) and check each against the handle API's sort
(dpd_build_cells), or against numpy's stable sort by cell, bit for bit, as the
other sort tests do.  Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

import oercel_b200 as ob
from gpu_util import params

pytestmark = pytest.mark.gpu

MAX_BEADS = 1048576
MAX_CELLS = 524288


def handle_sort(p, s):
    e = ob.Engine(p)
    e.set_state(0, s["x"], s["y"], s["vx"], s["vy"], s["type"], None, s["prev"], s["next"])
    e.build_cells()
    return e.cells(), e.state()["gid"].astype(np.int32)


def numpy_sort(L, x, y):
    """The stable cell sort the entry point documents: floor(float32(L)) cells
    per side, column-major, the index product in FP64, positions outside the
    box clamped into the edge cells; ties in input order."""
    Lf = np.float64(np.float32(L))
    nc = int(np.floor(Lf))
    ics = nc / Lf
    cx = np.clip((x.astype(np.float64) * ics).astype(np.int64), 0, nc - 1)
    cy = np.clip((y.astype(np.float64) * ics).astype(np.int64), 0, nc - 1)
    key = cx * nc + cy
    order = np.argsort(key, kind="stable").astype(np.int32)
    cs = np.concatenate([[0], np.cumsum(np.bincount(key, minlength=nc * nc))]).astype(np.int32)
    return cs, order


def noalloc_call(torch, L, x, y, n=None, ncs=None):
    lib = ob.load()
    n = len(x) if n is None else n
    nc = int(np.floor(np.float32(L)))
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda()
    cs = torch.full((ncs or nc * nc + 1,), -7, dtype=torch.int32, device="cuda")
    order = torch.full((len(x),), -7, dtype=torch.int32, device="cuda")
    rc = lib.dpd_sort_cells_noalloc(dx.data_ptr(), dy.data_ptr(), n, float(L), cs.data_ptr(),
                                    order.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, cs.cpu().numpy(), order.cpu().numpy()


def noalloc_sort(torch, L, x, y):
    rc, cs, order = noalloc_call(torch, L, x, y)
    assert rc == 0
    return cs, order


def test_noalloc_sort_matches_handle_sort_twice(cuda_ok):
    import torch
    for L, seed in ((100.0, 3), (32.0, 4)):  # larger first: the second call reuses a dirtier array
        p = params(L=L, seed=seed)
        s = ob.soup_for(p)
        want_cs, want_order = handle_sort(p, s)
        got_cs, got_order = noalloc_sort(torch, L, s["x"], s["y"])
        assert np.array_equal(got_cs, want_cs)
        assert np.array_equal(got_order, want_order)


def crowded_positions(rng, L, sizes, n_rest):
    """Beads piled into single cells (one pile per size, in columns x < 20)
    plus a uniform rest in the columns x >= 20, in shuffled input order so that
    the placement atomics scramble every cell."""
    xs, ys = [rng.uniform(20, L, n_rest)], [rng.uniform(0, L, n_rest)]
    for k, m in enumerate(sizes):
        cx, cy = 3 + 2 * k, 5 + k
        xs.append(cx + rng.uniform(0.01, 0.99, m))
        ys.append(cy + rng.uniform(0.01, 0.99, m))
    x = np.concatenate(xs).astype(np.float32)
    y = np.concatenate(ys).astype(np.float32)
    perm = rng.permutation(len(x))
    return x[perm], y[perm]


def test_noalloc_crowded_cells_in_stable_order(cuda_ok):
    """Cells far above the handful of beads a cell normally holds: each size
    path of the crowded-cell sort, at and around its limits (16 beads by one
    thread, up to 4096 in shared memory, more by compaction), then every bead
    in one cell, as zero-initialised positions give."""
    import torch
    rng = np.random.default_rng(11)
    L = 40.0
    x, y = crowded_positions(rng, L, (16, 17, 300, 4096, 4097, 9000), 3000)
    got_cs, got_order = noalloc_sort(torch, L, x, y)
    want_cs, want_order = numpy_sort(L, x, y)
    sizes = np.diff(want_cs)
    for m in (16, 17, 300, 4096, 4097, 9000):
        assert m in sizes
    assert np.array_equal(got_cs, want_cs)
    assert np.array_equal(got_order, want_order)
    z = np.zeros(200000, dtype=np.float32)
    got_cs, got_order = noalloc_sort(torch, 32.0, z, z)
    assert got_cs[0] == 0 and np.all(got_cs[1:] == len(z))
    assert np.array_equal(got_order, np.arange(len(z), dtype=np.int32))


def test_noalloc_sort_at_its_limits(cuda_ok):
    """n = DPD_NOALLOC_MAX_BEADS on the largest square grid under
    DPD_NOALLOC_MAX_CELLS (724 x 724): every scan block and block total in use."""
    import torch
    L = 724.5
    nc = int(np.floor(np.float32(L)))
    assert nc * nc <= MAX_CELLS < (nc + 1) ** 2
    rng = np.random.default_rng(12)
    x = rng.uniform(0, L, MAX_BEADS).astype(np.float32)
    y = rng.uniform(0, L, MAX_BEADS).astype(np.float32)
    got_cs, got_order = noalloc_sort(torch, L, x, y)
    want_cs, want_order = numpy_sort(L, x, y)
    assert np.array_equal(got_cs, want_cs)
    assert np.array_equal(got_order, want_order)
    # a smaller call right after: the full-size leftovers must not leak in
    xs, ys = x[:5000], y[:5000]
    got_cs, got_order = noalloc_sort(torch, 64.0, xs, ys)
    want_cs, want_order = numpy_sort(64.0, xs, ys)
    assert np.array_equal(got_cs, want_cs) and np.array_equal(got_order, want_order)


def test_noalloc_sort_refuses_oversize(cuda_ok):
    import torch
    lib = ob.load()
    x = torch.zeros(16, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = lib.dpd_sort_cells_noalloc(x.data_ptr(), x.data_ptr(), 16, 1000.0, out.data_ptr(), out.data_ptr(), None)
    assert rc == -1  # 1000^2 cells is above DPD_NOALLOC_MAX_CELLS
    # one bead over the limit is refused before any buffer is touched
    rc = lib.dpd_sort_cells_noalloc(x.data_ptr(), x.data_ptr(), MAX_BEADS + 1, 64.0, out.data_ptr(),
                                    out.data_ptr(), None)
    assert rc == -1


def test_noalloc_sort_refuses_a_box_side_that_fp32_rounds_up(cuda_ok):
    """31.9999999 rounds to 32.0f: the grid would be 32 x 32 while floor(L) is
    31, so cstart's size would be ambiguous.  The call refuses it and leaves
    the output alone; 32.0 itself is accepted."""
    import torch
    x = np.full(64, 0.5, dtype=np.float32)
    rc, cs, order = noalloc_call(torch, 31.9999999, x, x, ncs=31 * 31 + 1)
    assert rc == -1
    assert np.all(cs == -7) and np.all(order == -7)
    rc, cs, order = noalloc_call(torch, 32.0, x, x)
    assert rc == 0 and cs[-1] == 64
