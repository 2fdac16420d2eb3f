"""dpd_sort_cells_noalloc, the cell sort for callers that cannot allocate
device memory (code inside another framework's operator hook, where a
cudaMalloc and its device-wide synchronisation are not allowed).

Its scratch is one fixed device array of the library, shared by every call, so
the test makes two calls in a row of different sizes (the second must not see
the first one's leftovers) and checks each against the handle API's sort
(dpd_build_cells), bit for bit, as the other sort tests do.  Kept in its own
file, collected last."""
import ctypes as C

import numpy as np
import pytest

import oercel_b200 as ob
from gpu_util import params

pytestmark = pytest.mark.gpu


def handle_sort(p, s):
    e = ob.Engine(p)
    e.set_state(0, s["x"], s["y"], s["vx"], s["vy"], s["type"], None, s["prev"], s["next"])
    e.build_cells()
    return e.cells(), e.state()["gid"].astype(np.int32)


def noalloc_sort(torch, L, x, y):
    lib = ob.load()
    nc = int(np.floor(np.float32(L)))
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y).cuda()
    cs = torch.full((nc * nc + 1,), -7, dtype=torch.int32, device="cuda")
    order = torch.full((len(x),), -7, dtype=torch.int32, device="cuda")
    rc = lib.dpd_sort_cells_noalloc(dx.data_ptr(), dy.data_ptr(), len(x), float(L), cs.data_ptr(),
                                    order.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    return cs.cpu().numpy(), order.cpu().numpy()


def test_noalloc_sort_matches_handle_sort_twice(cuda_ok):
    import torch
    for L, seed in ((100.0, 3), (32.0, 4)):  # larger first: the second call reuses a dirtier array
        p = params(L=L, seed=seed)
        s = ob.soup_for(p)
        want_cs, want_order = handle_sort(p, s)
        got_cs, got_order = noalloc_sort(torch, L, s["x"], s["y"])
        assert np.array_equal(got_cs, want_cs)
        assert np.array_equal(got_order, want_order)


def test_noalloc_sort_refuses_oversize(cuda_ok):
    import torch
    lib = ob.load()
    x = torch.zeros(16, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = lib.dpd_sort_cells_noalloc(x.data_ptr(), x.data_ptr(), 16, 1000.0, out.data_ptr(), out.data_ptr(), None)
    assert rc == -1  # 1000^2 cells is above DPD_NOALLOC_MAX_CELLS
