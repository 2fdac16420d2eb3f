"""torch CUDA tensors as the device-memory carrier of the C ABI: the state set
from and read into device tensors (their data_ptr()), and the force VJP with
its cotangents and outputs on the device, give the same bits as the same
calls with numpy host arrays."""
import ctypes as C

import numpy as np
import pytest

import oercel_b200 as ob
from gpu_util import params

pytestmark = pytest.mark.gpu

F32 = ("x", "y", "vhx", "vhy", "vtx", "vty", "fx", "fy")


def read_state_into_tensors(torch, e, n):
    out = {k: torch.full((n,), -1.0, dtype=torch.float32, device="cuda") for k in F32}
    out["type"] = torch.zeros(n, dtype=torch.uint8, device="cuda")
    out["gid"] = torch.zeros(n, dtype=torch.int32, device="cuda")  # uint32 bits
    out["prev"] = torch.zeros(n, dtype=torch.int32, device="cuda")
    out["next"] = torch.zeros(n, dtype=torch.int32, device="cuda")
    args = [out[k].data_ptr() for k in F32 + ("type", "gid", "prev", "next")]
    ob._capi.check(e.lib.dpd_get_state(e.h, 0, *args))
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def test_state_through_cuda_tensors(cuda_ok):
    import torch
    p = params(L=24.0, seed=17, noise="philox", chem=1, n_chem=1, p_grow=0.05, p_bond=0.2, p_break=0.01)
    s = ob.soup_for(p)
    n = len(s["x"])
    host = ob.Engine(p)
    host.set_state(0, s["x"], s["y"], s["vx"], s["vy"], s["type"], None, s["prev"], s["next"])
    dev = ob.Engine(p)
    t = {k: torch.from_numpy(np.ascontiguousarray(s[k])).cuda() for k in ("x", "y", "vx", "vy", "type", "prev", "next")}
    ob._capi.check(dev.lib.dpd_set_state(dev.h, 0, t["x"].data_ptr(), t["y"].data_ptr(), t["vx"].data_ptr(),
                                         t["vy"].data_ptr(), t["type"].data_ptr(), None, t["prev"].data_ptr(),
                                         t["next"].data_ptr()))
    for e in (host, dev):
        e.prime()
        e.step(12)
    a = host.state()
    b = read_state_into_tensors(torch, dev, n)
    for k in F32:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["type"], b["type"])
    assert np.array_equal(a["gid"], b["gid"].view(np.uint32))
    assert np.array_equal(a["prev"], b["prev"]) and np.array_equal(a["next"], b["next"])


def test_force_vjp_through_cuda_tensors(cuda_ok):
    import torch
    p = params(L=12.0, seed=19, noise="philox", f_lip=0.3, c_N=0.1)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(6)
    step = e.step_no
    n = e.n_beads[0]
    rng = np.random.default_rng(2)
    gx, gy = rng.normal(size=(2, n)).astype(np.float32)
    want = e.force_vjp(0, step, gx, gy)
    tg = [torch.from_numpy(v).cuda() for v in (gx, gy)]
    outs = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(4)]
    grad = torch.zeros(ob._capi.NGRAD, dtype=torch.float64, device="cuda")
    ob._capi.check(e.lib.dpd_force_vjp(e.h, 0, int(step), tg[0].data_ptr(), tg[1].data_ptr(),
                                       *[o.data_ptr() for o in outs], grad.data_ptr()))
    torch.cuda.synchronize()
    for w, g in zip(want[:4], outs):
        assert np.array_equal(w, g.cpu().numpy())
    assert np.array_equal(want[4], grad.cpu().numpy())
