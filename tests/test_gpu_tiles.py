"""The tiled half-shell force kernels (one CTA per tile, staged by per-bead
loads or by bulk asynchronous copies) against the per-bead full-shell kernel: bit-identical forces for every box size and tile
shape (all round each pair term to the same fixed-point value and add the
terms in integers)."""
import numpy as np
import pytest

import oercel_b200 as ob
from gpu_util import params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fk", [0, 2])
@pytest.mark.parametrize("L", [9.0, 12.5, 32.0, 64.0])
@pytest.mark.parametrize("shape", [(8, 16), (14, 14), (4, 30), (1, 1)])
def test_tile_forces_equal_bead_forces(cuda_ok, L, shape, fk):
    p = params(L=L, seed=int(L * 10), noise="philox")
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(5)
    e.set_tuning(force_kernel=1)
    e.forces(123)
    a = e.state()
    e.set_tuning(force_kernel=fk, tile_w=shape[0], tile_h=shape[1])
    e.forces(123)
    b = e.state()
    assert np.array_equal(a["fx"], b["fx"]) and np.array_equal(a["fy"], b["fy"])


def test_tile_steps_equal_bead_steps(cuda_ok):
    p = params(L=24.0, seed=4, noise="philox", chem=1, n_chem=1, c_N=0.2, f_lip=0.3, p_grow=0.05, p_bond=0.2,
               p_break=0.01)
    runs = []
    for fk in (0, 1, 2):
        e = ob.Engine(p)
        e.set_tuning(force_kernel=fk)
        e.load_soup(0)
        e.prime()
        e.step(30)
        runs.append(e.state())
    for r in runs[1:]:
        for k in ("x", "y", "vhx", "fx", "type", "gid", "prev", "next"):
            assert np.array_equal(runs[0][k], r[k]), k


def test_tuning_validation(cuda_ok):
    e = ob.Engine(params(L=16.0, seed=1))
    before = e.tuning()
    assert before["tile_w"] * before["tile_h"] < 8 * 16  # a small box gets smaller tiles
    with pytest.raises(ob.DpdError):
        e.set_tuning(tile_w=20, tile_h=20)
    with pytest.raises(ob.DpdError):
        e.set_tuning(force_kernel=3)
    assert e.tuning() == before


def test_autotune_picks_a_valid_choice(cuda_ok, tmp_path):
    from oercel_b200.autotune import autotune
    p = params(L=48.0, seed=2, noise="philox")
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    out = autotune(e, repeats=1, cache_path=str(tmp_path / "t.json"))
    assert out["tuning"]["force_kernel"] in (0, 1, 2) and out["forces_ms"] > 0
    again = autotune(e, cache_path=str(tmp_path / "t.json"))  # from the cache
    assert again["tuning"] == out["tuning"]
    e.step(5)


@pytest.mark.parametrize("fk", [0, 2])
@pytest.mark.parametrize("noise", ["philox", "mix13"])
def test_tile_noise_modes(cuda_ok, noise, fk):
    p = params(L=20.0, seed=3, noise=noise)
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.set_tuning(force_kernel=1)
    e.forces(77)
    a = e.state()
    e.set_tuning(force_kernel=fk, tile_w=6, tile_h=10)
    e.forces(77)
    b = e.state()
    assert np.array_equal(a["fx"], b["fx"]) and np.array_equal(a["fy"], b["fy"])


def test_crowded_tile_falls_back_to_direct_sums(cuda_ok):
    """a tile whose beads overflow shared memory computes them straight from HBM, same bits"""
    from gpu_util import engine_with
    p = params(L=32.0, seed=9, noise="philox")
    s = ob.soup_for(p)
    rng = np.random.default_rng(0)
    x, y = s["x"].copy(), s["y"].copy()
    free = np.nonzero(s["prev"] + s["next"] == -2)[0][:1600]   # unbonded beads packed into a 6 x 6 patch
    x[free] = rng.uniform(1.0, 7.0, len(free)).astype(np.float32)
    y[free] = rng.uniform(1.0, 7.0, len(free)).astype(np.float32)
    runs = []
    for fk in (1, 0, 2):
        e = engine_with(p, x, y, s["vx"], s["vy"], s["type"], s["prev"], s["next"])
        e.set_tuning(force_kernel=fk, tile_w=14, tile_h=14)
        e.build_cells()
        e.forces(5)
        runs.append(e.state())
    for r in runs[1:]:
        assert np.array_equal(runs[0]["fx"], r["fx"]) and np.array_equal(runs[0]["fy"], r["fy"])


def test_bulk_staged_kernel_in_a_batch(cuda_ok):
    """replicas of uneven size in one engine (tiles of many replicas, with the
    rows of small boxes wrapping inside a tile): the bulk-staged kernel equals
    the per-bead-staged kernel bit for bit"""
    from oercel_b200 import workloads
    reps = workloads.config3(n_replicas=12, nmin=2048, nmax=16384)
    ps, nb = [p for p, _ in reps], [n for _, n in reps]
    runs = []
    for fk in (0, 2):
        e = ob.Engine(ps, nb)
        for r in range(len(ps)):
            e.load_soup(r)
        e.set_tuning(force_kernel=fk, tile_w=8, tile_h=16)
        e.prime()
        e.step(12)
        runs.append([e.state(r) for r in range(len(ps))])
    for a, b in zip(*runs):
        for k in ("x", "y", "fx", "fy", "type", "prev", "next"):
            assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("L", [9.0, 33.5, 64.0])
@pytest.mark.parametrize("shape", [(20, 20), (14, 30), (10, 40)])
def test_wide_tile_forces_equal_bead_forces(cuda_ok, L, shape):
    """512-thread CTAs with tiles of up to 512 cells (tile and halo): the same
    bits as the per-bead kernel"""
    p = params(L=L, seed=int(L * 7), noise="philox")
    e = ob.Engine(p)
    e.load_soup(0)
    e.prime()
    e.step(5)
    e.set_tuning(force_kernel=1)
    e.forces(321)
    a = e.state()
    e.set_tuning(force_kernel=0, tile_w=shape[0], tile_h=shape[1], tile_threads=512)
    e.forces(321)
    b = e.state()
    assert np.array_equal(a["fx"], b["fx"]) and np.array_equal(a["fy"], b["fy"])
    nc = int(np.floor(np.float32(L)))
    w, h = min(shape[0], nc - 2), min(shape[1], nc - 2)
    if (w + 2) * (h + 2) > 256:
        with pytest.raises(ob.DpdError):
            e.set_tuning(tile_threads=256)  # a tile of more than 256 cells does not fit 256 threads
    with pytest.raises(ob.DpdError):
        e.set_tuning(tile_threads=384)
