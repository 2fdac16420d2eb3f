"""Lipid templates and the soups of branched lipids against the reference
(host code of libdpd.so; no GPU).

tests/golden/templates.npz holds the reference's own template (mol_build,
cel/engine/oercel.c:478-576) for linear, pi, y and bola shapes with rungs and
junction terms; dpd_lipid_template must give the same bonds, angle terms and
coordinates bit for bit, in the same order.  tests/golden/mol_*.npz hold the
reference's soups of branched lipids (init_soup, oercel.c:1774-1814):
dpd_init_soup with the template must give the same state bit for bit.
"""
import json

import numpy as np
import pytest

import oercel_b200 as ob
from conftest import golden

INT_KEYS = ("bi", "bj", "ai", "aj", "ak", "akind")
DBL_KEYS = ("br0", "aK", "ac0", "px", "py", "ix", "iy")


def template_cases():
    g = golden("templates.npz")
    k = 0
    while f"c{k}_kv" in g:
        yield json.loads(bytes(g[f"c{k}_kv"]).decode()), {key[len(f"c{k}_"):]: g[key] for key in g.files
                                                          if key.startswith(f"c{k}_")}
        k += 1


@pytest.mark.parametrize("kv, ref", list(template_cases()), ids=lambda v: str(v.get("lip_arch", "")))
def test_template_matches_the_reference(kv, ref):
    t = ob.Params(**kv).template()
    assert (t.arch, t.mlen, t.nH, t.nb, t.na) == tuple(int(ref[k]) for k in ("arch", "mlen", "nH", "nb", "na"))
    for key in INT_KEYS:
        n = t.nb if key in ("bi", "bj") else t.na
        assert list(getattr(t, key)[:n]) == list(ref[key]), key
    for key in DBL_KEYS:
        n = t.nb if key == "br0" else t.na if key in ("aK", "ac0") else t.mlen
        assert np.array_equal(np.array(getattr(t, key)[:n]), ref[key]), key


def test_template_refuses_bad_shapes():
    with pytest.raises(ob.ParamError):
        ob.Params(lip_arch="star").validate()
    with pytest.raises(ob.ParamError):
        ob.Params(lip_arch="pi", lip_nT=0).validate()
    with pytest.raises(ob.ParamError):
        ob.Params(lip_arch="bola", lip_nT=7).validate()  # 17 beads


@pytest.mark.parametrize("name", ["mol_pi_L12_seed31.npz", "mol_y_L12_seed32.npz", "mol_bola_L12_seed33.npz"])
def test_branched_soup_matches_the_reference(name):
    g = golden(name)
    kv = dict(line.split(" = ", 1) for line in bytes(g["ini"]).decode().strip().split("\n"))
    p = ob.Params().update(list(kv.items()))
    s = ob.make_soup(float(kv["L"]), p.n_beads(), int(kv["seed"]), kT=p.kT, r0=p.r0, nH=p.lip_nH, nT=p.lip_nT,
                     f_lip=p.f_lip, f_Ka=p.f_Ka, f_Kb=p.f_Kb, c_N=p.c_N, mol=p.template())
    for k in ("x", "y", "vx", "vy", "type"):
        assert np.array_equal(s[k], g[f"{k}_soup"]), k
    assert np.array_equal(s["next"], g["nxt_soup"])
    assert np.array_equal(s["rng"], g["rng_soup"])
    assert s["n_lipid_beads"] == int((g["mpos_soup"] >= 0).sum())


def test_pi_snapshot_writer_is_byte_identical_to_the_reference(tmp_path):
    """the reference's version-3 checkpoint of a pi-lipid run (with catalyst
    chemistry) at step 24, written as a snapshot with the template's bond list,
    gives the reference's own snap_0000000024.bin byte for byte"""
    from oercel_b200 import cli
    g = golden("run_pi_L16_seed7.npz")
    kv = [tuple(line.split(" = ", 1)) for line in bytes(g["ini"]).decode().strip().split("\n")]
    p = ob.Params().update(kv)
    ck_path = tmp_path / "ckpt.bin"
    ck_path.write_bytes(bytes(g["ckpt_24"]))
    ck = cli.read_ckpt(str(ck_path))
    assert (ck["arch"], ck["mlen"], ck["nH"], ck["step"]) == (1, p.mlen(), 2, 24)
    out = tmp_path / "snap.bin"
    cli.write_snapshot(str(out), ck, ck["step"], ck["time"], ck["L"], p.template())
    assert out.read_bytes() == bytes(g["snap_24"])
