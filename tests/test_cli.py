"""The drop-in front end without a GPU: command-line contract, file formats
against the reference engine's own files (tests/golden/run_L10_seed3.npz, made
by the reference executable), checkpoint round trip, csv truncation."""
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG, golden
from oercel_b200 import cli

EXE = os.path.join(PKG, "bin", "oercel_b200")


def fixture_bytes(key):
    return bytes(golden("run_L10_seed3.npz")[key])


def test_usage_and_params_listing(capsys):
    assert cli.run(["oercel_b200"]) == 2
    assert "usage" in capsys.readouterr().err
    assert cli.run(["oercel_b200", "--params"]) == 0
    out = capsys.readouterr().out
    for key in ("`L`", "`warmup`", "`restart_reseed`", "`p_grow`"):
        assert key in out
    assert "**W**" in out  # the default repulsion matrix


def test_errors_exit_1(tmp_path, capsys):
    ini = tmp_path / "p.ini"
    ini.write_text("L = 16\nfoo = 3\n")
    assert cli.run(["x", str(ini), str(tmp_path / "o")]) == 1
    assert "unknown parameter 'foo'" in capsys.readouterr().err
    ini.write_text("L = 16\nf_Ka = 0\nkT_amp = 1.5\n")
    assert cli.run(["x", str(ini), str(tmp_path / "o")]) == 1
    assert "kT_amp" in capsys.readouterr().err
    ini.write_text("L = 16\nf_Ka = 0\nlip_arch = star\n")
    assert cli.run(["x", str(ini), str(tmp_path / "o")]) == 1
    assert "lip_arch" in capsys.readouterr().err
    ini.write_text("L = 16\nk_angle = 0\nf_Ka = 0\ninit = restart\n")
    assert cli.run(["x", str(ini), str(tmp_path / "o")]) == 1
    assert "needs restart" in capsys.readouterr().err
    ini.write_text("L = 16\nchem_kind = enzyme\n")
    assert cli.run(["x", str(ini), str(tmp_path / "o")]) == 1
    assert "chem_kind" in capsys.readouterr().err
    ini.write_text("L = 16\nk_angle = 0\n")
    assert cli.run(["x", str(ini), str(tmp_path / "o"), "seed"]) == 1
    assert "not key=value" in capsys.readouterr().err
    assert cli.run(["x", str(tmp_path / "missing.ini"), str(tmp_path / "o")]) == 1


def test_executable_wrapper():
    r = subprocess.run([sys.executable, EXE, "--params"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "`seed`" in r.stdout
    r = subprocess.run([sys.executable, EXE], capture_output=True, text=True, timeout=120)
    assert r.returncode == 2


def test_read_reference_snapshot(tmp_path):
    p = tmp_path / "snap.bin"
    p.write_bytes(fixture_bytes("snap_24"))
    s = cli.read_snapshot(str(p))
    assert (s["version"], s["N"], s["step"], s["L"]) == (1, 400, 24, 10.0)
    assert s["time"] == pytest.approx(0.48)
    assert np.bincount(s["type"], minlength=4)[:4].tolist() == [320, 20, 40, 20]
    assert s["bonds"].shape == (40, 2) and np.all(s["bonds"][:, 0] < s["bonds"][:, 1])


def test_snapshot_writer_is_byte_identical_to_the_reference(tmp_path):
    """the reference checkpoint at step 24, read and written as a snapshot,
    gives the reference's own snap_0000000024.bin byte for byte"""
    ck_path = tmp_path / "ckpt.bin"
    ck_path.write_bytes(fixture_bytes("ckpt_24"))
    ck = cli.read_ckpt(str(ck_path))
    assert (ck["N"], ck["step"], ck["L"], ck["seed"], ck["warm_end"]) == (400, 24, 10.0, 3, 8)
    out = tmp_path / "snap.bin"
    cli.write_snapshot(str(out), ck, ck["step"], ck["time"], ck["L"])
    assert out.read_bytes() == fixture_bytes("snap_24")


def test_reference_checkpoint_links_are_consistent(tmp_path):
    ck_path = tmp_path / "ckpt.bin"
    ck_path.write_bytes(fixture_bytes("ckpt_24"))
    ck = cli.read_ckpt(str(ck_path))
    n = ck["N"]
    assert sorted(ck["gid"].tolist()) == list(range(n))
    has = ck["next"] >= 0
    assert np.array_equal(ck["prev"][ck["next"][has]], np.nonzero(has)[0])
    # every link joins lipid beads (H or T)
    assert np.all(np.isin(ck["type"][has], [1, 2])) and np.all(np.isin(ck["type"][ck["next"][has]], [1, 2]))
    assert ck["anchor"] == (0.0, 0, 0.02)


def test_checkpoint_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    n = 50
    st = dict(gid=rng.permutation(n).astype(np.uint32), type=rng.integers(0, 4, n).astype(np.uint8),
              prev=np.full(n, -1, np.int32), next=np.full(n, -1, np.int32))
    st["next"][3], st["prev"][7] = 7, 3
    for k in ("x", "y", "vhx", "vhy", "fx", "fy"):
        st[k] = rng.random(n).astype(np.float32)
    path = str(tmp_path / "ckpt.bin")
    rng = np.array([1, 2**63, 3, 2**64 - 1], np.uint64)
    cli.write_ckpt(path, st, 1234, 24.68, 16.0, 2**63 + 5, 1000, (0.0, 0, 0.02), keep_copy=str(tmp_path / "k.bin"),
                   rng=rng)
    for p in (path, str(tmp_path / "k.bin")):
        ck = cli.read_ckpt(p)
        assert (ck["N"], ck["step"], ck["time"], ck["L"], ck["seed"], ck["warm_end"]) == \
            (n, 1234, 24.68, 16.0, 2**63 + 5, 1000)
        for k in st:
            assert np.array_equal(ck[k], st[k]), k
        assert np.array_equal(ck["rng"], rng)
    raw = open(path, "rb").read()
    with open(path, "wb") as f:
        f.write(raw[:-2])
    with pytest.raises(cli.EngineError):
        cli.read_ckpt(path)


def test_truncate_csv_after(tmp_path):
    p = tmp_path / "stats.csv"
    p.write_text("step,a\n0,1\n10,2\n20,3\n30,4\n40,5")  # the last line is partial
    cli.truncate_csv_after(str(p), 20)
    assert p.read_text() == "step,a\n0,1\n10,2\n20,3\n"
    p.write_text("step,a\n0,1\n10,2\n10,3\n")
    cli.truncate_csv_after(str(p), 10)
    assert p.read_text() == "step,a\n0,1\n10,2\n10,3\n"
    cli.truncate_csv_after(str(tmp_path / "none.csv"), 5)  # a missing file is left alone


def test_snapshot_header_layout(tmp_path):
    st = dict(x=np.array([1.5, 0.25], np.float32), y=np.array([2.0, 3.0], np.float32),
              type=np.array([2, 1], np.uint8), gid=np.array([1, 0], np.uint32), next=np.array([-1, 0], np.int32))
    p = str(tmp_path / "s.bin")
    cli.write_snapshot(p, st, 7, 0.14, 8.0)
    b = open(p, "rb").read()
    assert b[:4] == b"OCEL" and struct.unpack_from("<iiiqdd", b, 4) == (1, 2, 1, 7, 0.14, 8.0)
    s = cli.read_snapshot(p)
    assert s["x"].tolist() == [0.25, 1.5] and s["type"].tolist() == [1, 2] and s["bonds"].tolist() == [[0, 1]]


def _ref_ckpt_fields(b):
    ver, n, ml, nh = struct.unpack_from("<iiii", b, 4)
    o = 20 + (4 if ver == 3 else 0) + 32 + 32 + 48
    head = b[:o]
    out = {"head": head, "n": n}
    for k, dt in (("gid", np.uint32), ("type", np.uint8), ("mpos", np.int8), ("nxt", np.int32)):
        out[k] = np.frombuffer(b, dt, n, o)
        o += n * np.dtype(dt).itemsize
    for k in ("x", "y", "vx", "vy", "fx", "fy"):
        out[k] = np.frombuffer(b, np.float64, n, o)
        o += 8 * n
    assert b[o:] == b"END!"
    return out


def test_reference_checkpoint_writer_round_trip(tmp_path):
    """the reference's own checkpoint, read and written again: the same header,
    the same gids, types, template positions and links in the same slot order
    (the reference's cell order with nsub = 4), the state rounded to FP32.
    From the beads in a shuffled slot order: the reference's cell order again
    (within a cell the beads keep their given order; any order of a cell is a
    sorted order) and the same beads"""
    ref = fixture_bytes("ckpt_24")
    path = tmp_path / "ref.bin"
    path.write_bytes(ref)
    ck = cli.read_ckpt(str(path))
    a = _ref_ckpt_fields(ref)
    for order in (np.arange(ck["N"]), np.random.default_rng(5).permutation(ck["N"])):
        inv = np.empty_like(order)
        inv[order] = np.arange(len(order))
        st = {k: ck[k][order] for k in ("gid", "type", "x", "y", "vhx", "vhy", "fx", "fy")}
        nx = ck["next"][order]
        st["next"] = np.where(nx >= 0, inv[np.maximum(nx, 0)], -1).astype(np.int32)
        pv = ck["prev"][order]
        st["prev"] = np.where(pv >= 0, inv[np.maximum(pv, 0)], -1).astype(np.int32)
        out = tmp_path / "out.bin"
        cli.write_reference_ckpt(str(out), st, ck["step"], ck["time"], ck["L"], ck["seed"], ck["warm_end"],
                                 ck["anchor"], ck["rng"], 0.0, ck["soup_seed"], ck["mlen"], ck["nH"], ck["arch"], 4)
        b = _ref_ckpt_fields(out.read_bytes())
        assert b["head"] == a["head"]
        ncy = 10 * 4
        key = np.minimum((b["x"] * 1.0).astype(int), 9) * ncy + np.minimum((b["y"] * 4.0).astype(int), ncy - 1)
        assert np.all(np.diff(key) >= 0)
        ga, gb = a["gid"].astype(np.int64), b["gid"].astype(np.int64)

        def by_gid(f, g, k):
            v = np.empty_like(f[k])
            v[g] = f[k]
            return v

        for k in ("type", "mpos"):
            assert np.array_equal(by_gid(b, gb, k), by_gid(a, ga, k)), k
        nxa = np.where(a["nxt"] >= 0, ga[np.maximum(a["nxt"], 0)], -1)
        nxb = np.where(b["nxt"] >= 0, gb[np.maximum(b["nxt"], 0)], -1)
        assert np.array_equal(by_gid({"n": nxb}, gb, "n"), by_gid({"n": nxa}, ga, "n"))
        for k in ("x", "y", "vx", "vy", "fx", "fy"):
            assert np.array_equal(by_gid(b, gb, k), by_gid(a, ga, k).astype(np.float32).astype(np.float64)), k
        if order[0] == 0 and np.all(order == np.arange(len(order))):
            for k in ("gid", "type", "mpos", "nxt"):
                assert np.array_equal(b[k], a[k]), k


def test_reference_checkpoint_writer_refuses_grown_chains(tmp_path):
    """a chain longer than the template (grown by the lipid chemistry) or a free
    T has no form in the reference's checkpoint"""
    path = tmp_path / "ref.bin"
    path.write_bytes(fixture_bytes("ckpt_24"))
    ck = cli.read_ckpt(str(path))
    st = {k: ck[k].copy() for k in ("gid", "type", "x", "y", "vhx", "vhy", "fx", "fy", "prev", "next")}
    w = int(np.nonzero(st["type"] == 0)[0][0])
    tail = int(np.nonzero((st["type"] == 2) & (st["next"] < 0) & (st["prev"] >= 0))[0][0])
    st["type"][w] = 2
    st["next"][tail], st["prev"][w] = w, tail   # a W turned into a fourth chain bead
    args = (ck["step"], ck["time"], ck["L"], ck["seed"], ck["warm_end"], ck["anchor"], ck["rng"], 0.0,
            ck["soup_seed"], ck["mlen"], ck["nH"], ck["arch"], 4)
    with pytest.raises(cli.EngineError, match="reference checkpoint"):
        cli.write_reference_ckpt(str(tmp_path / "o.bin"), st, *args)
    st2 = {k: ck[k].copy() for k in ("gid", "type", "x", "y", "vhx", "vhy", "fx", "fy", "prev", "next")}
    st2["type"][w] = 2                                # a free T
    with pytest.raises(cli.EngineError, match="reference checkpoint"):
        cli.write_reference_ckpt(str(tmp_path / "o.bin"), st2, *args)
