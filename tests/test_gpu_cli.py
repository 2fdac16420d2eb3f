"""The drop-in executable on the GPU against runs of the reference executable
(tests/golden/run_L10_seed3.npz: a fresh soup with the repulsion warm-up, 24
steps, and a restart from its checkpoint to step 36; the same with the angle
terms, stirring and the temperature cycle, and with the catalyst chemistry),
plus the continuation, walltime and SIGTERM contract.

Criteria: the step-0 snapshot (the soup) is byte-identical; stats rows agree in
step, time, counts and chain numbers exactly and in T_kin and max_bond within
2e-3 relative (FP32 state against FP64 over <= 36 steps); snapshot positions
within 1e-3 (minimum image).  A continuation from this engine's own checkpoint
is bit-identical to the uninterrupted run.  With chemistry, the events are the
reference's (step, kind, bead, variant)."""
import os
import shutil
import signal
import subprocess
import sys
import time

import numpy as np
import pytest

from conftest import PKG, golden
from oercel_b200 import cli

pytestmark = pytest.mark.gpu
EXE = os.path.join(PKG, "bin", "oercel_b200")
G = "run_L10_seed3.npz"
# the same runs with angle terms (k_angle = 10, H-T-T-T lipids), stirring and the temperature cycle
G_EXTRAS = "run_extras_L10_seed4.npz"
# the same runs with the reference's catalyst chemistry every 4 steps (events on)
G_CAT = "run_cat_L16_seed5.npz"
# catalyst checks every step from a soup without warm-up at dt = 0.05: at step 5 a bead moves more
# than 0.5 and the reference sorts again before its check
G_CAT_RESORT = "run_cat_resort_L16_seed5.npz"
# pi lipids (the template's bonds, junction and rung) in a membranes-like soup with the catalyst chemistry
G_PI = "run_pi_L16_seed7.npz"


def fixture_bytes(key, name=G):
    return bytes(golden(name)[key])


def run_exe(ini, out, *over, timeout=600):
    r = subprocess.run([sys.executable, EXE, str(ini), str(out), *over], capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


@pytest.fixture
def ini(tmp_path):
    p = tmp_path / "p.ini"
    p.write_bytes(fixture_bytes("ini"))
    return p


def write_ini(tmp_path, name):
    p = tmp_path / "p.ini"
    p.write_bytes(fixture_bytes("ini", name))
    return p


def rows(text):
    lines = text.strip().split("\n")
    return [ln.split(",") for ln in lines[1:]]


def check_stats(got_text, ref_text):
    got, ref = rows(got_text), rows(ref_text)
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        assert g[0] == r[0] and g[1] == r[1], (g, r)             # step, time
        assert g[3:11] == r[3:11], (g, r)                        # type counts, n_lipids
        assert float(g[2]) == pytest.approx(float(r[2]), rel=2e-3), (g, r)   # T_kin
        assert float(g[11]) == pytest.approx(float(r[11]), rel=2e-3), (g, r)  # max_bond


def check_events(got_text, ref_text):
    """the same events (step, kind, bead, variant) in any order within a step"""
    key = lambda r: (int(r[0]), r[1], int(r[2]), r[5])
    assert got_text.startswith("step,kind,i,x,y,variant\n")
    assert sorted(map(key, rows(got_text))) == sorted(map(key, rows(ref_text)))


# positions: FP32 against FP64; at dt = 0.05 the hot start amplifies the rounding differences more
POS_TOL = {G_CAT_RESORT: 1e-2}


def check_snapshot(path, ref_key, name=G):
    ref_path = path + ".ref"
    with open(ref_path, "wb") as f:
        f.write(fixture_bytes(ref_key, name))
    a, b = cli.read_snapshot(path), cli.read_snapshot(ref_path)
    assert (a["N"], a["step"], a["L"]) == (b["N"], b["step"], b["L"])
    assert a["time"] == pytest.approx(b["time"], abs=1e-12)
    assert np.array_equal(a["type"], b["type"]) and np.array_equal(a["bonds"], b["bonds"])
    L = b["L"]
    for k in ("x", "y"):
        d = a[k].astype(np.float64) - b[k]
        d -= L * np.round(d / L)
        assert np.abs(d).max() < POS_TOL.get(name, 1e-3), k


@pytest.mark.parametrize("name", [G, G_EXTRAS, G_CAT, G_CAT_RESORT, G_PI])
def test_run_matches_the_reference_executable(cuda_ok, tmp_path, name):
    ini = write_ini(tmp_path, name)
    out = tmp_path / "run"
    run_exe(ini, out, "noise=mix13")
    assert (out / "snap_0000000000.bin").read_bytes() == fixture_bytes("snap_0", name)
    check_stats((out / "stats.csv").read_text(), fixture_bytes("stats_a", name).decode())
    if "events_a" in golden(name):
        check_events((out / "events.csv").read_text(), fixture_bytes("events_a", name).decode())
    check_snapshot(str(out / "snap_0000000012.bin"), "snap_12", name)
    check_snapshot(str(out / "snap_0000000024.bin"), "snap_24", name)
    log = (out / "log.txt").read_text()
    assert log.rstrip().endswith("done at step 24") and "timing:" in log
    warmup = dict(ln.split(" = ", 1) for ln in fixture_bytes("ini", name).decode().strip().split("\n"))["warmup"]
    assert f"warmup = {warmup}" in (out / "params.ini").read_text()
    assert cli.read_ckpt(str(out / "ckpt.bin"))["step"] == 24


@pytest.mark.parametrize("name", [G, G_EXTRAS, G_CAT, G_CAT_RESORT, G_PI])
def test_restart_from_a_reference_checkpoint(cuda_ok, tmp_path, name):
    ini = write_ini(tmp_path, name)
    ck = tmp_path / "ref_ckpt.bin"
    ck.write_bytes(fixture_bytes("ckpt_24", name))
    out = tmp_path / "cont"
    run_exe(ini, out, "noise=mix13", f"restart={ck}", "steps=36")
    check_stats((out / "stats.csv").read_text(), fixture_bytes("stats_b", name).decode())
    if "events_b" in golden(name):
        check_events((out / "events.csv").read_text(), fixture_bytes("events_b", name).decode())
    check_snapshot(str(out / "snap_0000000036.bin"), "snap_36", name)
    assert "restart from" in (out / "log.txt").read_text()


CHEM = ("chem=1", "chem_kind=lipid", "events=1", "n_chem=1", "p_grow=0.05", "p_bond=0.3", "p_break=0.02",
        "noise=philox", "ckpt_every=12", "ckpt_keep=1", "snap_every=6")


def test_own_checkpoint_continuation_is_bitwise(cuda_ok, ini, tmp_path):
    a = tmp_path / "a"
    run_exe(ini, a, *CHEM)
    events = (a / "events.csv").read_text()
    assert events.startswith("step,kind,i,x,y,variant\n")
    kinds = {r[1] for r in rows(events)}
    assert kinds and kinds <= {"grow", "brk", "bond"}
    # into a fresh directory
    b = tmp_path / "b"
    run_exe(ini, b, *CHEM, f"restart={a}/ckpt_0000000012.bin")
    for s in (18, 24):
        assert (b / f"snap_{s:010d}.bin").read_bytes() == (a / f"snap_{s:010d}.bin").read_bytes()
    sa = (a / "stats.csv").read_text().split("\n")
    sb = (b / "stats.csv").read_text().split("\n")
    assert sb[1:] == [ln for ln in sa[1:] if not ln or int(ln.split(",")[0]) > 12]
    # into the same directory: stats.csv and events.csv are truncated after step 12 and rewritten identically
    saved = {f: (a / f).read_text() for f in ("stats.csv", "events.csv")}
    shutil.copy(a / "ckpt_0000000012.bin", tmp_path / "c12.bin")
    run_exe(ini, a, *CHEM, f"restart={tmp_path}/c12.bin")
    for f, text in saved.items():
        assert (a / f).read_text() == text, f


def test_walltime_stop_writes_a_checkpoint(cuda_ok, ini, tmp_path):
    out = tmp_path / "w"
    run_exe(ini, out, "noise=philox", "steps=100000", "walltime=1e-9", "stats_every=5", "snap_every=0")
    log = (out / "log.txt").read_text()
    assert "(walltime), checkpoint written" in log and "stopped early; restart to continue" in log
    st = cli.read_ckpt(str(out / "ckpt.bin"))["step"]
    assert 0 < st < 100000 and f"stopping at step {st} " in log


def test_sigterm_stops_cleanly(cuda_ok, ini, tmp_path):
    out = tmp_path / "s"
    p = subprocess.Popen([sys.executable, EXE, str(ini), str(out), "noise=philox", "steps=100000000",
                          "stats_every=1000", "snap_every=0", "log_every=1000"], stdout=subprocess.PIPE,
                         stderr=subprocess.PIPE, text=True)
    try:
        t0 = time.time()
        while time.time() - t0 < 300:
            line = p.stdout.readline()
            if not line or line.startswith("step "):
                break
        time.sleep(0.5)
        p.send_signal(signal.SIGTERM)
        rc = p.wait(timeout=120)
    finally:
        if p.poll() is None:
            p.kill()
            p.wait()
    assert rc == 0
    log = (out / "log.txt").read_text()
    assert "(signal), checkpoint written" in log
    assert cli.read_ckpt(str(out / "ckpt.bin"))["step"] > 0


REF_EXE = os.path.join(os.path.dirname(PKG), "oracle", "_ref", "oercel_portable")


@pytest.mark.parametrize("name", [G, G_EXTRAS, G_CAT, G_PI])
def test_reference_executable_continues_our_checkpoint(cuda_ok, tmp_path, name):
    """ckpt_format = reference: this engine runs the first 24 steps and writes
    the reference's own checkpoint (OCKP v2, v3 for pi lipids); the reference
    executable (built from cel/engine/oercel.c, the build that made the
    fixtures) continues it to step 36.  Its stats rows, events and final
    snapshot must agree with the reference's continuation of its own run
    within the criteria above."""
    if not os.path.exists(REF_EXE):
        pytest.skip("the reference executable is not built (oracle/Makefile with the reference sources)")
    ini = write_ini(tmp_path, name)
    out = tmp_path / "ours"
    run_exe(ini, out, "noise=mix13", "ckpt_format=reference")
    ck = out / "ckpt.bin"
    assert ck.read_bytes()[:4] == b"OCKP"
    assert cli.read_ckpt(str(ck))["step"] == 24
    cont = tmp_path / "ref"
    r = subprocess.run([REF_EXE, str(ini), str(cont), f"restart={ck}", "steps=36"], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, (r.stdout + r.stderr)[-2000:]
    check_stats((cont / "stats.csv").read_text(), fixture_bytes("stats_b", name).decode())
    if "events_b" in golden(name):
        check_events((cont / "events.csv").read_text(), fixture_bytes("events_b", name).decode())
    check_snapshot(str(cont / "snap_0000000036.bin"), "snap_36", name)


def test_reference_checkpoint_refuses_grown_chains(cuda_ok, ini, tmp_path):
    """the lipid chemistry grows and cuts chains, which the reference's
    fixed-length templates cannot describe: a clear error, exit 1"""
    out = tmp_path / "g"
    r = subprocess.run([sys.executable, EXE, str(ini), str(out), *CHEM, "p_grow=0.5", "ckpt_format=reference"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 1
    assert "oercel: error:" in r.stderr and "reference checkpoint" in r.stderr
