"""Catalyst chemistry rates against the reference executable, statistically
(the reference's cross-engine criterion, tests/compare.py: per kind |z| < 4.5
or within 15 %): the drop-in engine with its default Philox noise runs the
reference's ini for 300 steps from the same soups (four seeds); its event
totals per kind (fed beads for the feed) are compared with the reference's
(tests/golden/catalyst_rates.npz, made by the reference executable).  The
trajectories differ (other noise), the rates must not."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG, golden

pytestmark = pytest.mark.gpu
EXE = os.path.join(PKG, "bin", "oercel_b200")


def test_catalyst_rates_match_the_reference(cuda_ok, tmp_path):
    g = golden("catalyst_rates.npz")
    kinds = bytes(g["kinds"]).decode().split(",")
    ini = tmp_path / "p.ini"
    ini.write_bytes(bytes(g["ini"]))
    totals = np.zeros_like(g["totals"])
    finals = []
    for a, seed in enumerate(g["seeds"]):
        out = tmp_path / f"run{seed}"
        r = subprocess.run([sys.executable, EXE, str(ini), str(out), f"seed={int(seed)}"], capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        rows = [ln.split(",") for ln in (out / "events.csv").read_text().strip().split("\n")[1:]]
        for row in rows:
            totals[a, kinds.index(row[1])] += int(row[2]) if row[1] == "feed" else 1
        finals.append([float(v) for v in (out / "stats.csv").read_text().strip().split("\n")[-1].split(",")])
    mine, ref = totals.sum(0).astype(float), g["totals"].sum(0).astype(float)
    for k, name in enumerate(kinds):
        z = abs(mine[k] - ref[k]) / np.sqrt(max(mine[k] + ref[k], 1.0))
        assert z < 4.5 or abs(mine[k] - ref[k]) <= 0.15 * ref[k], (name, mine[k], ref[k], z)
    # final composition (nW .. nKb and lipids) within 15 % on average over the seeds
    fm, fr = np.array(finals)[:, 3:11].mean(0), g["finals"][:, 3:11].mean(0)
    assert np.all(np.abs(fm - fr) <= 0.15 * np.maximum(fr, 10.0)), (fm, fr)


def block_mean(x, nb=10):
    x = x[: len(x) // nb * nb].reshape(nb, -1).mean(1)
    return x.mean(), x.std(ddof=1) / np.sqrt(nb)


def test_membrane_physics_matches_the_reference(cuda_ok, tmp_path):
    """membranes.ini physics (tied H2T2 pi lipids: template bonds with a rung,
    tail angle terms, k_bond 300, dt 0.03) on a 24 x 24 box for 4000 steps, two
    seeds: the mean kinetic temperature and the mean of the per-row max bond
    length over steps 1000-4000 agree with the reference executable's within
    the reference's criterion (4 combined block errors, or 0.003)"""
    g = golden("membrane_stats.npz")
    ini = tmp_path / "p.ini"
    ini.write_bytes(bytes(g["ini"]))
    mine_T, ref_T, mine_B, ref_B = [], [], [], []
    for seed in g["seeds"]:
        out = tmp_path / f"m{seed}"
        r = subprocess.run([sys.executable, EXE, str(ini), str(out), f"seed={int(seed)}"], capture_output=True,
                           text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
        rows = np.array([[float(v) for v in ln.split(",")]
                         for ln in (out / "stats.csv").read_text().strip().split("\n")[1:]])
        ref = g[f"stats_{int(seed)}"]
        for src, T, B in ((rows, mine_T, mine_B), (ref, ref_T, ref_B)):
            late = src[src[:, 0] > 1000]
            T.append(late[:, 2])
            B.append(late[:, 11])
    for mine, ref, name in ((mine_T, ref_T, "T_kin"), (mine_B, ref_B, "max_bond")):
        m, sm = block_mean(np.concatenate(mine))
        r_, sr = block_mean(np.concatenate(ref))
        assert abs(m - r_) < max(4 * np.hypot(sm, sr), 0.003), (name, m, sm, r_, sr)
