"""Generate the golden fixtures of this directory from the reference engine itself.

    OERCEL_REF_ROOT=<reference checkout> python tests/golden/make_golden.py

Runs the reference's own routines (cel/engine/oercel.c compiled by
oracle/Makefile into oracle/_ref/libref_oercel.so with FMA contraction off) and
stores their outputs as small .npz files.  The reference has no data files of
its own: its tests regenerate inputs from seeds (cel/engine/tests/forcetest.c),
and so does this script, with the reference's own soup initialisation.
Needs the reference sources (only in the build container); the fixtures are
committed so that the tests run anywhere.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("OERCEL_REF_ROOT", "")  # the reference checkout this generator reads
if not REF_ROOT or not os.path.isdir(os.path.join(REF_ROOT, "cel", "engine")):
    sys.exit("make_golden.py: set OERCEL_REF_ROOT to the reference checkout (the directory holding cel/engine)")
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402

# configuration 1 of the workload table mapped onto the reference's keys (P is the reference's N)
CONFIG1 = dict(L=32, rho=4, dt=0.02, gamma=4.5, kT=1, k_bond=100, r0=0.5, k_angle=0, lip_nH=1, lip_nT=2,
               f_lip=0.15, f_Ka=0, f_Kb=0, c_N=0.05, chem=0, events=0, warmup=0, seed=0, threads=1, nsub=1,
               a_W_H=25, a_W_T=75, a_H_T=50, a_W_N=25, a_H_N=25, a_N_T=75)


def f32(a):
    return np.asarray(a, np.float64).astype(np.float32).astype(np.float64)


def soup_fixture():
    r = O.Ref(**CONFIG1)
    a = r.get()
    np.savez_compressed(os.path.join(HERE, "soup_L32_seed0.npz"), x=a["x"], y=a["y"], vx=a["vx"], vy=a["vy"],
                        type=a["type"], nxt=a["nxt"])


def step_fixture(L, seed, name, steps=(12345,)):
    """one state at non-trivial L, sorted by the reference with nsub = 1, its
    pair forces (mix13 noise), bonded forces, and one integrator update"""
    kv = dict(CONFIG1, L=L, seed=seed, f_lip=0.15, c_N=0.1)
    r = O.Ref(**kv)
    a = r.get()
    rng = np.random.default_rng(seed)
    n = len(a["x"])
    for k in ("x", "y", "vx", "vy"):
        a[k] = f32(a[k])
    a["vtx"] = f32(a["vx"] + 0.3 * rng.standard_normal(n))
    a["vty"] = f32(a["vy"])
    # beads on cell edges and the box edge (cel/engine/tests/forcetest.c:46)
    Lf = float(np.float32(L))
    a["x"][0] = 0.0
    a["y"][1] = float(np.nextafter(np.float32(Lf), np.float32(0)))
    a["x"][2] = float(np.float32(3 * Lf / np.floor(L)))
    r.set(a)
    r.sort()
    b = r.get()
    cs = r.cells()
    out = dict(x0=a["x"], y0=a["y"], vx0=a["vx"], vy0=a["vy"], vtx0=a["vtx"], vty0=a["vty"], type0=a["type"],
               nxt0=a["nxt"], gid=b["gid"], cstart=cs, L=np.float64(L))
    for s in steps:
        r.pair(s)
        f = r.get()
        out[f"fx_{s}"] = f["fx"]
        out[f"fy_{s}"] = f["fy"]
    r.pair(steps[0])
    f0 = r.get()
    mb = r.bonded()
    f1 = r.get()
    out["bfx"] = f1["fx"] - f0["fx"]
    out["bfy"] = f1["fy"] - f0["fy"]
    out["maxbond"] = np.float64(mb)
    r.integrate()
    g = r.get()
    for k in ("x", "y", "vx", "vy", "vtx", "vty"):
        out[f"int_{k}"] = g[k]
    out["int_fx"], out["int_fy"] = f1["fx"], f1["fy"]
    np.savez_compressed(os.path.join(HERE, name), **out)


EXTRAS = dict(k_angle=10, lip_nT=3, stir_A=1.5, stir_n=2, kT_amp=0.4, kT_period=37)


def extras_fixture(L=12.5, seed=21, step=777):
    """angle terms, stirring and the temperature cycle: one sorted state
    (nsub = 1), the reference's pair forces at `step` (stirring body force and
    kT(t) noise included) and its bonded forces (bonds + angles)"""
    kv = dict(CONFIG1, L=L, seed=seed, f_lip=0.3, c_N=0.1, **EXTRAS)
    r = O.Ref(**kv)
    a = r.get()
    rng = np.random.default_rng(seed)
    n = len(a["x"])
    Lf = float(np.float32(L))
    for k in ("x", "y"):  # bent, stretched chains: bonds and angles under load
        a[k] = np.mod(a[k] + 0.12 * rng.standard_normal(n) * (a["mpos"] >= 0), Lf)
    for k in ("x", "y", "vx", "vy"):
        a[k] = f32(a[k])
        if k in ("x", "y"):
            a[k][a[k] >= Lf] = 0.0
    a["vtx"] = f32(a["vx"] + 0.3 * rng.standard_normal(n))
    a["vty"] = f32(a["vy"])
    r.set(a)
    r.sort()
    b = r.get()
    out = dict(x0=a["x"], y0=a["y"], vtx0=a["vtx"], vty0=a["vty"], type0=a["type"], nxt0=a["nxt"], gid=b["gid"],
               cstart=r.cells(), L=np.float64(L), step=np.int64(step), seed=np.int64(seed))
    r.pair(step)
    f = r.get()
    out["fx"], out["fy"] = f["fx"], f["fy"]
    mb = r.bonded()
    g = r.get()
    out["bfx"], out["bfy"] = g["fx"] - f["fx"], g["fy"] - f["fy"]
    out["maxbond"] = np.float64(mb)
    np.savez_compressed(os.path.join(HERE, f"extras_L{str(L).replace('.', 'p')}_seed{seed}.npz"), **out)


CATALYST = dict(L=16, rho=4, dt=0.02, gamma=4.5, kT=1, k_bond=100, r0=0.5, k_angle=10, lip_nH=1, lip_nT=3,
                f_lip=0.1, f_Ka=0.03, f_Kb=0.02, c_N=0.25, chem=1, n_chem=1, events=1, warmup=0, threads=1, nsub=1,
                p_syn_a=0.5, p_syn_b=0.6, p_rep_a=0.4, p_rep_b=0.4, mu=0.3, p_ld=0.05, p_kd=0.05, p_nd=0.03,
                feed="uniform", p_feed=0.05, feed_cap=0.27)


def catalyst_fixture(name, seed, step, **over):
    """one check of the reference's catalyst chemistry on a sorted soup state
    with FP32 positions: the state before (slot order) and after, the serial
    generator state before and after, and the events"""
    kv = dict(CATALYST, seed=seed, **over)
    r = O.Ref(**kv)
    r.prime()
    r.run(20)
    a = r.get()
    for k in ("x", "y", "vx", "vy", "vtx", "vty"):
        a[k] = f32(a[k])
    Lf = float(np.float32(kv["L"]))
    for k in ("x", "y"):
        a[k][a[k] >= Lf] = 0.0
    r.set(a)
    r.sort()
    b = r.get()
    out = {f"{k}0": b[k] for k in ("x", "y", "vx", "vy", "vtx", "vty", "type", "gid", "nxt", "mpos")}
    out["cstart"] = r.cells()
    out["rng0"] = r.rng()
    moved = r.chemistry(step)
    c = r.get()
    out.update({f"{k}1": c[k] for k in ("x", "y", "vx", "vy", "vtx", "vty", "type", "nxt")})
    out["rng1"] = r.rng()
    ev = r.events()
    out["events"] = np.array([(e[0], e[1], e[2], e[3], e[4], e[5]) for e in ev],
                             dtype=[("step", "i8"), ("kind", "i4"), ("i", "i8"), ("variant", "i4"), ("x", "f8"),
                                    ("y", "f8")])
    out["moved"] = np.int32(moved)
    out["step"] = np.int64(step)
    out["seed"] = np.int64(seed)
    out["ini"] = np.frombuffer("".join(f"{k} = {v}\n" for k, v in kv.items()).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, name), **out)


# lipid shapes whose templates are checked against the reference's mol_build
TEMPLATES = [dict(lip_arch="linear", lip_nH=2, lip_nT=3, k_angle=7), dict(lip_arch="pi", lip_nT=1),
             dict(lip_arch="pi", lip_nT=3, lip_tie=2, k_head=4, cos_head=0.2, r0_head=0.7),
             dict(lip_arch="y", lip_nT=2, lip_tie=1, k_head=3, cos_head=-0.3), dict(lip_arch="y", lip_nT=4, k_angle=0),
             dict(lip_arch="bola", lip_nT=2, lip_tie=1, k_head=2, r0_head=0.6), dict(lip_arch="bola", lip_nT=4, lip_tie=3)]


def template_fixture():
    """the reference's template (g_mol) for each shape of TEMPLATES"""
    import json
    out = {}
    for k, kv in enumerate(TEMPLATES):
        t = O.Ref(L=8, f_lip=0.1, seed=1, threads=1, **kv).template()
        for key, v in t.items():
            out[f"c{k}_{key}"] = np.asarray(v)
        out[f"c{k}_kv"] = np.frombuffer(json.dumps(kv).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "templates.npz"), **out)


def mol_fixture(name, seed, **over):
    """a soup of branched lipids (the reference's init_soup, gid order) and,
    after 10 reference steps with FP32-rounded positions, its bonded forces
    alone (bonded_forces with the template, maxbond)"""
    kv = dict(L=12, rho=4, dt=0.02, k_angle=8, f_lip=0.3, f_Ka=0.02, f_Kb=0.0, c_N=0.05, seed=seed, threads=1,
              nsub=1, warmup=0, **over)
    r = O.Ref(**kv)
    a0 = r.get()
    out = {f"{k}_soup": a0[k] for k in ("x", "y", "vx", "vy", "type", "nxt", "mpos")}
    out["rng_soup"] = r.rng()
    r.prime()
    r.run(10)
    a = r.get()
    for k in ("x", "y", "vx", "vy", "vtx", "vty"):
        a[k] = f32(a[k])
    Lf = float(np.float32(kv["L"]))
    for k in ("x", "y"):
        a[k][a[k] >= Lf] = 0.0
    a["fx"] = np.zeros_like(a["fx"])
    a["fy"] = np.zeros_like(a["fy"])
    r.set(a)
    mb = r.bonded()
    b = r.get()
    out.update({k: b[k] for k in ("x", "y", "type", "gid", "nxt", "mpos", "fx", "fy")})
    out["maxbond"] = np.float64(mb)
    out.update({f"t_{k}": np.asarray(v) for k, v in r.template().items()})
    out["ini"] = np.frombuffer("".join(f"{k} = {v}\n" for k, v in kv.items()).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, name), **out)


def tclust_fixture():
    """the reference's `snapcheck.py tclust` output (its printed line) on the
    reference snapshots of the run fixtures, with the snapshots' positions"""
    import contextlib
    import io
    import tempfile
    sys.path.insert(0, os.path.join(REF_ROOT, "cel", "engine", "tests"))
    import snapcheck
    out = {}
    cases = [("run_L10_seed3.npz", "snap_24"), ("run_cat_L16_seed5.npz", "snap_24"), ("run_pi_L16_seed7.npz", "snap_24"),
             ("run_extras_L10_seed4.npz", "snap_36")]
    for k, (name, key) in enumerate(cases):
        g = np.load(os.path.join(HERE, name))
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "s.bin")
            with open(path, "wb") as f:
                f.write(bytes(g[key]))
            buf = io.StringIO()
            with contextlib.redirect_stdout(buf):
                snapcheck.cmd_tclust(path)
            s = snapcheck.read_snap(path)
        out[f"c{k}_line"] = np.frombuffer(buf.getvalue().strip().encode(), np.uint8)
        out[f"c{k}_snap"] = g[key]
    np.savez_compressed(os.path.join(HERE, "tclust.npz"), **out)


# reference runs long enough to form membranes (tail aggregates of >= 12 molecules)
MEMBRANE_RUNS = [dict(lip_arch="linear", lip_nH=1, lip_nT=3, f_lip=0.3, k_angle=10, a_W_T=100),
                 dict(lip_arch="pi", lip_nT=2, lip_tie=1, f_lip=0.35, k_angle=15, a_W_T=200)]


def aggregates_fixture():
    """the reference cell detection's molecule and aggregate stages (its summary
    and per-bead aggregate index) on the reference snapshots of tclust.npz and on
    two 3000-step reference runs that form membranes"""
    import subprocess
    import tempfile
    sys.path.insert(0, os.path.join(REF_ROOT, "cel", "tools"))
    import cells
    import ocio
    g = np.load(os.path.join(HERE, "tclust.npz"))
    snaps = []
    k = 0
    while f"c{k}_snap" in g.files:
        snaps.append(bytes(g[f"c{k}_snap"]))
        k += 1
    exe = os.path.join(HERE, "..", "..", "oracle", "_ref", "oercel_portable")
    for lip in MEMBRANE_RUNS:
        kv = dict(L=24, dt=0.03, kT=1, gamma=4.5, warmup=200, f_Ka=0.0, f_Kb=0, c_N=0.05, chem=0, seed=11, threads=8,
                  steps=3000, snap_every=3000, stats_every=3000, ckpt_every=0, log_every=0, **lip)
        with tempfile.TemporaryDirectory() as td:
            ini = os.path.join(td, "p.ini")
            with open(ini, "w") as f:
                f.write("".join(f"{k_} = {v}\n" for k_, v in kv.items()))
            subprocess.run([exe, ini, os.path.join(td, "o")], check=True, capture_output=True)
            with open(os.path.join(td, "o", "snap_0000003000.bin"), "rb") as f:
                snaps.append(f.read())
    out = {}
    for k, raw in enumerate(snaps):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "s.bin")
            with open(path, "wb") as f:
                f.write(raw)
            res = cells.detect(ocio.read_snapshot(path))
        sm = res["summary"]
        for key in ("n_molecules", "n_aggregates", "n_membranes", "lipids_in_small_aggregates", "largest_aggregate"):
            out[f"c{k}_{key}"] = np.int64(sm[key])
        out[f"c{k}_bead_agg"] = np.asarray(res["bead_agg"], np.int64)
        out[f"c{k}_snap"] = np.frombuffer(raw, np.uint8)
    np.savez_compressed(os.path.join(HERE, "aggregates.npz"), **out)


# catalyst chemistry rates over 300 steps (a check every 5), compared statistically
RATES_INI = dict(L=24, dt=0.02, kT=1, gamma=4.5, warmup=50, f_lip=0.1, f_Ka=0.03, f_Kb=0.02, c_N=0.25, lip_nH=1,
                 lip_nT=3, k_angle=10, chem=1, events=1, n_chem=5, p_syn_a=0.05, p_syn_b=0.08, p_rep_a=0.03,
                 p_rep_b=0.03, mu=0.2, p_ld=0.005, p_kd=0.005, p_nd=0.004, feed="uniform", p_feed=0.01, feed_cap=0.3,
                 threads=4, steps=300, snap_every=0, stats_every=100, ckpt_every=0, log_every=0)
RATE_KINDS = ("syn", "rep", "mut", "dlip", "dK", "dN", "feed")


def catalyst_rates_fixture(seeds=(1, 2, 3, 4)):
    """the reference executable's event totals per kind (fed beads for feed)
    and final stats rows over 300 steps, for several seeds"""
    import subprocess
    import tempfile
    exe = os.path.join(HERE, "..", "..", "oracle", "_ref", "oercel_portable")
    totals = np.zeros((len(seeds), len(RATE_KINDS)), np.int64)
    finals = []
    for a, seed in enumerate(seeds):
        kv = dict(RATES_INI, seed=seed)
        with tempfile.TemporaryDirectory() as td:
            ini = os.path.join(td, "p.ini")
            with open(ini, "w") as f:
                f.write("".join(f"{k} = {v}\n" for k, v in kv.items()))
            subprocess.run([exe, ini, os.path.join(td, "o")], check=True, capture_output=True)
            with open(os.path.join(td, "o", "events.csv")) as f:
                rows = [ln.split(",") for ln in f.read().strip().split("\n")[1:]]
            with open(os.path.join(td, "o", "stats.csv")) as f:
                finals.append([float(v) for v in f.read().strip().split("\n")[-1].split(",")])
        for r in rows:
            k = RATE_KINDS.index(r[1])
            totals[a, k] += int(r[2]) if r[1] == "feed" else 1
    ini = "".join(f"{k} = {v}\n" for k, v in RATES_INI.items())
    np.savez_compressed(os.path.join(HERE, "catalyst_rates.npz"), seeds=np.array(seeds), totals=totals,
                        finals=np.array(finals), kinds=np.frombuffer(",".join(RATE_KINDS).encode(), np.uint8),
                        ini=np.frombuffer(ini.encode(), np.uint8))


def rdf_fixture():
    """the reference's `snapcheck.py rdf` output (all beads, and T beads) on the
    snapshots of aggregates.npz"""
    import contextlib
    import io
    import tempfile
    sys.path.insert(0, os.path.join(REF_ROOT, "cel", "engine", "tests"))
    import snapcheck
    g = np.load(os.path.join(HERE, "aggregates.npz"))
    out = {}
    k = 0
    while f"c{k}_snap" in g.files:
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "s.bin")
            with open(path, "wb") as f:
                f.write(bytes(g[f"c{k}_snap"]))
            for tag, typ in (("all", None), ("T", 2)):
                buf = io.StringIO()
                with contextlib.redirect_stdout(buf):
                    snapcheck.cmd_rdf([path], typ)
                out[f"c{k}_{tag}"] = np.frombuffer(buf.getvalue().encode(), np.uint8)
        k += 1
    np.savez_compressed(os.path.join(HERE, "rdf.npz"), **out)


# membrane physics of cel/engine/params/membranes.ini (tied H2T2 pi lipids, k_bond 300, dt 0.03) on a small box
MEMBRANE_INI = dict(L=24, dt=0.03, kT=1, gamma=4.5, warmup=200, f_lip=0.20, f_Ka=0.01, f_Kb=0, c_N=0.10, lip_arch="pi",
                    lip_nT=1, lip_tie=1, r0_head=0.7, k_head=0, k_bond=300, r0=0.5, k_angle=15, a_W_H=20, a_W_T=200,
                    a_H_T=50, a_W_N=45, a_H_N=22, a_T_N=120, a_W_K=45, a_H_K=30, a_T_K=200, chem=0, threads=8,
                    steps=4000, snap_every=0, stats_every=10, ckpt_every=0, log_every=0)


def membrane_stats_fixture(seeds=(5, 6)):
    """the reference executable's stats rows (T_kin, max_bond every 10 steps)
    over 4000 steps of the membrane physics, for two seeds"""
    import subprocess
    import tempfile
    exe = os.path.join(HERE, "..", "..", "oracle", "_ref", "oercel_portable")
    out = {}
    for seed in seeds:
        with tempfile.TemporaryDirectory() as td:
            ini = os.path.join(td, "p.ini")
            with open(ini, "w") as f:
                f.write("".join(f"{k} = {v}\n" for k, v in dict(MEMBRANE_INI, seed=seed).items()))
            subprocess.run([exe, ini, os.path.join(td, "o")], check=True, capture_output=True)
            with open(os.path.join(td, "o", "stats.csv")) as f:
                out[f"stats_{seed}"] = np.array([[float(v) for v in ln.split(",")]
                                                 for ln in f.read().strip().split("\n")[1:]])
    out["seeds"] = np.array(seeds)
    out["ini"] = np.frombuffer("".join(f"{k} = {v}\n" for k, v in MEMBRANE_INI.items()).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "membrane_stats.npz"), **out)


def theta_fixture():
    lib = O.Ref.lib()
    rows = []
    for seed in (0, 1, 99, 2**63 + 5):
        for step in (0, 1, 7, 12345, 2**40 + 3):
            for gi, gj in ((0, 1), (5, 9), (9, 5), (123456, 7), (2**28, 2**29 - 1)):
                rows.append((seed, step, gi, gj, lib.ref_theta(seed, step, gi, gj)))
    arr = np.array(rows, dtype=[("seed", "u8"), ("step", "i8"), ("gi", "u4"), ("gj", "u4"), ("theta", "f8")])
    np.save(os.path.join(HERE, "theta_mix13.npy"), arr)


def trajectory_fixture():
    """the reference's own primed start and 20 plain steps at L = 16 (kinetic T per step)"""
    kv = dict(CONFIG1, L=16, seed=5)
    r = O.Ref(**kv)
    r.prime()
    T = []
    for _ in range(20):
        r.run(1)
        T.append(r.kinetic_T(None, None))
    a = r.get()
    np.savez_compressed(os.path.join(HERE, "traj_L16_seed5.npz"), T=np.array(T), gid=a["gid"], x=a["x"], y=a["y"])


def stats_fixture(nsteps=10000, equil=1000, every=10):
    """time averages of the reference at configuration 1: kinetic temperature,
    conservative virial and the T-T pair histogram (64 bins on [0, 2)), with
    block standard errors (20 blocks)"""
    r = O.Ref(**CONFIG1)
    r.prime()
    r.run(equil)
    amat = np.full((8, 8), 25.0)
    for (i, j, v) in ((0, 2, 75.0), (3, 2, 75.0), (1, 2, 50.0)):
        amat[i, j] = amat[j, i] = v
    p = O.params(32.0, amat)
    T, vir, hist = [], [], []
    for _ in range((nsteps - equil) // every):
        r.run(every)
        T.append(r.kinetic_T(None, None))
        a = r.get()
        x, y = a["x"].astype(np.float32), a["y"].astype(np.float32)
        key, cs, src = O.sort(p, x, y)
        st = dict(x=x[src], y=y[src], vhx=np.zeros(len(x), np.float32), vhy=np.zeros(len(x), np.float32),
                  fx=np.zeros(len(x), np.float32), fy=np.zeros(len(x), np.float32), type=a["type"][src].copy(),
                  next=np.full(len(x), -1, np.int32))
        vir.append(O.observables(p, st, cs)["virial"])
        hist.append(O.pair_hist(p, st, cs, 2, 2, 2.0, 64))
    T, vir, hist = np.array(T), np.array(vir), np.array(hist)

    def blocks(v):
        b = np.array([c.mean(axis=0) for c in np.array_split(v, 20)])
        return v.mean(axis=0), b.std(axis=0, ddof=1) / np.sqrt(20)

    (Tm, Te), (Vm, Ve), (Hm, He) = blocks(T), blocks(vir), blocks(hist)
    np.savez_compressed(os.path.join(HERE, "stats_config1.npz"), T=Tm, T_err=Te, virial=Vm, virial_err=Ve,
                        tt_hist=Hm, tt_hist_err=He, nsteps=nsteps, equil=equil, every=every,
                        n_t=int((r.get()["type"] == 2).sum()))


RUN_INI = dict(L=10, rho=4, dt=0.02, gamma=4.5, kT=1, k_bond=100, r0=0.5, k_angle=0, lip_nH=1, lip_nT=2,
               f_lip=0.15, f_Ka=0, f_Kb=0, c_N=0.05, chem=0, events=0, warmup=8, seed=3, threads=1, steps=24,
               snap_every=12, stats_every=4, ckpt_every=24, log_every=0, a_W_H=25, a_W_T=75, a_H_T=50, a_W_N=25,
               a_H_N=25, a_N_T=75)


def run_fixture(name="run_L10_seed3.npz", **over):
    """two runs of the reference engine's executable (oracle/_ref/oercel_portable):
    a fresh soup with the repulsion warm-up for 24 steps, then a restart from its
    checkpoint to step 36.  Stores the ini, stats.csv texts, snapshots and the
    checkpoint as bytes.  `over` replaces keys of RUN_INI."""
    import subprocess
    import tempfile
    exe = os.path.join(HERE, "..", "..", "oracle", "_ref", "oercel_portable")
    with tempfile.TemporaryDirectory() as td:
        ini = os.path.join(td, "p.ini")
        text = "".join(f"{k} = {v}\n" for k, v in dict(RUN_INI, **over).items())
        with open(ini, "w") as f:
            f.write(text)
        a, b = os.path.join(td, "a"), os.path.join(td, "b")
        subprocess.run([exe, ini, a], check=True, capture_output=True)
        subprocess.run([exe, ini, b, f"restart={a}/ckpt.bin", "steps=36"], check=True, capture_output=True)

        def rd(path):
            with open(path, "rb") as f:
                return np.frombuffer(f.read(), np.uint8)

        extra = {}
        for tag, d in (("a", a), ("b", b)):
            if os.path.exists(f"{d}/events.csv"):
                extra[f"events_{tag}"] = rd(f"{d}/events.csv")
        np.savez_compressed(os.path.join(HERE, name), **extra, ini=np.frombuffer(text.encode(), np.uint8),
                            stats_a=rd(f"{a}/stats.csv"), stats_b=rd(f"{b}/stats.csv"),
                            snap_0=rd(f"{a}/snap_0000000000.bin"), snap_12=rd(f"{a}/snap_0000000012.bin"),
                            snap_24=rd(f"{a}/snap_0000000024.bin"), snap_36=rd(f"{b}/snap_0000000036.bin"),
                            ckpt_24=rd(f"{a}/ckpt.bin"))


# hand-built scenes for cell detection (cell_scenes.py): (scene, seed, k x k tiling, configuration)
CELL_CASES = [("vesicles", 1, 1, {}), ("vesicles", 2, 1, {}), ("vesicles", 3, 1, {}), ("network", 1, 1, {}),
              ("network", 2, 1, {}), ("network", 3, 1, {}), ("vesicles", 1, 2, {}),
              ("vesicles", 1, 1, dict(min_lumen_area=30.0)),
              ("vesicles", 2, 1, dict(min_exposure=0.95, leaflet_in=1.2, r_stamp=0.8)),
              ("network", 1, 1, dict(h=0.3)),
              ("vesicles", 3, 1, dict(h=0.3, pad=1.0, min_membrane_lipids=20, inner_frac_range=(0.3, 0.5))),
              ("vesicles", 1, 1, dict(min_lumen_area=30.0, inner_frac_range=(0.362, 0.62))),
              ("water", 1, 1, {}), ("micelles", 2, 1, {}), ("tiny", 3, 1, {}), ("lone", 4, 1, {}),
              ("empty", 5, 1, {})]


# reference runs that grow membranes (linear and tied pi lipids), L = 48, 30000 steps; their
# snapshots at the listed steps are the evolved cases of cells_fixture
EVOLVED_CELL_RUNS = {
    "lin48": (dict(L=48, dt=0.03, kT=1, gamma=4.5, warmup=200, f_Ka=0.0, f_Kb=0, c_N=0.05, chem=0, seed=21,
                   lip_arch="linear", lip_nH=1, lip_nT=3, f_lip=0.3, k_angle=10, a_W_T=100), (20000, 30000)),
    "pi48": (dict(L=48, dt=0.03, kT=1, gamma=4.5, warmup=200, f_Ka=0.0, f_Kb=0, c_N=0.05, chem=0, seed=22,
                  lip_arch="pi", lip_nT=2, lip_tie=1, f_lip=0.35, k_angle=15, a_W_T=200), (20000, 30000)),
}


def cells_fixture():
    """every output of the reference's cells.detect (cells with their rounding,
    label grid, per-bead maps, aggregates, summary) on the scenes of CELL_CASES
    and on snapshots of the reference engine's EVOLVED_CELL_RUNS, with the
    snapshot files it read"""
    import json
    import tempfile
    sys.path.insert(0, os.path.join(REF_ROOT, "cel", "tools"))
    import cell_scenes as cs
    import cells
    import ocio

    def js(v):
        return np.frombuffer(json.dumps(v, default=lambda o: o.item()).encode(), np.uint8)

    out = {}
    for k, (name, seed, tile, cfg) in enumerate(CELL_CASES):
        sc = cs.SCENES[name](seed)
        L = sc.L
        x, y, t, b = sc.arrays()
        if tile > 1:
            L, x, y, t, b = cs.tile(L, x, y, t, b, tile)
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "s.bin")
            cs.write_snap(path, L, x, y, t, b)
            with open(path, "rb") as f:
                raw = f.read()
            r = cells.detect(ocio.read_snapshot(path), cfg)
        out[f"c{k}_snap"] = np.frombuffer(raw, np.uint8)
        out[f"c{k}_cfg"] = js(cfg)
        out[f"c{k}_cells"] = js(r["cells"])
        out[f"c{k}_aggregates"] = js(r["aggregates"])
        out[f"c{k}_summary"] = js(r["summary"])
        out[f"c{k}_label"] = r["label"]
        for key in ("bead_cell", "mol", "bead_agg"):
            out[f"c{k}_{key}"] = np.asarray(r[key], np.int32)
        out[f"c{k}_h"] = np.float64(r["h"])
        out[f"c{k}_ng"] = np.int64(r["ng"])
        print(name, seed, tile, cfg, r["summary"], len(r["cells"]), "cells")
    import subprocess
    exe = os.path.join(HERE, "..", "..", "oracle", "_ref", "oercel_portable")
    k = len(CELL_CASES)
    for name, (kv, steps) in EVOLVED_CELL_RUNS.items():
        kv = dict(kv, threads=16, steps=max(steps), snap_every=10000, stats_every=max(steps), ckpt_every=0,
                  log_every=0)
        with tempfile.TemporaryDirectory() as td:
            ini = os.path.join(td, "p.ini")
            with open(ini, "w") as f:
                f.write("".join(f"{a} = {v}\n" for a, v in kv.items()))
            subprocess.run([exe, ini, os.path.join(td, "o")], check=True, capture_output=True)
            for st in steps:
                path = os.path.join(td, "o", f"snap_{st:010d}.bin")
                with open(path, "rb") as f:
                    raw = f.read()
                r = cells.detect(ocio.read_snapshot(path))
                out[f"c{k}_snap"] = np.frombuffer(raw, np.uint8)
                out[f"c{k}_cfg"] = js({})
                out[f"c{k}_cells"] = js(r["cells"])
                out[f"c{k}_aggregates"] = js(r["aggregates"])
                out[f"c{k}_summary"] = js(r["summary"])
                out[f"c{k}_label"] = r["label"]
                for key in ("bead_cell", "mol", "bead_agg"):
                    out[f"c{k}_{key}"] = np.asarray(r[key], np.int32)
                out[f"c{k}_h"] = np.float64(r["h"])
                out[f"c{k}_ng"] = np.int64(r["ng"])
                print(name, st, r["summary"], len(r["cells"]), "cells")
                k += 1
    np.savez_compressed(os.path.join(HERE, "cells.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) > 1:  # only the named fixtures, e.g. `make_golden.py cells`
        for name in sys.argv[1:]:
            globals()[f"{name}_fixture"]()
        sys.exit(0)
    if not O.Ref.available():
        sys.exit("oracle/_ref/libref_oercel.so is missing: run make -C oracle with the reference sources present")
    soup_fixture()
    step_fixture(12.5, 99, "step_L12p5_seed99.npz")
    step_fixture(9.0, 7, "step_L9_seed7.npz", steps=(3,))
    theta_fixture()
    trajectory_fixture()
    stats_fixture()
    run_fixture()
    run_fixture("run_extras_L10_seed4.npz", seed=4, k_angle=10, lip_nT=3, stir_A=1.0, stir_n=1, kT_amp=0.3,
                kT_period=5)
    run_fixture("run_cat_L16_seed5.npz", L=16, seed=5, chem=1, n_chem=4, events=1, nsub=1, k_angle=10, lip_nT=3,
                f_Ka=0.03, f_Kb=0.02, c_N=0.25, p_syn_a=0.3, p_syn_b=0.3, p_rep_a=0.2, p_rep_b=0.2, mu=0.2,
                p_ld=0.01, p_kd=0.01, p_nd=0.01, p_feed=0.02, feed_cap=0.27)
    # a fresh soup without warm-up at dt = 0.05: the reference sorts again before the check of step 5
    run_fixture("run_cat_resort_L16_seed5.npz", L=16, seed=5, chem=1, n_chem=1, events=1, nsub=1, k_angle=10,
                lip_nT=3, f_Ka=0.03, f_Kb=0.02, c_N=0.25, p_syn_a=0.3, p_syn_b=0.3, p_rep_a=0.2, p_rep_b=0.2, mu=0.2,
                p_ld=0.01, p_kd=0.01, p_nd=0.01, p_feed=0.02, feed_cap=0.27, warmup=0, dt=0.05)
    extras_fixture()
    template_fixture()
    mol_fixture("mol_pi_L12_seed31.npz", 31, lip_arch="pi", lip_nT=3, lip_tie=1, k_head=5, cos_head=0.1,
                r0_head=0.7)
    mol_fixture("mol_y_L12_seed32.npz", 32, lip_arch="y", lip_nT=2, lip_tie=1, k_head=3, cos_head=-0.3)
    mol_fixture("mol_bola_L12_seed33.npz", 33, lip_arch="bola", lip_nT=3, lip_tie=2, k_head=2, r0_head=0.6)
    catalyst_fixture("catalyst_pi_L16_seed14.npz", 14, 21, lip_arch="pi", lip_nT=2, lip_tie=1, k_head=5, cos_head=0.1,
                     r0_head=0.7, k_bond=300)
    # a membranes-like pi-lipid soup (tied H2T2 lipids, water-shy tails and catalysts) with catalyst chemistry
    run_fixture("run_pi_L16_seed7.npz", L=16, seed=7, chem=1, n_chem=4, events=1, nsub=1, lip_arch="pi", lip_nT=1,
                lip_tie=1, r0_head=0.7, k_bond=300, dt=0.02, f_lip=0.2, f_Ka=0.03, f_Kb=0.01, c_N=0.2, a_W_T=120,
                a_W_N=45, a_H_N=22, a_N_T=120, p_syn_a=0.3, p_syn_b=0.3, p_rep_a=0.2, p_rep_b=0.2, mu=0.2, p_ld=0.01,
                p_kd=0.01, p_nd=0.01, p_feed=0.02, feed_cap=0.25)
    catalyst_fixture("catalyst_L16_seed12.npz", 12, 21)
    catalyst_fixture("catalyst_vent_L16_seed13.npz", 13, 21, syn_nN=2, feed="vent", vent_shape="disk", vent_r=4,
                     feed_cap=0.3)
    tclust_fixture()
    aggregates_fixture()
    rdf_fixture()
    catalyst_rates_fixture()
    membrane_stats_fixture()
    cells_fixture()
    for f in sorted(os.listdir(HERE)):
        print(f, os.path.getsize(os.path.join(HERE, f)))
