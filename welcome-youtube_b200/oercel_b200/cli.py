"""Drop-in front end: `oercel_b200 params.ini outdir [key=value ...]`.

The reference engine's command line and outputs (cel/engine/oercel.c:2125-2414),
so its Python driver can run this engine in its place (`longrun.py --engine
<path>`, cel/pc/longrun.py:723; `OERCEL_ENGINE_GPU`, cel/pc/pclib.py:28):
  --params            parameter table, exit 0 (oercel.c:2107-2129)
  bad usage           usage on stderr, exit 2 (oercel.c:2130-2133)
  any error           "oercel: error: ..." on stderr, exit 1 (oercel.c:74-90)
  params.ini          every key with its value (oercel.c:626-653)
  stats.csv           step,time,T_kin,nW,nH,nT,nN,nKa,nKb,nZ,n_lipids,max_bond
  events.csv          step,kind,i,x,y,variant (kinds of the lipid chemistry:
                      grow, brk, bond; variant "-")
  snap_<step>.bin     SPEC section 5 snapshot (cel/SPEC.md:116-130)
  ckpt.bin            this engine's checkpoint (format in write_ckpt below),
                      or with ckpt_format = reference the reference's own
                      (write_reference_ckpt), which its executable continues;
                      written atomically; ckpt_keep keeps ckpt_<step>.bin
  log.txt             progress lines, "timing: ..." and "done at step N"
SIGTERM / SIGINT / walltime: finish the step, write the checkpoint, log
"stopping at step N (...)" and exit 0 (oercel.c:2376-2397).  A restart into
the same directory truncates stats.csv and events.csv after the checkpoint
step (oercel.c:2013-2034).
"""
from __future__ import annotations

import math
import os
import signal
import struct
import sys
import time

import numpy as np

from .params import ARCHS, PDEFS, ParamError, Params, param_table, parse_override, read_ini

KINDS = ("grow", "brk", "bond", "syn", "rep", "mut", "dlip", "dK", "dN", "feed")
CKPT_MAGIC = b"OCKB"
CKPT_VERSION = 2
MAX_CHUNK = 1000   # steps per engine call: bounds the signal latency and the events held on the device


class EngineError(RuntimeError):
    pass


class Log:
    def __init__(self, path):
        self.f = open(path, "a")

    def __call__(self, msg):
        sys.stdout.write(msg + "\n")
        sys.stdout.flush()
        self.f.write(msg + "\n")
        self.f.flush()


def template_bonds(state, mol):
    """gid pairs of the template bonds of every molecule (a molecule starts at a
    bead without prev and with next; its beads follow next in template order),
    ordered by the gid of the bond's first template bead, then by template order
    (write_snapshot, oercel.c:1859-1876)"""
    g = state["gid"].astype(np.int64)
    nx, pv = state["next"], state["prev"]
    heads = np.nonzero((pv < 0) & (nx >= 0))[0]
    ml = mol.mlen
    sl = np.empty((len(heads), ml), np.int64)
    sl[:, 0] = heads
    for b in range(1, ml):
        prevcol = sl[:, b - 1]
        if np.any(nx[prevcol] < 0):
            raise EngineError("broken lipid chain")
        sl[:, b] = nx[prevcol]
    keys, subs, lo, hi = [], [], [], []
    for q in range(mol.nb):
        gi, gj = g[sl[:, mol.bi[q]]], g[sl[:, mol.bj[q]]]
        keys.append(gi)
        subs.append(np.full(len(gi), q))
        lo.append(np.minimum(gi, gj))
        hi.append(np.maximum(gi, gj))
    if not keys:
        return np.zeros((0, 2), np.int32)
    keys, subs, lo, hi = (np.concatenate(a) for a in (keys, subs, lo, hi))
    order = np.lexsort((subs, keys))
    return np.stack([lo[order], hi[order]], axis=1).astype(np.int32)


def snapshot_arrays(state, mol=None):
    """the contents of a snapshot: positions and types in gid order, bonds (i < j)
    in the reference's order; mol: the template of branched lipids (their
    bonds), None for linear chains"""
    n = len(state["x"])
    g = state["gid"].astype(np.int64)
    x = np.empty(n, np.float32)
    y = np.empty(n, np.float32)
    t = np.empty(n, np.uint8)
    x[g], y[g], t[g] = state["x"], state["y"], state["type"]
    if mol is not None:
        bonds = template_bonds(state, mol)
    else:
        nx = state["next"]
        has = nx >= 0
        gi, gj = g[has], g[nx[has]]
        order = np.lexsort((gj, gi))  # by the bond's chain-side (prev) bead, as the reference orders by template start
        lo, hi = np.minimum(gi, gj)[order], np.maximum(gi, gj)[order]
        bonds = np.stack([lo, hi], axis=1).astype(np.int32)
    return x, y, t, bonds


def write_snapshot(path, state, step, time_, L, mol=None):
    """SPEC section 5: OCEL v1, positions and types in gid order, bonds (i < j);
    mol: the template of branched lipids (their bonds), None for linear chains"""
    x, y, t, bonds = snapshot_arrays(state, mol)
    n = len(t)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(b"OCEL")
        f.write(struct.pack("<iiiqdd", 1, n, len(bonds), int(step), float(time_), float(L)))
        f.write(x.tobytes())
        f.write(y.tobytes())
        f.write(t.tobytes())
        f.write(bonds.tobytes())
    os.replace(tmp, path)


def read_snapshot(path):
    with open(path, "rb") as f:
        b = f.read()
    if b[:4] != b"OCEL":
        raise ValueError(f"{path} is not a snapshot")
    ver, n, nb, step, time_, L = struct.unpack_from("<iiiqdd", b, 4)
    o = 4 + struct.calcsize("<iiiqdd")
    x = np.frombuffer(b, np.float32, n, o)
    y = np.frombuffer(b, np.float32, n, o + 4 * n)
    t = np.frombuffer(b, np.uint8, n, o + 8 * n)
    bonds = np.frombuffer(b, np.int32, 2 * nb, o + 9 * n).reshape(nb, 2)
    return dict(version=ver, N=n, step=step, time=time_, L=L, x=x, y=y, type=t, bonds=bonds)


CKPT_HEAD = "<iiqddQqdqd"


def write_ckpt(path, st, step, time_, L, seed, warm_end, anchor, keep_copy=None, rng=None):
    """OCKB v2 (little endian): magic, int32 version, int32 N, int64 step,
    float64 time, float64 L, uint64 seed, int64 warm_end, float64 t_anchor,
    int64 step_anchor, float64 dt_anchor (time = t_anchor + (step -
    step_anchor) dt while dt = dt_anchor, oercel.c:1984-1985), uint64 rng[4]
    (the serial generator of the catalyst chemistry), then in slot order
    uint32 gid[N], uint8 type[N], int32 prev[N], int32 next[N], float32
    x, y, vhx, vhy, fx, fy [N each], "END!".  Written to a temporary file,
    synced and renamed (oercel.c:1891-1936)."""
    n = len(st["x"])
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(CKPT_MAGIC)
        f.write(struct.pack(CKPT_HEAD, CKPT_VERSION, n, int(step), float(time_), float(L), int(seed) & (2**64 - 1),
                            int(warm_end), float(anchor[0]), int(anchor[1]), float(anchor[2])))
        f.write(np.ascontiguousarray(np.zeros(4, np.uint64) if rng is None else rng, np.uint64).tobytes())
        for k, dt in (("gid", np.uint32), ("type", np.uint8), ("prev", np.int32), ("next", np.int32)):
            f.write(np.ascontiguousarray(st[k], dt).tobytes())
        for k in ("x", "y", "vhx", "vhy", "fx", "fy"):
            f.write(np.ascontiguousarray(st[k], np.float32).tobytes())
        f.write(b"END!")
        f.flush()
        os.fsync(f.fileno())
    if keep_copy:
        try:
            os.link(tmp, keep_copy)
        except OSError:
            pass
    os.replace(tmp, path)


REF_CKPT_MAGIC = b"OCKP"


def reference_mpos(st, mlen, nH):
    """The reference's per-bead template position (mpos, oercel.c:800-806) from
    this engine's prev/next links: every H and T bead must sit in a chain of
    exactly mlen beads whose k-th bead is an H for k < nH and a T after, and no
    other bead may be linked.  Anything else (chains grown or cut by the lipid
    chemistry, free H or T beads) has no form in the reference's checkpoint:
    EngineError."""
    prev, nxt, ty = st["prev"], st["next"], st["type"]
    n = len(ty)
    mpos = np.full(n, -1, np.int8)
    lipid = (ty == 1) | (ty == 2)
    linked = (prev >= 0) | (nxt >= 0)
    if np.any(linked & ~lipid):
        raise EngineError("a bead other than H or T is bonded: not representable in the reference checkpoint")
    for h in np.nonzero((prev < 0) & (nxt >= 0))[0]:
        c, k = h, 0
        while c >= 0:
            if k >= mlen or ty[c] != (1 if k < nH else 2):
                raise EngineError("a chain does not match the lipid template (grown or cut by the lipid chemistry): "
                                  "not representable in the reference checkpoint")
            mpos[c] = k
            c = nxt[c]
            k += 1
        if k != mlen:
            raise EngineError(f"a chain of {k} beads (the template has {mlen}): not representable in the reference "
                              f"checkpoint")
    if np.any(lipid & (mpos < 0)):
        raise EngineError("a free H or T bead: not representable in the reference checkpoint")
    return mpos


def reference_order(x, y, L, nsub):
    """the slot order the reference engine keeps: a stable sort by its cell
    (floor(L) columns, floor(L) nsub rows, column-major, the index products in
    FP64; cell_of_pos / sort_cells, oercel.c:739-745,779-786,832-933)"""
    ncx = int(math.floor(L))
    ncy = ncx * int(nsub)
    cx = np.minimum((np.asarray(x, np.float64) * (ncx / L)).astype(np.int64), ncx - 1)
    cy = np.minimum((np.asarray(y, np.float64) * (ncy / L)).astype(np.int64), ncy - 1)
    return np.argsort(np.maximum(cx, 0) * ncy + np.maximum(cy, 0), kind="stable")


def write_reference_ckpt(path, st, step, time_, L, seed, warm_end, anchor, rng, maxbond, soup_seed, mlen, nH, arch,
                         nsub, keep_copy=None):
    """The reference engine's checkpoint (write_ckpt, oercel.c:1891-1936),
    version 2 for linear lipids and 3 (with the shape code) otherwise, so that
    its executable can continue this run: little endian "OCKP", int32 version,
    N, mlen, nH, [arch], int64 step, float64 time, L, uint64 seed, rng[4],
    float64 maxbond, int64 warm_end, float64 t_anchor, int64 step_anchor,
    float64 dt_anchor, uint64 soup_seed, then in slot order uint32 gid, uint8
    type, int8 mpos, int32 nxt, float64 x, y, vx, vy, fx, fy (the FP32 state
    widened; vx/vy the stored half-step velocity), "END!".  The beads are
    written in the reference's own slot order (reference_order, with the
    nsub of the run): its restart sorts the state once more but leaves the
    forces where they are (sort_cells permutes every array except fx, fy), so
    the file must already be in the order that sort keeps.  Written to a
    temporary file, synced and renamed."""
    n = len(st["x"])
    if np.any(st["type"] >= 6):
        raise EngineError("bead type Z or above: not representable in the reference checkpoint")
    mpos = reference_mpos(st, mlen, nH)
    perm = reference_order(st["x"], st["y"], float(L), nsub)
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    nx = np.asarray(st["next"], np.int64)[perm]
    nxt = np.where(nx >= 0, inv[np.maximum(nx, 0)], -1).astype(np.int32)
    st = {k: np.asarray(st[k])[perm] for k in ("gid", "type", "x", "y", "vhx", "vhy", "fx", "fy")}
    mpos = mpos[perm]
    ver = 2 if arch == 0 else 3
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(REF_CKPT_MAGIC)
        f.write(struct.pack("<iiii", ver, n, int(mlen), int(nH)))
        if ver == 3:
            f.write(struct.pack("<i", int(arch)))
        f.write(struct.pack("<qddQ", int(step), float(time_), float(L), int(seed) & (2**64 - 1)))
        f.write(np.ascontiguousarray(rng, np.uint64).tobytes())
        f.write(struct.pack("<dqdqdQ", float(maxbond), int(warm_end), float(anchor[0]), int(anchor[1]),
                            float(anchor[2]), int(soup_seed) & (2**64 - 1)))
        f.write(np.ascontiguousarray(st["gid"], np.uint32).tobytes())
        f.write(np.ascontiguousarray(st["type"], np.uint8).tobytes())
        f.write(mpos.tobytes())
        f.write(nxt.tobytes())
        for k in ("x", "y", "vhx", "vhy", "fx", "fy"):
            f.write(np.ascontiguousarray(st[k], np.float64).tobytes())
        f.write(b"END!")
        f.flush()
        os.fsync(f.fileno())
    if keep_copy:
        try:
            os.link(tmp, keep_copy)
        except OSError:
            pass
    os.replace(tmp, path)


def read_ckpt(path):
    with open(path, "rb") as f:
        b = f.read()
    if b[:4] == b"OCKP":
        return read_reference_ckpt(path, b)
    if b[:4] != CKPT_MAGIC:
        raise EngineError(f"{path} is not an oercel_b200 checkpoint")
    ver, n, step, time_, L, seed, warm_end, ta, sa, da = struct.unpack_from(CKPT_HEAD, b, 4)
    if ver not in (1, 2):
        raise EngineError(f"unsupported checkpoint version {ver}")
    o = 4 + struct.calcsize(CKPT_HEAD)
    out = dict(N=n, step=step, time=time_, L=L, seed=seed, warm_end=warm_end, anchor=(ta, sa, da),
               rng=np.zeros(4, np.uint64))
    if ver >= 2:
        out["rng"] = np.frombuffer(b, np.uint64, 4, o).copy()
        o += 32
    for k, dt in (("gid", np.uint32), ("type", np.uint8), ("prev", np.int32), ("next", np.int32)):
        a = np.frombuffer(b, dt, n, o)
        out[k] = a.copy()
        o += n * np.dtype(dt).itemsize
    for k in ("x", "y", "vhx", "vhy", "fx", "fy"):
        out[k] = np.frombuffer(b, np.float32, n, o).copy()
        o += 4 * n
    if b[o:o + 4] != b"END!":
        raise EngineError("checkpoint truncated (end marker missing)")
    return out


def read_reference_ckpt(path, b):
    """the reference engine's checkpoint, version 2 (linear lipids) or 3 (the
    same with the lipid shape code after nH; layout of write_ckpt,
    oercel.c:1891-1936): continue a reference run on the GPU.  The FP64 state
    is rounded to FP32; prev links are the inverse of nxt."""
    ver, n, ml, nh = struct.unpack_from("<iiii", b, 4)
    if ver not in (2, 3):
        raise EngineError(f"{path}: reference checkpoint version {ver} (versions 2 and 3 are read)")
    arch, o0 = (struct.unpack_from("<i", b, 20)[0], 24) if ver == 3 else (0, 20)
    step, time_, L, seed = struct.unpack_from("<qddQ", b, o0)
    rng = np.frombuffer(b, np.uint64, 4, o0 + 32).copy()
    o = o0 + 32 + 32 + 8          # rng state, maxbond
    warm_end, ta, sa, da, soup_seed = struct.unpack_from("<qdqdQ", b, o)
    o += 32 + 8                   # warm_end, anchors, soup seed
    gid = np.frombuffer(b, np.uint32, n, o).copy()
    o += 4 * n
    typ = np.frombuffer(b, np.uint8, n, o).copy()
    o += 2 * n                    # type, then mpos
    nxt = np.frombuffer(b, np.int32, n, o).copy()
    o += 4 * n
    out = dict(N=n, step=step, time=time_, L=L, seed=seed, warm_end=warm_end, anchor=(ta, sa, da), gid=gid,
               type=typ, next=nxt, rng=rng, arch=arch, mlen=ml, nH=nh, soup_seed=soup_seed)
    for k, ref in (("x", "x"), ("y", "y"), ("vhx", "vx"), ("vhy", "vy"), ("fx", "fx"), ("fy", "fy")):
        out[k] = np.frombuffer(b, np.float64, n, o).astype(np.float32)
        o += 8 * n
    if b[o:o + 4] != b"END!":
        raise EngineError("checkpoint end marker missing")
    if np.any(typ >= 6):
        raise EngineError(f"{path}: bead type Z is not used (SPEC section 6)")
    Lf = np.float32(L)
    for k in ("x", "y"):
        out[k][out[k] >= Lf] = np.float32(0.0)
    prev = np.full(n, -1, np.int32)
    has = nxt >= 0
    prev[nxt[has]] = np.nonzero(has)[0].astype(np.int32)
    out["prev"] = prev
    return out


def truncate_csv_after(path, step):
    """drop rows after `step` and any partial last line (oercel.c:2013-2034)"""
    if not os.path.exists(path):
        return
    with open(path, "rb") as f:
        data = f.read()
    lines = data.split(b"\n")
    keep, first = [], True
    for ln in lines[:-1]:
        if not first:
            try:
                if int(ln.split(b",", 1)[0]) > step:
                    break
            except ValueError:
                break
        keep.append(ln)
        first = False
    with open(path, "wb") as f:
        f.write(b"".join(l + b"\n" for l in keep))


def stats_row(step, t, o, maxbond):
    """one stats.csv row; the fresh start's row prints its time as "0" (oercel.c:2280)"""
    c = o["counts"]
    ts = "0" if step == 0 and t == 0.0 else f"{t:.6f}"
    return (f"{step},{ts},{o['T']:.6f},{c[0]},{c[1]},{c[2]},{c[3]},{c[4]},{c[5]},{c[6]},{o['n_chains']},"
            f"{maxbond:.6f}\n")


def run(argv):
    if len(argv) == 2 and argv[1] == "--params":
        print(param_table())
        return 0
    if len(argv) < 3:
        sys.stderr.write(f"usage: {argv[0]} params.ini outdir [key=value ...]\n       {argv[0]} --params   "
                         "(print all parameters)\n")
        return 2
    ini, outdir, over = argv[1], argv[2], argv[3:]
    try:
        p = Params()
        p.update(read_ini(ini) + [parse_override(o) for o in over])
        p.validate()
    except (ParamError, OSError) as e:
        sys.stderr.write(f"oercel: error: {e}\n")
        return 1
    if not p.restart and p.init != "soup":
        sys.stderr.write(f"oercel: error: init = {p.init} needs restart = <checkpoint>\n")
        return 1
    try:
        return _run(p, outdir, over)
    except (EngineError, ParamError) as e:
        sys.stderr.write(f"oercel: error: {e}\n")
        return 1


def _run(p, outdir, over):
    from . import Engine, soup_for
    from ._capi import DpdError
    os.makedirs(outdir, exist_ok=True)
    log = Log(os.path.join(outdir, "log.txt"))
    stop = {"flag": None}

    def on_sig(sig, frame):
        stop["flag"] = "signal"

    signal.signal(signal.SIGTERM, on_sig)
    signal.signal(signal.SIGINT, on_sig)
    t_start = time.time()
    restarting = bool(p.restart)
    try:
        if restarting:
            ck = read_ckpt(p.restart)
            if abs(ck["L"] - p.L) > 1e-12:
                raise EngineError(f"checkpoint L={ck['L']:g} differs from parameter L={p.L:g}")
            if "arch" in ck and (ck["arch"] != ARCHS.index(p.lip_arch) or ck["mlen"] != p.mlen()):
                raise EngineError("checkpoint lipid architecture differs from parameters")
            seed = p.seed if p.restart_reseed else ck["seed"]
            if p.restart_reseed:
                log(f"restart: reseeded with seed={p.seed} (branch, not an exact continuation)")
            elif seed != p.seed:
                log(f"note: using checkpoint seed {seed} (ini seed {p.seed} ignored; set restart_reseed=1 to branch)")
            warm_end = ck["warm_end"]
            soup_seed = ck.get("soup_seed", ck["seed"])
            ta, sa, da = ck["anchor"]
            anchor = (ta, sa, da) if da == p.dt else (ck["time"], ck["step"], p.dt)  # dt changed: new anchor
            e = Engine(p, n_beads=ck["N"])
            # the checkpoint's seed (unless restart_reseed), warm-up end and time anchor (oercel.c:1965-1990)
            e.set_params(0, p, seed=seed, warm_end=warm_end, t_anchor=anchor[0], step_anchor=anchor[1])
            e.set_state(0, ck["x"], ck["y"], ck["vhx"], ck["vhy"], ck["type"], ck["gid"], ck["prev"], ck["next"])
            e.set_dynamics(0, ck["vhx"], ck["vhy"], ck["fx"], ck["fy"])
            # the serial generator: the checkpoint's, or reseeded for a branch (oercel.c:2177-2180)
            e.set_rng(0, reseeded_rng(p.seed, ck["step"]) if p.restart_reseed else ck["rng"])
            e.resume()
            e.set_step(ck["step"])
            log(f"restart from {p.restart} at step {ck['step']} (t={ck['time']:.4f}), N={ck['N']}")
        else:
            e = Engine(p)
            s = soup_for(p)
            e.set_state(0, s["x"], s["y"], s["vx"], s["vy"], s["type"], None, s["prev"], s["next"])
            e.set_rng(0, s["rng"])
            e.prime()
            warm_end, seed, anchor = p.warmup, p.seed, (0.0, 0, p.dt)
            soup_seed = p.seed
            log(f"init soup: N={len(s['x'])} lipid beads={s['n_lipid_beads']}")
    except DpdError as err:
        raise EngineError(str(err)) from None
    step0 = e.step_no
    n = e.n_beads[0]
    L = float(p.L)
    mol = p.template() if p.lip_arch != "linear" else None  # the bonds of branched lipids in snapshots
    # params.ini (keep the previous one if a restart changed the parameters)
    pp = os.path.join(outdir, "params.ini")
    newp = pp + ".new"
    p.write(newp, over)
    if restarting and os.path.exists(pp) and open(pp).read() != open(newp).read():
        os.replace(pp, os.path.join(outdir, f"params_before_{step0:010d}.ini"))
    os.replace(newp, pp)
    spath, epath = os.path.join(outdir, "stats.csv"), os.path.join(outdir, "events.csv")
    if restarting and os.path.exists(spath):
        truncate_csv_after(spath, step0)
        sf = open(spath, "a")
    else:
        sf = open(spath, "w")
        sf.write("step,time,T_kin,nW,nH,nT,nN,nKa,nKb,nZ,n_lipids,max_bond\n")
    ef = None
    if p.events:
        if restarting and os.path.exists(epath):
            truncate_csv_after(epath, step0)
            ef = open(epath, "a")
        else:
            ef = open(epath, "w")
            ef.write("step,kind,i,x,y,variant\n")
    nc = int(math.floor(L))
    log(f"oercel_b200: N={n} L={p.L:g} cells={nc}x{nc} dt={p.dt:g} gamma={p.gamma:g} sigma={p.sigma():g} "
        f"steps->{p.steps}")

    def kT_at(t):
        return p.kT + (p.kT_amp * math.sin(2.0 * math.pi * t / p.kT_period) if p.kT_amp != 0 else 0.0)

    def tnow(step):
        return anchor[0] + (step - anchor[1]) * p.dt

    def write_events():
        if ef is None:
            e.events()
            return
        rows = sorted(e.events(), key=lambda r: r[:4])
        for (st, k, g, pg, x, y, _) in rows:
            var = "-" if k < 3 else {0: "a", 1: "b"}.get(pg, "-")  # the reference's variant column
            xy = "nan,nan" if math.isnan(x) else f"{x:.4f},{y:.4f}"
            ef.write(f"{st},{KINDS[k]},{g},{xy},{var}\n")
        ef.flush()

    def ckpt(step):
        st = e.state(0)
        keep = os.path.join(outdir, f"ckpt_{step:010d}.bin") if p.ckpt_keep else None
        path = os.path.join(outdir, "ckpt.bin")
        if p.ckpt_format == "reference":
            obs()  # the device's running max bond, folded into the row's maximum
            t = p.template()
            write_reference_ckpt(path, st, step, tnow(step), L, seed, warm_end, anchor, e.rng(0), mb["acc"],
                                 soup_seed, t.mlen, t.nH, ARCHS.index(p.lip_arch), p.nsub, keep)
        else:
            write_ckpt(path, st, step, tnow(step), L, seed, warm_end, anchor, keep, e.rng(0))

    # max_bond of a stats row is the largest bond length since the previous row
    # (oercel.c:2365-2369); every device read restarts the device maximum
    mb = {"acc": 0.0}

    def obs():
        o = e.observables(0, virial=False)
        mb["acc"] = max(mb["acc"], o["maxbond"])
        return o

    def stats(step):
        o = obs()
        sf.write(stats_row(step, tnow(step), o, mb["acc"]))
        mb["acc"] = 0.0
        return o

    if not restarting:
        if p.stats_every > 0:
            stats(0)
        if p.snap_every > 0:
            write_snapshot(os.path.join(outdir, f"snap_{0:010d}.bin"), e.state(0), 0, 0.0, L, mol)
    elif p.snap_every > 0 and step0 % p.snap_every == 0:
        sp = os.path.join(outdir, f"snap_{step0:010d}.bin")
        if not os.path.exists(sp):
            write_snapshot(sp, e.state(0), step0, tnow(step0), L, mol)
    step = step0
    t_loop = time.time()
    t_last, step_last = t_loop, step
    stopped = None
    while step < p.steps:
        marks = [p.steps, step + MAX_CHUNK]
        for every in (p.stats_every, p.snap_every, p.ckpt_every, p.log_every):
            if every > 0:
                marks.append((step // every + 1) * every)
        nxt = min(marks)
        try:
            e.step(nxt - step)
        except DpdError as err:
            raise EngineError(f"{err} (near step {nxt})") from None
        step = nxt
        write_events()
        if p.stats_every > 0 and step % p.stats_every == 0:
            o = stats(step)
            if not math.isfinite(o["T"]):
                raise EngineError(f"non-finite temperature at step {step}")
        if p.snap_every > 0 and step % p.snap_every == 0:
            write_snapshot(os.path.join(outdir, f"snap_{step:010d}.bin"), e.state(0), step, tnow(step), L, mol)
        if stop["flag"] is None and p.walltime > 0 and time.time() - t_start > p.walltime:
            stop["flag"] = "walltime"
        if (p.ckpt_every > 0 and step % p.ckpt_every == 0) or stop["flag"] or step >= p.steps:
            sf.flush()
            ckpt(step)
        if p.log_every > 0 and step % p.log_every == 0:
            o = obs()
            now = time.time()
            c = o["counts"]
            log(f"step {step} t={tnow(step):.2f} T={o['T']:.4f} (kT={kT_at(tnow(step)):.4f}) p=({o['px']:.2e},{o['py']:.2e}) "
                f"lip={o['n_chains']} Ka={c[4]} Kb={c[5]} N={c[3]}  "
                f"{1e3 * (now - t_last) / max(step - step_last, 1):.3f} ms/step")
            t_last, step_last = now, step
        if stop["flag"]:
            stopped = stop["flag"]
            log(f"stopping at step {step} ({stopped}), checkpoint written")
            break
    sf.close()
    if ef:
        ef.close()
    nst = step - step0
    if nst > 0:
        ms = 1e3 * (time.time() - t_loop) / nst
        log(f"timing: {nst} steps, {ms:.4f} ms/step (GPU step incl. outputs)")
    log(f"done at step {step}" + (" (stopped early; restart to continue)" if stopped else ""))
    e.close()
    return 0


def _mix13(z):
    m = (1 << 64) - 1
    z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & m
    z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & m
    return z ^ (z >> 31)


def reseeded_rng(seed, step):
    """rng_seed(seed ^ mix13(step)) of a branching restart (oercel.c:143-174, 2177-2180)"""
    m = (1 << 64) - 1
    z = (int(seed) ^ _mix13(int(step) & m)) & m
    out = []
    for _ in range(4):
        z = (z + 0x9e3779b97f4a7c15) & m
        out.append(_mix13(z))
    return np.array(out, np.uint64)


def main():
    sys.exit(run(sys.argv))


if __name__ == "__main__":
    main()
