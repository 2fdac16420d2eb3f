"""ctypes front end of the CPU checker (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (the restatement in ``dpd_oracle.c``) and, when it
was built, ``oracle/_ref/libref_oercel.so`` (the reference engine's own routines
from ``cel/engine/oercel.c``).  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` import this module; the product package
never does.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_oercel.so")
MAXT = 8

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")


class OraParams(C.Structure):
    _fields_ = [("L", C.c_double), ("ncx", C.c_int32), ("ncy", C.c_int32),
                ("icsx", C.c_double), ("icsy", C.c_double),
                ("dt", C.c_double), ("lam", C.c_double), ("gamma", C.c_double), ("kT", C.c_double),
                ("a", C.c_double * (MAXT * MAXT)), ("k_bond", C.c_double), ("r0", C.c_double),
                ("seed", C.c_uint64), ("noise", C.c_int32), ("pad", C.c_int32),
                ("k_angle", C.c_double), ("stir_A", C.c_double), ("stir_n", C.c_int32), ("pad2", C.c_int32),
                ("kT_amp", C.c_double), ("kT_period", C.c_double), ("t_anchor", C.c_double),
                ("step_anchor", C.c_int64)]


class OraF32(C.Structure):
    _fields_ = [("dt", C.c_float), ("dt2", C.c_float), ("cvt", C.c_float), ("L", C.c_float)]


class OraChem(C.Structure):
    _fields_ = [("thr_break", C.c_uint32), ("thr_grow", C.c_uint32), ("thr_bond", C.c_uint32),
                ("r2_grow", C.c_float), ("r2_bond", C.c_float), ("n_t_min", C.c_int32),
                ("max_chain", C.c_int32)]


class OraCat(C.Structure):
    _fields_ = [("r_cat", C.c_double), ("syn_tries", C.c_int32), ("syn_relax", C.c_int32), ("syn_nN", C.c_int32),
                ("nH", C.c_int32), ("nT", C.c_int32), ("feed_mode", C.c_int32), ("vent_kind", C.c_int32),
                ("pad", C.c_int32), ("p_syn_a", C.c_double), ("p_syn_b", C.c_double), ("p_rep_a", C.c_double),
                ("p_rep_b", C.c_double), ("mu", C.c_double), ("p_ld", C.c_double), ("p_kd", C.c_double),
                ("p_nd", C.c_double), ("p_feed", C.c_double), ("feed_cap", C.c_double), ("vent_x", C.c_double),
                ("vent_y", C.c_double), ("vent_r", C.c_double), ("vent_w", C.c_double)]


class OraEvent(C.Structure):
    _fields_ = [("step", C.c_int64), ("kind", C.c_int32), ("gid", C.c_uint32), ("partner", C.c_uint32),
                ("x", C.c_float), ("y", C.c_float), ("pad", C.c_int32)]


def build():
    """Compile the checker (and the reference shim when the sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER(OraParams)
    lib.ora_philox4x32_10.argtypes = [u32p, u32p, u32p]
    lib.ora_philox_word.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int64]
    lib.ora_philox_word.restype = C.c_uint32
    lib.ora_mix13.argtypes = [C.c_uint64]
    lib.ora_mix13.restype = C.c_uint64
    lib.ora_step_seed.argtypes = [C.c_uint64, C.c_int64]
    lib.ora_step_seed.restype = C.c_uint64
    lib.ora_theta.argtypes = [P, C.c_int64, C.c_uint32, C.c_uint32]
    lib.ora_theta.restype = C.c_double
    lib.ora_theta_matrix.argtypes = [P, C.c_int64, C.c_int, C.c_void_p, C.c_void_p]
    lib.ora_theta_matrix.restype = None
    lib.ora_decision_word.argtypes = [C.c_uint64, C.c_int64, C.c_uint32, C.c_uint32]
    lib.ora_decision_word.restype = C.c_uint32
    lib.ora_cell_of.argtypes = [P, C.c_float, C.c_float]
    lib.ora_cell_of.restype = C.c_int32
    lib.ora_sort.argtypes = [P, C.c_int32, f32p, f32p, i32p, i32p, i32p]
    lib.ora_stir_forces.argtypes = [P, C.c_int32, f32p, f64p]
    u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
    lib.ora_catalyst_chemistry.argtypes = [P, C.POINTER(OraCat), u64p, C.c_int32, f32p, f32p, f32p, f32p, f32p,
                                           f32p, u8p, u32p, i32p, i32p, i32p, C.c_int64, C.POINTER(OraEvent),
                                           C.c_int32, C.POINTER(C.c_int32)]
    lib.ora_catalyst_chemistry.restype = C.c_int32
    lib.ora_sdt_at.argtypes = [P, C.c_int64]
    lib.ora_sdt_at.restype = C.c_double
    lib.ora_pair_forces.argtypes = [P, C.c_int32, f32p, f32p, f32p, f32p, u8p, u32p, i32p, C.c_int64, C.c_int32,
                                    f64p, f64p]
    lib.ora_pair_forces_brute.argtypes = [P, C.c_int32, f32p, f32p, f32p, f32p, u8p, u32p, C.c_int64, C.c_int32,
                                          f64p, f64p]
    lib.ora_bond_forces.argtypes = [P, C.c_int32, f32p, f32p, i32p, f64p, f64p, C.POINTER(C.c_double)]
    lib.ora_mol_forces.argtypes = [P, C.POINTER(OraMol), C.c_int32, f32p, f32p, i32p, f64p, f64p,
                                   C.POINTER(C.c_double)]
    lib.ora_integrate_f32.argtypes = [C.POINTER(OraF32), C.c_int32, f32p, f32p, f32p, f32p, f32p, f32p, f32p, f32p]
    lib.ora_integrate_f32.restype = C.c_int32
    lib.ora_integrate_f64.argtypes = [P, C.c_int32, f64p, f64p, f64p, f64p, f64p, f64p, f64p, f64p]
    lib.ora_chemistry.argtypes = [P, C.POINTER(OraChem), C.c_int32, f32p, f32p, u8p, u32p, i32p, i32p, i32p,
                                  C.c_int64, C.POINTER(OraEvent), C.c_int32]
    lib.ora_chemistry.restype = C.c_int32
    lib.ora_observables.argtypes = [P, C.c_int32, f32p, f32p, f32p, f32p, f32p, f32p, u8p, i32p, i32p, f64p]
    lib.ora_pair_hist.argtypes = [P, C.c_int32, f32p, f32p, u8p, i32p, C.c_int32, C.c_int32, C.c_double,
                                  C.c_int32, f64p]
    lib.ora_init_soup.argtypes = [C.c_double, C.c_int32, C.c_uint64, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                  C.c_double, C.c_double, C.c_double, C.c_double, f64p, f64p, f64p, f64p, u8p, u32p,
                                  i32p, i32p]
    lib.ora_init_soup.restype = C.c_int32
    lib.ora_sdt.argtypes = [P]
    lib.ora_sdt.restype = C.c_double
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def params(L, amat, *, dt=0.02, lam=0.65, gamma=4.5, kT=1.0, k_bond=100.0, r0=0.5, seed=0, noise=0, k_angle=0.0,
           stir_A=0.0, stir_n=1, kT_amp=0.0, kT_period=1000.0, t_anchor=0.0, step_anchor=0):
    """Oracle parameter block; amat is a square array of up to 8x8 repulsions."""
    p = OraParams()
    p.k_angle, p.stir_A, p.stir_n = float(k_angle), float(stir_A), int(stir_n)
    p.kT_amp, p.kT_period, p.t_anchor, p.step_anchor = float(kT_amp), float(kT_period), float(t_anchor), int(step_anchor)
    p.L = float(L)
    p.ncx = p.ncy = int(math.floor(L))
    p.icsx = p.ncx / p.L
    p.icsy = p.ncy / p.L
    p.dt, p.lam, p.gamma, p.kT = dt, lam, gamma, kT
    a = np.zeros((MAXT, MAXT))
    am = np.asarray(amat, dtype=np.float64)
    a[: am.shape[0], : am.shape[1]] = am
    for k, v in enumerate(a.ravel()):
        p.a[k] = v
    p.k_bond, p.r0, p.seed, p.noise = k_bond, r0, seed, noise
    return p


def theta_matrix(p, step, gid):
    """theta of every pair of the beads with these gids at one step (n x n, zero diagonal)"""
    g = np.ascontiguousarray(gid, np.uint32)
    out = np.empty((len(g), len(g)), np.float64)
    lib().ora_theta_matrix(C.byref(p), int(step), len(g), g.ctypes.data, out.ctypes.data)
    return out


def f32consts(p):
    c = OraF32()
    c.dt = np.float32(p.dt)
    c.dt2 = np.float32(p.dt * p.dt)
    c.cvt = np.float32((0.5 + p.lam) * p.dt)
    c.L = np.float32(p.L)
    return c


def chem(p_break=1e-5, p_grow=1e-3, p_bond=1e-2, r_grow=1.0, r_bond=0.6, n_t_min=2, max_chain=12):
    c = OraChem()
    c.thr_break, c.thr_grow, c.thr_bond = (threshold(p_break), threshold(p_grow), threshold(p_bond))
    c.r2_grow = np.float32(r_grow * r_grow)
    c.r2_bond = np.float32(r_bond * r_bond)
    c.n_t_min, c.max_chain = n_t_min, max_chain
    return c


def threshold(p):
    """decision threshold: an event happens when the 32-bit draw u < thr = floor(p * 2^32)"""
    return int(min(max(math.floor(p * 4294967296.0), 0), 0xFFFFFFFF))


def sort(p, x, y):
    n = len(x)
    key = np.empty(n, np.int32)
    cstart = np.empty(p.ncx * p.ncy + 1, np.int32)
    src = np.empty(n, np.int32)
    lib().ora_sort(C.byref(p), n, np.ascontiguousarray(x, np.float32), np.ascontiguousarray(y, np.float32),
                   key, cstart, src)
    return key, cstart, src


def pair_forces(p, st, cstart, step, noise=True):
    n = len(st["x"])
    fx = np.zeros(n)
    fy = np.zeros(n)
    lib().ora_pair_forces(C.byref(p), n, st["x"], st["y"], st["vtx"], st["vty"], st["type"], st["gid"], cstart,
                          step, int(noise), fx, fy)
    return fx, fy


def pair_forces_brute(p, st, step, noise=True):
    n = len(st["x"])
    fx = np.zeros(n)
    fy = np.zeros(n)
    lib().ora_pair_forces_brute(C.byref(p), n, st["x"], st["y"], st["vtx"], st["vty"], st["type"], st["gid"],
                                step, int(noise), fx, fy)
    return fx, fy


def bond_forces(p, st, fx=None, fy=None):
    n = len(st["x"])
    fx = np.zeros(n) if fx is None else fx
    fy = np.zeros(n) if fy is None else fy
    mb = C.c_double(0.0)
    lib().ora_bond_forces(C.byref(p), n, st["x"], st["y"], st["next"], fx, fy, C.byref(mb))
    return fx, fy, mb.value


class OraMol(C.Structure):
    _fields_ = [("mlen", C.c_int32), ("nb", C.c_int32), ("na", C.c_int32), ("pad", C.c_int32),
                ("bi", C.c_int32 * 32), ("bj", C.c_int32 * 32), ("br0", C.c_double * 32), ("ai", C.c_int32 * 32),
                ("aj", C.c_int32 * 32), ("ak", C.c_int32 * 32), ("akind", C.c_int32 * 32), ("aK", C.c_double * 32),
                ("ac0", C.c_double * 32)]


def mol(t):
    """oracle template from a dict of template fields (as Ref.template() gives)"""
    m = OraMol()
    m.mlen, m.nb, m.na = int(t["mlen"]), int(t["nb"]), int(t["na"])
    for key in ("bi", "bj", "br0", "ai", "aj", "ak", "akind", "aK", "ac0"):
        arr = getattr(m, key)
        for q, v in enumerate(t[key]):
            arr[q] = v
    return m


def mol_forces(p, m, st, fx=None, fy=None):
    """bonded forces of branched lipids (template m) added to fx, fy"""
    n = len(st["x"])
    fx = np.zeros(n) if fx is None else fx
    fy = np.zeros(n) if fy is None else fy
    mb = C.c_double(0.0)
    lib().ora_mol_forces(C.byref(p), C.byref(m), n, st["x"], st["y"], st["next"], fx, fy, C.byref(mb))
    return fx, fy, mb.value


CAT_DEFAULTS = dict(r_cat=1.2, syn_tries=8, syn_relax=20, syn_nN=0, nH=1, nT=3, feed_mode=1, vent_kind=0,
                    p_syn_a=0.02, p_syn_b=0.06, p_rep_a=0.001, p_rep_b=0.001, mu=0.02, p_ld=2e-4, p_kd=5e-4,
                    p_nd=1e-4, p_feed=1e-3, feed_cap=0.12, vent_x=-1.0, vent_y=-1.0, vent_r=5.0, vent_w=4.0)


def cat(**kv):
    """parameters of the catalyst chemistry (the reference's defaults, oercel.c:262-290)"""
    c = OraCat()
    for k, v in dict(CAT_DEFAULTS, **kv).items():
        setattr(c, k, v)
    return c


def catalyst_chemistry(p, c, st, cstart, step, rng, evcap=1 << 14):
    """one check of the reference's catalyst chemistry on the sorted state st
    (dict of slot arrays, changed in place); rng (4 uint64) advanced in place.
    Returns (moved, events as tuples (step, kind, i, variant, x, y))."""
    ev = (OraEvent * evcap)()
    nev = C.c_int32(0)
    moved = lib().ora_catalyst_chemistry(C.byref(p), C.byref(c), rng, len(st["x"]), st["x"], st["y"], st["vhx"],
                                         st["vhy"], st["vtx"], st["vty"], st["type"], st["gid"], st["prev"],
                                         st["next"], cstart, int(step), ev, evcap, C.byref(nev))
    out = [(e.step, e.kind, e.gid, (e.partner if e.partner < 2**31 else e.partner - 2**32), e.x, e.y)
           for e in ev[: min(nev.value, evcap)]]
    return moved, out


def stir_forces(p, st, fx):
    """add the stirring body force (mean removed) to fx in place"""
    lib().ora_stir_forces(C.byref(p), len(st["y"]), st["y"], fx)
    return fx


def sdt_at(p, step):
    return lib().ora_sdt_at(C.byref(p), int(step))


def integrate_f32(p, st):
    """advance st (dict of float32 arrays) in place; returns the count of beads left outside the box"""
    c = f32consts(p)
    return lib().ora_integrate_f32(C.byref(c), len(st["x"]), st["x"], st["y"], st["vhx"], st["vhy"], st["vtx"],
                                   st["vty"], st["fx"], st["fy"])


def chemistry(p, c, st, cstart, step, evcap=1 << 16):
    ev = (OraEvent * evcap)()
    n = lib().ora_chemistry(C.byref(p), C.byref(c), len(st["x"]), st["x"], st["y"], st["type"], st["gid"],
                            st["prev"], st["next"], cstart, step, ev, evcap)
    out = [(e.step, e.kind, e.gid, e.partner, e.x, e.y) for e in ev[: min(n, evcap)]]
    return n, out


def observables(p, st, cstart):
    out = np.zeros(5)
    lib().ora_observables(C.byref(p), len(st["x"]), st["x"], st["y"], st["vhx"], st["vhy"], st["fx"], st["fy"],
                          st["type"], st["next"], cstart, out)
    return dict(T=out[0], px=out[1], py=out[2], virial=out[3], maxbond=out[4])


def pair_hist(p, st, cstart, ta, tb, rmax, nbin):
    h = np.zeros(nbin)
    lib().ora_pair_hist(C.byref(p), len(st["x"]), st["x"], st["y"], st["type"], cstart, ta, tb, rmax, nbin, h)
    return h


def init_soup(L, rho, seed, *, kT=1.0, r0=0.5, nH=1, nT=2, f_lip=0.15, f_Ka=0.0, f_Kb=0.0, c_N=0.05):
    """the reference's random soup (same draws): float64 arrays in gid order"""
    N = int(round(rho * L * L))
    x, y, vx, vy = (np.empty(N) for _ in range(4))
    t = np.empty(N, np.uint8)
    g = np.empty(N, np.uint32)
    pv = np.empty(N, np.int32)
    nx = np.empty(N, np.int32)
    nl = lib().ora_init_soup(L, N, seed, kT, r0, nH, nT, f_lip, f_Ka, f_Kb, c_N, x, y, vx, vy, t, g, pv, nx)
    if nl < 0:
        raise ValueError("soup composition exceeds N")
    return dict(x=x, y=y, vx=vx, vy=vy, type=t, gid=g, prev=pv, next=nx)


def permute(st, src):
    """apply a sort permutation (new slot d <- old bead src[d]) to a state dict, remapping links"""
    dest = np.empty_like(src)
    dest[src] = np.arange(len(src), dtype=np.int32)
    out = {}
    for k, v in st.items():
        if k in ("prev", "next"):
            o = v[src]
            out[k] = np.where(o >= 0, dest[np.maximum(o, 0)], -1).astype(np.int32)
        else:
            out[k] = np.ascontiguousarray(v[src])
    return out


# ----------------------------------------------------------------------------- reference shim


class Ref:
    """The reference engine's own routines (oracle/_ref/libref_oercel.so)."""

    _lib = None

    @classmethod
    def available(cls):
        return os.path.exists(REF_PATH)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(REF_PATH)
            vp = C.c_void_p
            lib.ref_create.argtypes = [C.c_char_p]
            lib.ref_create.restype = vp
            for f in ("ref_prime", "ref_sort", "ref_integrate", "ref_destroy"):
                getattr(lib, f).argtypes = [vp]
            for f in ("ref_n", "ref_ncell", "ref_ncy"):
                getattr(lib, f).argtypes = [vp]
                getattr(lib, f).restype = C.c_int32
            lib.ref_get.argtypes = [vp] + [f64p] * 8 + [u8p, u32p, i32p, i8p]
            lib.ref_set.argtypes = [vp] + [f64p] * 8 + [u8p, u32p, i32p, i8p]
            lib.ref_cells.argtypes = [vp, i32p]
            lib.ref_cell_of.argtypes = [vp, C.c_double, C.c_double]
            lib.ref_cell_of.restype = C.c_int32
            lib.ref_pair.argtypes = [vp, C.c_int64]
            lib.ref_bonded.argtypes = [vp]
            lib.ref_bonded.restype = C.c_double
            lib.ref_run.argtypes = [vp, C.c_int64]
            lib.ref_step.argtypes = [vp]
            lib.ref_step.restype = C.c_int64
            lib.ref_theta.argtypes = [C.c_uint64, C.c_int64, C.c_uint32, C.c_uint32]
            lib.ref_theta.restype = C.c_double
            lib.ref_kinetic_T.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
            lib.ref_kinetic_T.restype = C.c_double
            lib.ref_chemistry.argtypes = [vp, C.c_int64]
            lib.ref_chemistry.restype = C.c_int32
            lib.ref_nev.argtypes = [vp]
            lib.ref_nev.restype = C.c_int32
            i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
            u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
            lib.ref_events.argtypes = [vp, i64p, i32p, i64p, f64p, f64p, i32p]
            lib.ref_get_rng.argtypes = [vp, u64p]
            lib.ref_set_rng.argtypes = [vp, u64p]
            lib.ref_template.argtypes = [vp, i32p, f64p]
            cls._lib = lib
        return cls._lib

    def __init__(self, **kv):
        text = "\n".join(f"{k}={v}" for k, v in kv.items())
        self.h = self.lib().ref_create(text.encode())
        self.n = self.lib().ref_n(self.h)

    def get(self):
        n = self.n
        a = {k: np.empty(n) for k in ("x", "y", "vx", "vy", "vtx", "vty", "fx", "fy")}
        t = np.empty(n, np.uint8)
        g = np.empty(n, np.uint32)
        nx = np.empty(n, np.int32)
        mp = np.empty(n, np.int8)
        self.lib().ref_get(self.h, a["x"], a["y"], a["vx"], a["vy"], a["vtx"], a["vty"], a["fx"], a["fy"], t, g, nx,
                           mp)
        a.update(type=t, gid=g, nxt=nx, mpos=mp)
        return a

    def set(self, a):
        c = {k: np.ascontiguousarray(a[k], np.float64) for k in ("x", "y", "vx", "vy", "vtx", "vty", "fx", "fy")}
        self.lib().ref_set(self.h, c["x"], c["y"], c["vx"], c["vy"], c["vtx"], c["vty"], c["fx"], c["fy"],
                           np.ascontiguousarray(a["type"], np.uint8), np.ascontiguousarray(a["gid"], np.uint32),
                           np.ascontiguousarray(a["nxt"], np.int32), np.ascontiguousarray(a["mpos"], np.int8))

    def cells(self):
        cs = np.empty(self.lib().ref_ncell(self.h) + 1, np.int32)
        self.lib().ref_cells(self.h, cs)
        return cs

    def events(self):
        n = self.lib().ref_nev(self.h)
        st, kd, i, v = (np.empty(n, np.int64), np.empty(n, np.int32), np.empty(n, np.int64), np.empty(n, np.int32))
        x, y = np.empty(n), np.empty(n)
        self.lib().ref_events(self.h, st, kd, i, x, y, v)
        return [(int(st[k]), int(kd[k]), int(i[k]), int(v[k]), float(x[k]), float(y[k])) for k in range(n)]

    def rng(self):
        r = np.empty(4, np.uint64)
        self.lib().ref_get_rng(self.h, r)
        return r

    def set_rng(self, r):
        self.lib().ref_set_rng(self.h, np.ascontiguousarray(r, np.uint64))

    def template(self):
        """the reference's lipid template for this handle's parameters (a dict)"""
        ints, dbls = np.zeros(512, np.int32), np.zeros(512)
        self.lib().ref_template(self.h, ints, dbls)
        arch, ml, nh, nb, na = (int(v) for v in ints[:5])
        k, d, t = 5, 0, dict(arch=arch, mlen=ml, nH=nh, nb=nb, na=na)
        for key, n in (("bi", nb), ("bj", nb), ("ai", na), ("aj", na), ("ak", na), ("akind", na)):
            t[key] = ints[k:k + n].copy()
            k += n
        for key, n in (("br0", nb), ("aK", na), ("ac0", na), ("px", ml), ("py", ml), ("ix", ml), ("iy", ml)):
            t[key] = dbls[d:d + n].copy()
            d += n
        return t

    def __getattr__(self, name):
        f = getattr(self.lib(), "ref_" + name)
        return lambda *a: f(self.h, *a)
