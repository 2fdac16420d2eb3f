"""Hand-built snapshots for cell detection: vesicles (closed bilayer rings of
H-T-T-T lipids) with water, nutrients and catalysts inside; vesicles across
the box edge and on the corner; a nested pair; a dry vesicle (no water
inside); an open ring; micelles and free lipids; and a membrane network that
wraps the periodic box and encloses lumens (one of them across the edge).

The scenes are geometry only (no dynamics): every position is a float32, as in
a snapshot file.  write_snap() writes the engine's snapshot format, tile()
makes k x k periodic copies of a scene.
"""
from __future__ import annotations

import struct

import numpy as np

W, H, T, N, KA, KB, Z = 0, 1, 2, 3, 4, 5, 6
BOND = 0.5          # bead spacing along a lipid
HEAD = 1.65         # head distance from the bilayer midline
STEP = 0.62         # lipid spacing along a leaflet


class Scene:
    def __init__(self, L, seed):
        self.L = float(L)
        self.rng = np.random.default_rng(seed)
        self.pos, self.typ, self.bonds = [], [], []
        self.dry = []        # (cx, cy, r): no solvent inside
        self.memb = []       # (kind, params) bands kept free of solvent

    def _lipid(self, base, u, jitter):
        """a lipid whose head sits at base, tail pointing along -u"""
        i0 = len(self.typ)
        for k in range(4):
            p = base - k * BOND * u + self.rng.normal(0, jitter, 2)
            self.pos.append(p % self.L)
            self.typ.append(H if k == 0 else T)
        for k in range(3):
            self.bonds.append((i0 + k, i0 + k + 1))

    def ring(self, cx, cy, r, jitter=0.05, gap=0.0, solvent=True):
        """a closed bilayer along a circle of radius r (midline); gap: the
        angular fraction left open"""
        c = np.array([cx, cy])
        for side in (+1, -1):
            rr = r + side * HEAD
            k = max(int(2 * np.pi * rr / STEP), 6)
            a0 = self.rng.uniform(0, 2 * np.pi)
            for j in range(k):
                a = a0 + 2 * np.pi * j / k
                if gap and ((a - 0.3) % (2 * np.pi)) < 2 * np.pi * gap:
                    continue
                u = np.array([np.cos(a), np.sin(a)]) * side
                self._lipid(c + rr * u * side, u, jitter)
        self.memb.append(("ring", (cx, cy, r)))
        if not solvent:
            self.dry.append((cx, cy, r))

    def stripe(self, y0, jitter=0.05, axis=0, lo=None, hi=None):
        """a straight bilayer at coordinate y0 across the box (axis 0: along x),
        or the segment lo..hi of it"""
        lo = 0.0 if lo is None else lo
        hi = self.L if hi is None else hi
        for side in (+1, -1):
            k = max(int((hi - lo) / STEP), 2)
            s0 = self.rng.uniform(0, (hi - lo) / k)
            for j in range(k):
                s = lo + s0 + j * (hi - lo) / k
                u = np.array([0.0, side]) if axis == 0 else np.array([side, 0.0])
                base = (np.array([s, y0]) if axis == 0 else np.array([y0, s])) + HEAD * u
                self._lipid(base, u, jitter)
        self.memb.append(("stripe", (y0, axis, lo, hi)))

    def micelle(self, cx, cy, k, jitter=0.05):
        a0 = self.rng.uniform(0, 2 * np.pi)
        for j in range(k):
            a = a0 + 2 * np.pi * j / k
            u = np.array([np.cos(a), np.sin(a)])
            self._lipid(np.array([cx, cy]) + 1.7 * u, u, jitter)

    def free_lipids(self, n):
        for _ in range(n):
            a = self.rng.uniform(0, 2 * np.pi)
            self._lipid(self.rng.uniform(0, self.L, 2), np.array([np.cos(a), np.sin(a)]), 0.05)

    def _in_membrane(self, p):
        L = self.L
        for kind, q in self.memb:
            if kind == "ring":
                cx, cy, r = q
                d = np.hypot(*(((p - (cx, cy)) + L / 2) % L - L / 2).T)
                if abs(d - r) < HEAD + 0.3:
                    return True
            else:
                y0, axis, lo, hi = q
                c = p[1] if axis == 0 else p[0]
                s = p[0] if axis == 0 else p[1]
                dc = (c - y0 + L / 2) % L - L / 2
                if abs(dc) < HEAD + 0.3 and (lo - 0.3 <= s <= hi + 0.3 or hi - lo >= L):
                    return True
        return False

    def _dry(self, p):
        L = self.L
        for cx, cy, r in self.dry:
            if np.hypot(*(((p - (cx, cy)) + L / 2) % L - L / 2).T) < r:
                return True
        return False

    def solvent(self, rho=3.0, f_N=0.05, f_K=0.01, f_Z=0.01):
        """water (with nutrients N, catalysts Ka/Kb and waste Z) at density rho
        outside the membranes and the dry vesicles"""
        n = self.rng.poisson(rho * self.L * self.L)
        for p in self.rng.uniform(0, self.L, (n, 2)):
            if self._in_membrane(p) or self._dry(p):
                continue
            u = self.rng.random()
            t = N if u < f_N else KA if u < f_N + f_K else KB if u < f_N + 2 * f_K else \
                Z if u < f_N + 2 * f_K + f_Z else W
            self.pos.append(p)
            self.typ.append(t)

    def arrays(self):
        p = np.asarray(self.pos, np.float64).reshape(-1, 2) % self.L
        x = p[:, 0].astype(np.float32)
        y = p[:, 1].astype(np.float32)
        x[x >= np.float32(self.L)] = 0
        y[y >= np.float32(self.L)] = 0
        return x, y, np.asarray(self.typ, np.uint8), np.asarray(self.bonds, np.int32).reshape(-1, 2)


def write_snap(path, L, x, y, t, bonds, step=0, time=0.0):
    with open(path, "wb") as f:
        f.write(b"OCEL" + struct.pack("<iiiqdd", 1, len(t), len(bonds), step, time, L))
        f.write(np.asarray(x, "<f4").tobytes())
        f.write(np.asarray(y, "<f4").tobytes())
        f.write(np.asarray(t, "u1").tobytes())
        f.write(np.asarray(bonds, "<i4").tobytes())


def tile(L, x, y, t, bonds, k):
    """k x k periodic copies of a box (positions in FP64, each copy shifted by
    whole boxes); a bond that crosses the box edge joins the bead of one copy
    to the neighbouring copy's"""
    n = len(t)
    b = np.asarray(bonds, np.int64)
    d = np.stack([x[b[:, 1]].astype(np.float64) - x[b[:, 0]], y[b[:, 1]].astype(np.float64) - y[b[:, 0]]])
    sh = np.where(d > L / 2, -1, np.where(d < -L / 2, 1, 0))
    xs, ys, bs = [], [], []
    for a in range(k):
        for c in range(k):
            xs.append(x.astype(np.float64) + a * L)
            ys.append(y.astype(np.float64) + c * L)
            other = ((a + sh[0]) % k) * k + (c + sh[1]) % k
            bs.append(np.stack([b[:, 0] + (a * k + c) * n, b[:, 1] + other * n], 1))
    return L * k, np.concatenate(xs), np.concatenate(ys), np.tile(t, k * k), np.concatenate(bs).astype(np.int32)


def vesicles(seed):
    """L = 56: a free vesicle, one across x = L, one on the corner, a nested
    pair, a dry vesicle, an open ring, micelles and free lipids"""
    s = Scene(56, seed)
    s.ring(14, 18, 6.0)
    s.ring(38, 16, 10.0)
    s.ring(38, 16, 4.8)
    s.ring(54, 36, 6.0)
    s.ring(1.0, 55.0, 6.0)
    s.ring(16, 40, 5.5, solvent=False)
    s.ring(34, 44, 5.0, gap=0.2)
    for c, k in (((25, 32), 7), ((47, 52), 8), ((7, 29), 6), ((27, 52), 9)):
        s.micelle(*c, k)
    s.free_lipids(25)
    s.solvent()
    return s


def network(seed):
    """L = 48: two bilayers across the box along x (y = 8, 28) joined by two
    along y (x = 12, 36): one aggregate that wraps the box and encloses two
    lumens, one across x = L; a vesicle fused onto the upper bilayer (part of
    the wrapping aggregate) and a free vesicle in the open band"""
    s = Scene(48, seed)
    s.stripe(8.0)
    s.stripe(28.0)
    for x0 in (12.0, 36.0):
        s.stripe(x0, axis=1, lo=8 + HEAD - 0.2, hi=28 - HEAD + 0.2)
    s.ring(20, 28 + HEAD - 0.5 + 0.6 + 5.5 + 0.15, 5.5)
    s.ring(40, 44, 4.5)
    s.micelle(4, 40, 7)
    s.free_lipids(10)
    s.solvent()
    return s


def water(seed):
    """L = 20: solvent only, no lipid"""
    s = Scene(20, seed)
    s.solvent()
    return s


def micelles(seed):
    """L = 20: two micelles and free lipids, no membrane"""
    s = Scene(20, seed)
    s.micelle(5, 5, 8)
    s.micelle(14, 14, 7)
    s.free_lipids(5)
    s.solvent()
    return s


def tiny(seed):
    """L = 2.5, a box under three tail-contact cells wide: three lipids in water"""
    s = Scene(2.5, seed)
    s.free_lipids(3)
    s.solvent()
    return s


def lone(seed):
    """L = 16: one vesicle whose lumen is too small to count"""
    s = Scene(16, seed)
    s.ring(8, 8, 4.5)
    s.solvent()
    return s


def empty(seed):
    """L = 16 with no bead at all"""
    return Scene(16, seed)


SCENES = {"vesicles": vesicles, "network": network, "water": water, "micelles": micelles, "tiny": tiny,
          "lone": lone, "empty": empty}
