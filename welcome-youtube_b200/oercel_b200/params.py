"""Parameters with the reference engine's keys, defaults and parsing rules.

The reference keeps one table of (key, type, default, help) that drives ini
parsing, defaults, validation and the `--params` listing
(cel/engine/oercel.c:226-299, set_param :338-395, read_ini :409-434).  The
drop-in front end must accept the same keys with the same defaults, so the
key names and default values below are the reference's; the table itself and
the help texts are written here.  Keys marked NEW exist only in this engine.
"""
from __future__ import annotations

import math
import re

TYPE_NAMES = ["W", "H", "T", "N", "Ka", "Kb", "Z"]   # reference TNAME, oercel.c:49
TYPE_ALIASES = {"P": 3}                              # the precursor of the lipid chemistry is type 3
MAXT = 8

# (key, kind, default, help); kinds: int, long, float, str, u64
PDEFS = [
    ("L", "float", "64", "box side; beads N = round(rho L^2)"),
    ("rho", "float", "3", "number density"),
    ("dt", "float", "0.03", "time step"),
    ("lambda", "float", "0.65", "Groot-Warren predictor lambda"),
    ("gamma", "float", "4.5", "friction; sigma = sqrt(2 gamma kT)"),
    ("kT", "float", "1", "temperature"),
    ("k_bond", "float", "100", "bond constant, U = k/2 (r - r0)^2"),
    ("r0", "float", "0.5", "bond rest length"),
    ("k_angle", "float", "10", "angle constant, U = k (1 - cos theta) on consecutive chain triplets"),
    ("lip_nH", "int", "1", "head beads per lipid"),
    ("lip_nT", "int", "3", "tail beads per lipid"),
    ("lip_arch", "str", "linear", "lipid shape: linear, pi (two bonded heads, one tail each), y (one head, two "
                                  "tails) or bola (a head pair and a third head joined by two tails)"),
    ("r0_head", "float", "0.5", "pi / bola: rest length of the head-head bond and of pi's rungs"),
    ("k_head", "float", "0", "pi / y / bola: junction angle term k_head (cos theta - cos_head)^2 (0 = none)"),
    ("cos_head", "float", "0", "pi / y / bola: preferred cos of the junction angle"),
    ("lip_tie", "int", "0", "pi / y / bola: rungs between the two tails (tail beads m = 1..lip_tie)"),
    ("syn_nN", "int", "0", "N consumed per new lipid (0 = one per lipid bead; the rest are the nearest W)"),
    ("steps", "long", "10000", "run until this step number"),
    ("snap_every", "long", "1000", "snapshot interval (0 = none)"),
    ("stats_every", "long", "100", "stats.csv interval (0 = none)"),
    ("ckpt_every", "long", "10000", "checkpoint interval (0 = at the end only)"),
    ("ckpt_keep", "int", "0", "1 = keep ckpt_<step>.bin copies"),
    ("log_every", "long", "1000", "log line interval"),
    ("warmup", "long", "1000", "fresh soups: repulsions above 25 ramp in linearly over the first warmup steps"),
    ("threads", "int", "2", "host threads (the step runs on the GPU)"),
    ("nsub", "int", "4", "reference sub-cells per cell (the GPU grid is 1x1)"),
    ("seed", "u64", "1", "random seed"),
    ("init", "str", "soup", "soup or restart"),
    ("restart", "str", "", "checkpoint to continue from"),
    ("restart_reseed", "int", "0", "1 = branch with this seed on restart"),
    ("walltime", "float", "0", "stop cleanly after this many seconds (0 = off)"),
    ("chem", "int", "1", "1 = run the chemistry pass (chem_kind picks which)"),
    ("n_chem", "long", "10", "chemistry interval in steps"),
    ("r_cat", "float", "1.2", "catalyst reaction radius"),
    ("syn_tries", "int", "8", "new lipid: orientation = lowest overlap energy of this many random ones"),
    ("syn_relax", "int", "20", "new lipid: steepest-descent iterations moving only its own beads"),
    ("p_syn_a", "float", "0.02", "lipid synthesis probability per check, Ka"),
    ("p_syn_b", "float", "0.06", "lipid synthesis probability per check, Kb"),
    ("p_rep_a", "float", "0.001", "catalyst replication probability per check, Ka"),
    ("p_rep_b", "float", "0.001", "catalyst replication probability per check, Kb"),
    ("mu", "float", "0.02", "mutation probability per replication (a <-> b)"),
    ("p_ld", "float", "2e-4", "lipid decay probability per molecule per check"),
    ("p_kd", "float", "5e-4", "catalyst decay probability per check"),
    ("p_nd", "float", "1e-4", "N decay probability per check"),
    ("feed", "str", "uniform", "food supply W -> N: none, uniform or vent"),
    ("p_feed", "float", "1e-3", "W -> N probability per check"),
    ("feed_cap", "float", "0.12", "cap on the N fraction (0 = no cap)"),
    ("vent_shape", "str", "disk", "vent: disk, vstrip or hstrip"),
    ("vent_x", "float", "-1", "vent centre x (-1 = L/2)"),
    ("vent_y", "float", "-1", "vent centre y (-1 = L/2)"),
    ("vent_r", "float", "5", "vent disk radius"),
    ("vent_w", "float", "4", "vent strip width"),
    ("events", "int", "1", "1 = write events.csv"),
    ("stir_A", "float", "0", "stirring body force f_x = stir_A sin(2 pi stir_n y / L), net force removed"),
    ("stir_n", "int", "1", "stirring periods"),
    ("kT_amp", "float", "0", "temperature cycle kT(t) = kT + kT_amp sin(2 pi t / kT_period) in the noise"),
    ("kT_period", "float", "1000", "temperature cycle period"),
    ("f_lip", "float", "0.10", "soup: fraction of beads in lipids"),
    ("f_Ka", "float", "0.005", "soup: fraction of Ka beads"),
    ("f_Kb", "float", "0", "soup: fraction of Kb beads"),
    ("c_N", "float", "0.12", "soup: fraction of N (P) beads"),
    # NEW: this engine's noise generator and lipid chemistry
    ("noise", "str", "philox", "NEW pair noise: philox (Philox4x32-10) or mix13 (the reference's hash)"),
    ("chem_kind", "str", "catalyst", "NEW chemistry of chem = 1: catalyst (the reference's) or lipid (below)"),
    ("p_grow", "float", "1e-3", "NEW P -> T growth probability per check"),
    ("p_break", "float", "1e-5", "NEW H-T bond break probability per check"),
    ("p_bond", "float", "1e-2", "NEW free T + free H bonding probability per check"),
    ("r_grow", "float", "1.0", "NEW growth radius"),
    ("r_bond", "float", "0.6", "NEW bonding radius"),
    ("n_t_min", "int", "2", "NEW T beads a P needs within r_grow"),
    ("max_chain", "int", "12", "NEW longest chain growth may produce"),
    ("ckpt_format", "str", "own", "NEW checkpoint format: own (exact FP32 continuation here) or reference (the "
                                  "reference engine's OCKP v2/v3, which its executable can continue)"),
]
PKEYS = {k: (t, d, h) for k, t, d, h in PDEFS}
ARCHS = ("linear", "pi", "y", "bola")
REMOVED = {"seed_R", "seed_spacing", "seed_cN_in", "seed_nKa", "feed_every", "feed_grid", "feed_tmin"}


class ParamError(ValueError):
    pass


def default_amatrix():
    """the reference's default repulsions (oercel.c:303-320)"""
    a = [[25.0] * MAXT for _ in range(MAXT)]

    def s(i, j, v):
        a[i][j] = a[j][i] = v

    s(0, 1, 20.0)
    s(0, 2, 80.0)
    s(1, 2, 50.0)
    s(3, 0, 25.0)
    s(3, 1, 25.0)
    s(3, 2, 40.0)
    for k in (4, 5):
        s(k, 0, 25.0)
        s(k, 1, 30.0)
        s(k, 2, 120.0)
        s(k, 3, 25.0)
    return a


def _type_index(name):
    if name in TYPE_NAMES:
        return [TYPE_NAMES.index(name)]
    if name in TYPE_ALIASES:
        return [TYPE_ALIASES[name]]
    if name == "K":
        return [4, 5]
    return None


def _parse(kind, key, val):
    val = val.strip()
    try:
        if kind == "int":
            if not re.fullmatch(r"[+-]?\d+", val):
                raise ValueError
            return int(val)
        if kind == "long":
            return int(round(float(val)))
        if kind == "u64":
            return int(val, 0)
        if kind == "float":
            return float(val)
        return val
    except ValueError:
        raise ParamError(f"bad value for {key}: '{val}'") from None


class Params:
    """Parameter set; attribute access by key (p.L, p["lambda"])."""

    def __init__(self, **overrides):
        self.v = {k: _parse(t, k, d) for k, t, d, _ in PDEFS}
        self.a = default_amatrix()
        for k, val in overrides.items():
            self.set(k, str(val))

    def __getattr__(self, k):
        v = self.__dict__.get("v")
        if v is not None and k in v:
            return v[k]
        raise AttributeError(k)

    def __getitem__(self, k):
        return self.v[k]

    def set(self, key: str, val: str):
        key = key.strip()
        if key.startswith("a_"):
            parts = key[2:].split("_")
            if len(parts) != 2:
                raise ParamError(f"bad repulsion key '{key}' (use a_X_Y)")
            t1, t2 = _type_index(parts[0]), _type_index(parts[1])
            if t1 is None or t2 is None:
                raise ParamError(f"bad repulsion key '{key}'")
            x = _parse("float", key, val)
            for i in t1:
                for j in t2:
                    self.a[i][j] = self.a[j][i] = x
            return
        if key in PKEYS:
            self.v[key] = _parse(PKEYS[key][0], key, val)
            return
        if key in REMOVED:
            raise ParamError(f"parameter '{key}' was removed in the reference engine")
        raise ParamError(f"unknown parameter '{key}'")

    def update(self, items):
        """apply (key, value) pairs: generic catalyst keys a_K_X first (oercel.c:2155-2158)"""
        items = list(items)
        gen = [kv for kv in items if _generic(kv[0])]
        for k, v in gen + [kv for kv in items if not _generic(kv[0])]:
            self.set(k, v)
        return self

    @classmethod
    def from_ini(cls, path, overrides=()):
        p = cls()
        return p.update(read_ini(path) + [parse_override(o) for o in overrides])

    def n_beads(self):
        return int(round(self.rho * self.L * self.L))

    def validate(self):
        """the reference's finalize_params checks that apply here, plus this engine's limits"""
        if self.L < 8:
            raise ParamError("L must be >= 8")
        if self.dt <= 0:
            raise ParamError("dt must be > 0")
        if self.kT <= 0:
            raise ParamError("kT must be > 0")
        if self.lip_arch not in ARCHS:
            raise ParamError("lip_arch must be linear, pi, y or bola")
        if self.lip_arch != "linear" and self.lip_nT < 1:
            raise ParamError("branched lipids need lip_nT >= 1")
        if self.mlen() > 16:
            raise ParamError("lipids of at most 16 beads")
        if self.k_angle < 0:
            raise ParamError("k_angle must be >= 0")
        if self.stir_n < 1:
            raise ParamError("stir_n must be >= 1")
        if self.kT_amp != 0 and self.kT_period <= 0:
            raise ParamError("kT_period must be > 0")
        if self.kT_amp != 0 and self.kT - abs(self.kT_amp) <= 0:
            raise ParamError("kT - |kT_amp| must be > 0")
        if self.noise not in ("philox", "mix13"):
            raise ParamError("noise must be philox or mix13")
        if self.init not in ("soup", "restart"):
            raise ParamError("init must be soup or restart")
        if self.ckpt_format not in ("own", "reference"):
            raise ParamError("ckpt_format must be own or reference")
        if self.chem_kind not in ("catalyst", "lipid"):
            raise ParamError("chem_kind must be catalyst or lipid")
        if self.feed not in ("none", "0", "uniform", "vent"):
            raise ParamError("feed must be none, uniform or vent")
        if self.vent_shape not in ("disk", "vstrip", "hstrip"):
            raise ParamError("vent_shape must be disk, vstrip or hstrip")
        if not (0 <= self.p_feed <= 1) or not (0 <= self.feed_cap < 1):
            raise ParamError("p_feed must be in [0, 1] and feed_cap in [0, 1)")
        if not (0 <= self.syn_nN <= self.lip_nH + self.lip_nT):
            raise ParamError("syn_nN must be 0..mlen")
        if self.syn_tries > 64:
            raise ParamError("syn_tries must be <= 64 (orientation trials held in shared memory)")
        return self

    def sigma(self):
        return math.sqrt(2.0 * self.gamma * self.kT)

    def mlen(self):
        """beads of one lipid (oercel.c:486-553)"""
        nT = int(self.lip_nT)
        return {"linear": int(self.lip_nH) + nT, "pi": 2 + 2 * nT, "y": 1 + 2 * nT, "bola": 3 + 2 * nT}.get(
            self.lip_arch, int(self.lip_nH) + nT)

    def template(self):
        """the lipid molecule template (dpd_lipid_template): a DpdTemplate"""
        from ._capi import DpdTemplate, check, load
        t = DpdTemplate()
        check(load().dpd_lipid_template(self.to_struct(), t))
        return t

    def to_struct(self, seed=None, warm_end=None, t_anchor=0.0, step_anchor=0):
        from ._capi import DpdParams, load
        s = DpdParams()
        load().dpd_params_default(s)
        s.L = float(self.L)
        s.dt = float(self.dt)
        s.lam = float(self["lambda"])
        s.gamma = float(self.gamma)
        s.kT = float(self.kT)
        for i in range(MAXT):
            for j in range(MAXT):
                s.a[i * MAXT + j] = float(self.a[i][j])
        s.k_bond = float(self.k_bond)
        s.r0 = float(self.r0)
        s.seed = int(self.seed if seed is None else seed) & 0xFFFFFFFFFFFFFFFF
        s.noise = 0 if self.noise == "philox" else 1
        s.chem = int(self.chem)
        s.n_chem = int(self.n_chem)
        s.n_t_min = int(self.n_t_min)
        s.max_chain = int(self.max_chain)
        s.p_break, s.p_grow, s.p_bond = float(self.p_break), float(self.p_grow), float(self.p_bond)
        s.r_grow, s.r_bond = float(self.r_grow), float(self.r_bond)
        s.warmup = max(int(self.warmup), 0)
        s.warm_end = int(self.warmup if warm_end is None else warm_end)
        s.k_angle = float(self.k_angle)
        s.stir_A, s.stir_n = float(self.stir_A), int(self.stir_n)
        s.kT_amp, s.kT_period = float(self.kT_amp), float(self.kT_period)
        s.t_anchor, s.step_anchor = float(t_anchor), int(step_anchor)
        s.chem_kind = 1 if self.chem_kind == "catalyst" else 0
        s.syn_tries, s.syn_relax, s.syn_nN = max(int(self.syn_tries), 1), int(self.syn_relax), int(self.syn_nN)
        s.lip_nH, s.lip_nT = int(self.lip_nH), int(self.lip_nT)
        s.lip_arch = ARCHS.index(self.lip_arch) if self.lip_arch in ARCHS else -1
        s.lip_tie = int(self.lip_tie)
        s.r0_head, s.k_head, s.cos_head = float(self.r0_head), float(self.k_head), float(self.cos_head)
        s.feed_mode = {"none": 0, "0": 0, "uniform": 1, "vent": 2}[self.feed]
        s.vent_kind = {"disk": 0, "vstrip": 1, "hstrip": 2}[self.vent_shape]
        for k in ("r_cat", "p_syn_a", "p_syn_b", "p_rep_a", "p_rep_b", "mu", "p_ld", "p_kd", "p_nd", "p_feed",
                  "feed_cap", "vent_x", "vent_y", "vent_r", "vent_w"):
            setattr(s, k, float(self[k]))
        return s

    def write(self, path, overrides=()):
        """params.ini with every key (reference write_params, oercel.c:626-653)"""
        with open(path, "w") as f:
            f.write("# oercel_b200 parameters actually used (all keys, defaults filled in)\n")
            if overrides:
                f.write("# command-line overrides: " + " ".join(overrides) + "\n")
            for k, t, _, h in PDEFS:
                v = self.v[k]
                vs = repr(float(v)) if t == "float" else str(v)
                f.write(f"{k} = {vs}    # {h}\n")
            f.write(f"# derived: sigma = {self.sigma()!r}\n# repulsion matrix a_ij (symmetric)\n")
            for i in range(len(TYPE_NAMES)):
                for j in range(i, len(TYPE_NAMES)):
                    f.write(f"a_{TYPE_NAMES[i]}_{TYPE_NAMES[j]} = {self.a[i][j]!r}\n")


def _generic(key):
    if not key.startswith("a_"):
        return False
    parts = key[2:].split("_")
    return len(parts) == 2 and "K" in parts


def read_ini(path):
    """key = value lines, '#' comments (reference read_ini, oercel.c:409-434)"""
    out = []
    with open(path) as f:
        for ln, line in enumerate(f, 1):
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            if "=" not in line:
                raise ParamError(f"{path}:{ln}: expected key = value")
            k, v = line.split("=", 1)
            out.append((k.strip(), v.strip()))
    return out


def parse_override(o):
    if "=" not in o:
        raise ParamError(f"override '{o}' is not key=value")
    k, v = o.split("=", 1)
    return k.strip(), v.strip()


def param_table():
    """markdown table of every key, as the reference's --params (oercel.c:2107-2123)"""
    lines = ["| key | default | meaning |", "|---|---|---|"]
    for k, _, d, h in PDEFS:
        lines.append(f"| `{k}` | {d if d else '(empty)'} | {h} |")
    a = default_amatrix()
    lines.append("")
    lines.append("Default repulsion matrix a_ij (key `a_X_Y`, symmetric; `a_K_X` sets Ka and Kb at once):")
    lines.append("")
    lines.append("|    |" + "".join(f" {n} |" for n in TYPE_NAMES))
    lines.append("|---|" + "---|" * len(TYPE_NAMES))
    for i, n in enumerate(TYPE_NAMES):
        lines.append(f"| **{n}** |" + "".join(f" {a[i][j]:g} |" for j in range(len(TYPE_NAMES))))
    return "\n".join(lines)
