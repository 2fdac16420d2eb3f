"""In-process engine: the reference engine's step / parameter / state interface
over libdpd.so.

The reference engine (cel/engine/oercel.c) owns its state in one process and
advances it with the loop of main() (:2300-2361).  Engine does the same on
the GPU: one handle holds one or more replicas (independent boxes packed into
one set of device arrays) and every method is one C-ABI call.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import DpdEvent, check, load, ptr
from .params import Params

# lipid chemistry 0..2, then the reference's catalyst chemistry (its EVNAME, oercel.c:659)
EVENT_KINDS = ("grow", "brk", "bond", "syn", "rep", "mut", "dlip", "dK", "dN", "feed")


def make_soup(L, N, seed, *, kT=1.0, r0=0.5, nH=1, nT=3, f_lip=0.10, f_Ka=0.0, f_Kb=0.0, c_N=0.12, mol=None):
    """The reference's random soup (same draws as init_soup/set_velocities) from
    libdpd's host routine; float64 arrays in gid order.  mol: the lipid template
    of a branched shape (Params.template()), None for linear lipids."""
    lib = load()
    x, y, vx, vy = (np.empty(N, np.float64) for _ in range(4))
    t = np.empty(N, np.uint8)
    pv = np.empty(N, np.int32)
    nx = np.empty(N, np.int32)
    nl = C.c_int32(0)
    rng = np.zeros(4, np.uint64)
    check(lib.dpd_init_soup(float(L), int(N), int(seed) & 0xFFFFFFFFFFFFFFFF, float(kT), float(r0), int(nH),
                            int(nT), float(f_lip), float(f_Ka), float(f_Kb), float(c_N), ptr(x), ptr(y), ptr(vx),
                            ptr(vy), ptr(t), ptr(pv), ptr(nx), C.byref(nl), ptr(rng),
                            C.byref(mol) if mol is not None else None))
    return dict(x=x, y=y, vx=vx, vy=vy, type=t, prev=pv, next=nx, n_lipid_beads=nl.value, rng=rng)


def soup_for(p: Params, seed=None):
    """soup of a parameter set (positions rounded to FP32 inside [0, L))"""
    s = make_soup(np.float32(p.L), p.n_beads(), p.seed if seed is None else seed, kT=p.kT, r0=p.r0,
                  nH=p.lip_nH, nT=p.lip_nT, f_lip=p.f_lip, f_Ka=p.f_Ka, f_Kb=p.f_Kb, c_N=p.c_N,
                  mol=p.template() if p.lip_arch != "linear" else None)
    L = np.float32(p.L)
    for k in ("x", "y"):
        v = s[k].astype(np.float32)
        v[v >= L] = np.float32(0.0)   # a coordinate that rounds up to L wraps to 0
        s[k] = v
    s["vx"] = s["vx"].astype(np.float32)
    s["vy"] = s["vy"].astype(np.float32)
    return s


class Engine:
    """GPU simulation of one or more replicas.

    params: a Params (one replica) or a list of Params (one per replica).
    n_beads: bead count per replica (default round(rho L^2))."""

    def __init__(self, params, n_beads=None):
        self.lib = load()
        plist = list(params) if isinstance(params, (list, tuple)) else [params]
        self.params = plist
        self.nrep = len(plist)
        if n_beads is None:
            n_beads = [p.n_beads() for p in plist]
        n_beads = [int(n) for n in (n_beads if hasattr(n_beads, "__len__") else [n_beads])]
        structs = (_capi.DpdParams * self.nrep)(*[p.to_struct() for p in plist])
        nb = (C.c_int32 * self.nrep)(*n_beads)
        self.h = C.c_void_p()
        check(self.lib.dpd_create(structs, self.nrep, nb, C.byref(self.h)))
        self.n_beads = n_beads

    # ---------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.lib.dpd_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------------------------------------------------------- state
    def set_state(self, replica, x, y, vx, vy, type, gid=None, prev=None, next=None):
        f32 = lambda a: np.ascontiguousarray(a, np.float32) if isinstance(a, np.ndarray) else a
        args = [f32(x), f32(y), f32(vx), f32(vy)]
        t = np.ascontiguousarray(type, np.uint8) if isinstance(type, np.ndarray) else type
        g = np.ascontiguousarray(gid, np.uint32) if isinstance(gid, np.ndarray) else gid
        pv = np.ascontiguousarray(prev, np.int32) if isinstance(prev, np.ndarray) else prev
        nx = np.ascontiguousarray(next, np.int32) if isinstance(next, np.ndarray) else next
        check(self.lib.dpd_set_state(self.h, replica, *[ptr(a) for a in args], ptr(t), ptr(g), ptr(pv), ptr(nx)))

    def load_soup(self, replica=0, seed=None):
        """the reference's soup for this replica's parameters; the serial
        generator continues from where the soup left it"""
        s = soup_for(self.params[replica], seed)
        self.set_state(replica, s["x"], s["y"], s["vx"], s["vy"], s["type"], None, s["prev"], s["next"])
        self.set_rng(replica, s["rng"])
        return s

    def set_rng(self, replica, state):
        check(self.lib.dpd_set_rng(self.h, replica, ptr(np.ascontiguousarray(state, np.uint64))))

    def rng(self, replica=0):
        r = np.zeros(4, np.uint64)
        check(self.lib.dpd_get_rng(self.h, replica, ptr(r)))
        return r

    def state(self, replica=0):
        n = self.n_beads[replica]
        out = {k: np.empty(n, np.float32) for k in ("x", "y", "vhx", "vhy", "vtx", "vty", "fx", "fy")}
        out["type"] = np.empty(n, np.uint8)
        out["gid"] = np.empty(n, np.uint32)
        out["prev"] = np.empty(n, np.int32)
        out["next"] = np.empty(n, np.int32)
        o = out
        check(self.lib.dpd_get_state(self.h, replica, ptr(o["x"]), ptr(o["y"]), ptr(o["vhx"]), ptr(o["vhy"]),
                                     ptr(o["vtx"]), ptr(o["vty"]), ptr(o["fx"]), ptr(o["fy"]), ptr(o["type"]),
                                     ptr(o["gid"]), ptr(o["prev"]), ptr(o["next"])))
        return out

    def set_dynamics(self, replica, vhx=None, vhy=None, fx=None, fy=None, vtx=None, vty=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        a = [c(vhx), c(vhy), c(fx), c(fy), c(vtx), c(vty)]
        check(self.lib.dpd_set_dynamics(self.h, replica, *[ptr(v) for v in a]))

    def cells(self, replica=0):
        nc = C.c_int32()
        check(self.lib.dpd_sizes(self.h, replica, None, None, C.byref(nc)))
        cs = np.empty(nc.value + 1, np.int32)
        check(self.lib.dpd_get_cells(self.h, replica, ptr(cs)))
        return cs

    # ---------------------------------------------------------------- stepping
    def prime(self):
        check(self.lib.dpd_prime(self.h))

    def resume(self):
        check(self.lib.dpd_resume(self.h))

    def step(self, n=1):
        check(self.lib.dpd_step(self.h, int(n)))

    def step_async(self, n=1):
        check(self.lib.dpd_step_async(self.h, int(n)))

    def sync(self):
        check(self.lib.dpd_sync(self.h))

    def set_graph_steps(self, n):
        check(self.lib.dpd_set_graph_steps(self.h, int(n)))

    def tuning(self):
        t = _capi.DpdTuning()
        check(self.lib.dpd_get_tuning(self.h, C.byref(t)))
        return dict(force_kernel=t.force_kernel, tile_w=t.tile_w, tile_h=t.tile_h, graph_steps=t.graph_steps,
                    sort_mode=t.sort_mode, tile_threads=t.tile_threads)

    def set_tuning(self, **kv):
        cur = self.tuning()
        cur.update(kv)
        t = _capi.DpdTuning(int(cur["force_kernel"]), int(cur["tile_w"]), int(cur["tile_h"]), int(cur["graph_steps"]),
                            int(cur["sort_mode"]), int(cur["tile_threads"]))
        check(self.lib.dpd_set_tuning(self.h, C.byref(t)))

    def profile_step(self):
        """device time (ms) of each kernel of one real step, in launch order"""
        ms = (C.c_float * 32)()
        n = C.c_int32()
        check(self.lib.dpd_profile_step(self.h, ms, 32, C.byref(n)))
        return [ms[k] for k in range(n.value)]

    @property
    def step_no(self):
        s = C.c_int64()
        check(self.lib.dpd_get_step(self.h, C.byref(s)))
        return s.value

    def set_step(self, s):
        check(self.lib.dpd_set_step(self.h, int(s)))

    # ---------------------------------------------------------------- phases
    def build_cells(self):
        check(self.lib.dpd_build_cells(self.h))

    def forces(self, step):
        check(self.lib.dpd_forces(self.h, int(step)))

    def pair_forces(self, replica, step):
        n = self.n_beads[replica]
        fx, fy = np.empty(n, np.float32), np.empty(n, np.float32)
        check(self.lib.dpd_pair_forces(self.h, replica, int(step), ptr(fx), ptr(fy)))
        return fx, fy

    def bond_forces(self, replica):
        n = self.n_beads[replica]
        fx, fy = np.empty(n, np.float32), np.empty(n, np.float32)
        mb = C.c_float()
        check(self.lib.dpd_bond_forces(self.h, replica, ptr(fx), ptr(fy), C.byref(mb)))
        return fx, fy, mb.value

    def integrate(self):
        check(self.lib.dpd_integrate(self.h))

    def chemistry(self, step):
        check(self.lib.dpd_chemistry(self.h, int(step)))

    # ---------------------------------------------------------------- outputs
    def events(self):
        """(step, kind, gid, partner gid, x, y, replica) of the events since the last call"""
        n = C.c_int32()
        check(self.lib.dpd_get_events(self.h, None, 0, C.byref(n)))
        cap = max(n.value, 1)
        buf = (DpdEvent * cap)()
        check(self.lib.dpd_get_events(self.h, buf, cap, C.byref(n)))
        return [(e.step, e.kind, e.gid, e.partner, e.x, e.y, e.replica) for e in buf[: n.value]]

    # a DpdEvent as a numpy record (the layout of dpd_event)
    EVENT_DTYPE = np.dtype([("step", np.int64), ("kind", np.int32), ("gid", np.uint32), ("partner", np.uint32),
                            ("x", np.float32), ("y", np.float32), ("replica", np.int32)])

    def events_async(self, buf, count):
        """enqueue a read of the events since the last read into buf (pinned
        host memory with EVENT_DTYPE records, e.g. a numpy view of
        torch.empty(..., pin_memory=True)) and their number into count (a
        pinned int32 array of one element; more than len(buf) means the rest
        were dropped); both are valid once the stream has passed this point
        (sync, or an event recorded after it).  Nothing waits."""
        assert buf.dtype == self.EVENT_DTYPE and buf.ndim == 1 and buf.flags.c_contiguous
        assert count.dtype == np.int32 and count.size >= 1 and count.flags.c_contiguous
        check(self.lib.dpd_events_async(self.h, buf.ctypes.data, int(buf.shape[0]), count.ctypes.data))

    @staticmethod
    def event_tuples(buf, n):
        """records of an events_async read as (step, kind, gid, partner gid, x, y, replica), like events()"""
        return [(int(e["step"]), int(e["kind"]), int(e["gid"]), int(e["partner"]), float(e["x"]), float(e["y"]),
                 int(e["replica"])) for e in buf[:min(int(n), len(buf))]]

    def observables(self, replica=0, virial=True):
        o = np.zeros(16)
        f = self.lib.dpd_observables if virial else self.lib.dpd_stats
        check(f(self.h, replica, ptr(o)))
        return dict(T=o[0], px=o[1], py=o[2], virial=o[3], maxbond=o[4], n_chains=int(o[5]),
                    counts=o[8:16].astype(np.int64))

    def stats_async(self, replica, raw):
        """enqueue the stats row; its 16 raw sums land in raw (a pinned uint64
        array) once the stream passes (sync); stats_decode reads them"""
        check(self.lib.dpd_stats_async(self.h, int(replica), ptr(raw)))

    def stats_decode(self, replica, raw):
        o = np.zeros(16)
        check(self.lib.dpd_stats_decode(self.h, int(replica), ptr(np.ascontiguousarray(raw, np.uint64)), ptr(o)))
        return dict(T=o[0], px=o[1], py=o[2], virial=o[3], maxbond=o[4], n_chains=int(o[5]),
                    counts=o[8:16].astype(np.int64))

    def stats_ring(self, replica, ring):
        """every step writes the replica's stats row into ring[step % len(ring)]
        (ring: pinned uint64 host memory, shape (slots, 16), e.g. a numpy view
        of torch.empty(..., pin_memory=True); word 6 of a row holds its step);
        None stops it"""
        if ring is None:
            check(self.lib.dpd_stats_ring(self.h, int(replica), None, 0))
            self._ring = None
            return
        assert ring.dtype == np.uint64 and ring.ndim == 2 and ring.shape[1] == 16 and ring.flags.c_contiguous
        check(self.lib.dpd_stats_ring(self.h, int(replica), ptr(ring), int(ring.shape[0])))
        self._ring = ring  # kept alive while the device writes into it

    def type_clusters(self, replica=0, type=2, rcut=1.0):
        """clusters of the beads of `type` joined within rcut, and their neighbour
        fraction within 1.0 (the reference's `snapcheck.py tclust`)"""
        out = np.zeros(6, np.int64)
        check(self.lib.dpd_type_clusters(self.h, int(replica), int(type), float(rcut), ptr(out)))
        n, nc, largest, sq, nb_all, nb_same = (int(v) for v in out)
        return dict(n=n, clusters=nc, largest=largest, sum_sq=sq, mean_size=sq / max(n, 1), nb_all=nb_all,
                    nb_same=nb_same, fraction=nb_same / max(nb_all, 1))

    def aggregates(self, replica=0, r_tail=1.0, min_lipids=12, labels=False):
        """molecules and membrane aggregates (the first stages of the reference's
        cell detection); labels: per bead in gid order the smallest gid of its
        aggregate (-1 for non-lipid beads)"""
        out = np.zeros(5, np.int64)
        lab = np.empty(self.n_beads[replica], np.int32) if labels else None
        check(self.lib.dpd_aggregates(self.h, int(replica), float(r_tail), int(min_lipids), ptr(out), ptr(lab)))
        res = dict(n_molecules=int(out[0]), n_aggregates=int(out[1]), n_membranes=int(out[2]),
                   lipids_in_small_aggregates=int(out[3]), largest_aggregate=int(out[4]))
        if labels:
            res["labels"] = lab
        return res

    def snapshot(self, replica=0):
        """the replica's current configuration as the reference's tools read a
        snapshot file (oercel_b200.cells.Snapshot: FP64 positions in gid order,
        wrapped into [0, L), types, bonds)"""
        from . import cells, cli
        p = self.params[replica]
        mol = p.template() if p.lip_arch != "linear" else None
        x, y, t, b = cli.snapshot_arrays(self.state(replica), mol)
        L = float(p.L)
        return cells.Snapshot(step=self.step_no, time=0.0, L=L, x=cells._wrap(x.astype(np.float64), L),
                              y=cells._wrap(y.astype(np.float64), L), type=t, bonds=b.astype(np.int64))

    def detect_cells(self, replica=0, cfg=None):
        """the reference's cell detection (cells.detect) on the replica's current
        configuration, without a snapshot file"""
        from . import cells
        return cells.detect(self.snapshot(replica), cfg)

    def pair_hist(self, replica, ta, tb, rmax, nbin):
        h = np.zeros(nbin)
        check(self.lib.dpd_pair_hist(self.h, replica, ta, tb, float(rmax), nbin, ptr(h)))
        return h

    # ---------------------------------------------------------------- parameters and reverse mode
    def set_params(self, replica, p: Params, **kv):
        """replace the parameters of one replica (same box); kv go to Params.to_struct
        (seed, warm_end, t_anchor, step_anchor)"""
        self.params[replica] = p
        check(self.lib.dpd_set_params(self.h, replica, C.byref(p.to_struct(**kv))))

    @staticmethod
    def rdf_spec(ta=2, tb=2, nbin=64, rmax=2.0, sigma=0.05, last_steps=50, horizon=0):
        return _capi.DpdRdfSpec(int(ta), int(tb), int(nbin), int(last_steps), float(rmax), float(sigma),
                                int(horizon), 0)

    def window_loss(self, nsteps, spec, target):
        """advance nsteps (chemistry off); per-replica loss and averaged g(r)"""
        tgt = np.ascontiguousarray(np.broadcast_to(target, (self.nrep, spec.nbin)), np.float64)
        loss = np.zeros(self.nrep)
        rdf = np.zeros((self.nrep, spec.nbin))
        check(self.lib.dpd_window_loss(self.h, int(nsteps), C.byref(spec), ptr(tgt), ptr(loss), ptr(rdf)))
        return loss, rdf

    def window_adjoint(self, nsteps, ckpt_every, spec, target):
        """window loss and its gradient (nrep x 66: a_ij upper triangle, gamma, k_bond)"""
        tgt = np.ascontiguousarray(np.broadcast_to(target, (self.nrep, spec.nbin)), np.float64)
        loss = np.zeros(self.nrep)
        rdf = np.zeros((self.nrep, spec.nbin))
        grad = np.zeros((self.nrep, _capi.NGRAD))
        check(self.lib.dpd_window_adjoint(self.h, int(nsteps), int(ckpt_every), C.byref(spec), ptr(tgt), ptr(loss),
                                          ptr(grad), ptr(rdf)))
        return loss, grad, rdf

    def fit_graph(self, keys, nsteps, ckpt_every, spec, target, iters, lr=1.0, betas=(0.9, 0.999), eps=1e-8):
        """iters optimizer iterations of the repulsions `keys` (a_X_Y, shared by
        every replica) replayed as one captured CUDA graph (dpd_fit_graph): each a
        differentiated window and an Adam step on the device.  Returns (loss
        (iters x nrep), summed gradient (iters x len(keys)), values the windows
        ran with, then the last values ((iters + 1) x len(keys))); the engine
        keeps the last values."""
        from .fit import param_index
        f = _capi.DpdFitSpec()
        f.n = len(keys)
        for k, key in enumerate(keys):
            f.slot[k] = param_index(key)
            if f.slot[k] >= 64:
                raise ValueError(f"{key}: only repulsions a_X_Y are fitted this way")
        f.lr, f.beta1, f.beta2, f.eps = float(lr), float(betas[0]), float(betas[1]), float(eps)
        tgt = np.ascontiguousarray(np.broadcast_to(target, (self.nrep, spec.nbin)), np.float64)
        loss = np.zeros((iters, self.nrep))
        grad = np.zeros((iters, len(keys)))
        vals = np.zeros((iters + 1, len(keys)))
        check(self.lib.dpd_fit_graph(self.h, int(nsteps), int(ckpt_every), C.byref(spec), ptr(tgt), C.byref(f),
                                     int(iters), ptr(loss), ptr(grad), ptr(vals)))
        for r in range(self.nrep):  # the host copies of the parameters follow the handle's
            for k, key in enumerate(keys):
                i, j = divmod(int(f.slot[k]), 8)
                self.params[r].a[i][j] = self.params[r].a[j][i] = float(vals[-1, k])
        return loss, grad, vals

    def window_adjoint_state(self, nsteps, ckpt_every, spec, target):
        """window_adjoint plus the cotangents of the start state (horizon 0):
        (loss, grad, rdf, xbar, vhbar, vtbar), the last three (N_total, 2) in gid
        order packed by replica (replica r's gid g at row sum(n_beads[:r]) + g)"""
        tgt = np.ascontiguousarray(np.broadcast_to(target, (self.nrep, spec.nbin)), np.float64)
        loss = np.zeros(self.nrep)
        rdf = np.zeros((self.nrep, spec.nbin))
        grad = np.zeros((self.nrep, _capi.NGRAD))
        N = int(sum(self.n_beads))
        st = [np.zeros((N, 2), np.float32) for _ in range(3)]
        check(self.lib.dpd_window_adjoint_state(self.h, int(nsteps), int(ckpt_every), C.byref(spec), ptr(tgt),
                                                ptr(loss), ptr(grad), ptr(rdf), *[ptr(a) for a in st]))
        return loss, grad, rdf, st[0], st[1], st[2]

    def force_vjp(self, replica, step, gx, gy):
        n = self.n_beads[replica]
        g = [np.ascontiguousarray(v, np.float32) for v in (gx, gy)]
        out = [np.empty(n, np.float32) for _ in range(4)]
        grad = np.zeros(_capi.NGRAD)
        check(self.lib.dpd_force_vjp(self.h, replica, int(step), ptr(g[0]), ptr(g[1]), *[ptr(o) for o in out],
                                     ptr(grad)))
        return out[0], out[1], out[2], out[3], grad

    def stream(self):
        s = C.c_void_p()
        check(self.lib.dpd_get_stream(self.h, C.byref(s)))
        return s.value

    def kernels_per_step(self):
        a, b = C.c_int32(), C.c_int32()
        check(self.lib.dpd_kernels_per_step(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value
