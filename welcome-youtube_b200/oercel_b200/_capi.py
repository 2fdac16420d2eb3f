"""ctypes binding of libdpd.so (include/dpd.h).

The library is the product: there is no Python or CPU implementation of the
step behind this module.  Loading fails loudly when libdpd.so is missing, and
every call that returns a negative code raises DpdError with the library's
message.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdpd.so")
MAXT = 8

ERRORS = {
    -1: "DPD_E_ARG", -2: "DPD_E_CUDA", -3: "DPD_E_SORT_OVERFLOW", -4: "DPD_E_CHAIN",
    -5: "DPD_E_EVENT_OVERFLOW", -6: "DPD_E_TIMEOUT", -7: "DPD_E_STATE", -8: "DPD_E_NOMEM",
}


class DpdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class DpdParams(C.Structure):
    _fields_ = [
        ("L", C.c_double), ("dt", C.c_double), ("lam", C.c_double), ("gamma", C.c_double), ("kT", C.c_double),
        ("a", C.c_double * (MAXT * MAXT)), ("k_bond", C.c_double), ("r0", C.c_double), ("seed", C.c_uint64),
        ("noise", C.c_int32), ("chem", C.c_int32), ("n_chem", C.c_int32), ("n_t_min", C.c_int32),
        ("max_chain", C.c_int32), ("pad", C.c_int32),
        ("p_break", C.c_double), ("p_grow", C.c_double), ("p_bond", C.c_double),
        ("r_grow", C.c_double), ("r_bond", C.c_double), ("warmup", C.c_int64), ("warm_end", C.c_int64),
        ("k_angle", C.c_double), ("stir_A", C.c_double), ("stir_n", C.c_int32), ("pad2", C.c_int32),
        ("kT_amp", C.c_double), ("kT_period", C.c_double), ("t_anchor", C.c_double), ("step_anchor", C.c_int64),
        ("chem_kind", C.c_int32), ("syn_tries", C.c_int32), ("syn_relax", C.c_int32), ("syn_nN", C.c_int32),
        ("lip_nH", C.c_int32), ("lip_nT", C.c_int32), ("feed_mode", C.c_int32), ("vent_kind", C.c_int32),
        ("r_cat", C.c_double), ("p_syn_a", C.c_double), ("p_syn_b", C.c_double), ("p_rep_a", C.c_double),
        ("p_rep_b", C.c_double), ("mu", C.c_double), ("p_ld", C.c_double), ("p_kd", C.c_double),
        ("p_nd", C.c_double), ("p_feed", C.c_double), ("feed_cap", C.c_double), ("vent_x", C.c_double),
        ("vent_y", C.c_double), ("vent_r", C.c_double), ("vent_w", C.c_double),
        ("lip_arch", C.c_int32), ("lip_tie", C.c_int32), ("r0_head", C.c_double), ("k_head", C.c_double),
        ("cos_head", C.c_double),
    ]


MAXML = 16
MAXMB = 2 * MAXML


class DpdTemplate(C.Structure):
    _fields_ = [
        ("arch", C.c_int32), ("mlen", C.c_int32), ("nH", C.c_int32), ("nb", C.c_int32), ("na", C.c_int32),
        ("pad", C.c_int32), ("bi", C.c_int32 * MAXMB), ("bj", C.c_int32 * MAXMB), ("br0", C.c_double * MAXMB),
        ("ai", C.c_int32 * MAXMB), ("aj", C.c_int32 * MAXMB), ("ak", C.c_int32 * MAXMB),
        ("akind", C.c_int32 * MAXMB), ("aK", C.c_double * MAXMB), ("ac0", C.c_double * MAXMB),
        ("px", C.c_double * MAXML), ("py", C.c_double * MAXML), ("ix", C.c_double * MAXML),
        ("iy", C.c_double * MAXML),
    ]


class DpdTuning(C.Structure):
    _fields_ = [("force_kernel", C.c_int32), ("tile_w", C.c_int32), ("tile_h", C.c_int32),
                ("graph_steps", C.c_int32), ("sort_mode", C.c_int32), ("tile_threads", C.c_int32)]


class DpdFitSpec(C.Structure):
    _fields_ = [("n", C.c_int32), ("pad", C.c_int32), ("slot", C.c_int32 * 64), ("lr", C.c_double),
                ("beta1", C.c_double), ("beta2", C.c_double), ("eps", C.c_double)]


class DpdRdfSpec(C.Structure):
    _fields_ = [("ta", C.c_int32), ("tb", C.c_int32), ("nbin", C.c_int32), ("last_steps", C.c_int32),
                ("rmax", C.c_double), ("sigma", C.c_double), ("horizon", C.c_int32), ("pad", C.c_int32)]


class DpdCellsCfg(C.Structure):
    _fields_ = [("r_tail", C.c_double), ("h", C.c_double), ("r_stamp", C.c_double),
                ("min_membrane_lipids", C.c_int32), ("pad0", C.c_int32),
                ("min_lumen_area", C.c_double), ("min_aqueous_frac", C.c_double), ("rho", C.c_double),
                ("pad", C.c_double), ("leaflet_in", C.c_double), ("leaflet_max", C.c_double),
                ("min_exposure", C.c_double), ("wall_extra", C.c_double), ("inner_frac_lo", C.c_double),
                ("inner_frac_hi", C.c_double)]


CELL_COLS = 20


class DpdEvent(C.Structure):
    _fields_ = [("step", C.c_int64), ("kind", C.c_int32), ("gid", C.c_uint32), ("partner", C.c_uint32),
                ("x", C.c_float), ("y", C.c_float), ("replica", C.c_int32)]


EXPORTS = [
    "dpd_last_error", "dpd_version", "dpd_params_default", "dpd_create", "dpd_destroy", "dpd_sizes",
    "dpd_set_state", "dpd_get_state", "dpd_set_dynamics", "dpd_prime", "dpd_resume", "dpd_get_step",
    "dpd_set_step", "dpd_step", "dpd_init_soup", "dpd_build_cells", "dpd_get_cells", "dpd_forces",
    "dpd_pair_forces", "dpd_bond_forces", "dpd_integrate", "dpd_chemistry", "dpd_get_events", "dpd_events_async",
    "dpd_observables", "dpd_pair_hist", "dpd_get_stream", "dpd_kernels_per_step", "dpd_step_async",
    "dpd_sync", "dpd_set_graph_steps", "dpd_profile_step", "dpd_stats", "dpd_set_tuning", "dpd_get_tuning",
    "dpd_sort_cells_noalloc", "dpd_set_params", "dpd_window_loss", "dpd_window_adjoint", "dpd_window_adjoint_state",
    "dpd_fit_graph",
    "dpd_force_vjp",
    "dpd_set_rng", "dpd_get_rng", "dpd_lipid_template", "dpd_type_clusters", "dpd_xoshiro_jump",
    "dpd_aggregates", "dpd_stats_async", "dpd_stats_decode", "dpd_stats_ring", "dpd_cells_default",
    "dpd_cells_detect",
    "dpd_cells_info", "dpd_cells_fetch", "dpd_cells_free",
]
NGRAD = 66

_lib = None


def load(path: str | None = None):
    """Load libdpd.so (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("DPD_LIB") or LIB_PATH
    if path == LIB_PATH:
        try:
            import importlib.util
            spec = importlib.util.spec_from_file_location("_dpd_build", os.path.join(os.path.dirname(HERE),
                                                                                       "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            if mod.stale() and os.path.exists("/usr/local/cuda/bin/nvcc"):
                mod.build()
        except FileNotFoundError:
            pass
    if not os.path.exists(path):
        raise OSError(f"libdpd.so not found at {path}: build it with welcome-youtube_b200/build.py")
    lib = C.CDLL(path)
    vp = C.c_void_p
    fp = C.c_void_p  # data pointers are passed as integers (host or device)
    i32, i64, u64, dbl = C.c_int32, C.c_int64, C.c_uint64, C.c_double
    sig = {
        "dpd_last_error": ([], C.c_char_p),
        "dpd_version": ([], C.c_char_p),
        "dpd_params_default": ([C.POINTER(DpdParams)], C.c_int),
        "dpd_create": ([C.POINTER(DpdParams), i32, C.POINTER(C.c_int32), C.POINTER(vp)], C.c_int),
        "dpd_destroy": ([vp], C.c_int),
        "dpd_sizes": ([vp, i32, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
        "dpd_set_state": ([vp, i32] + [fp] * 8, C.c_int),
        "dpd_get_state": ([vp, i32] + [fp] * 12, C.c_int),
        "dpd_set_dynamics": ([vp, i32] + [fp] * 6, C.c_int),
        "dpd_prime": ([vp], C.c_int),
        "dpd_resume": ([vp], C.c_int),
        "dpd_get_step": ([vp, C.POINTER(C.c_int64)], C.c_int),
        "dpd_set_step": ([vp, i64], C.c_int),
        "dpd_step": ([vp, i64], C.c_int),
        "dpd_init_soup": ([dbl, i32, u64, dbl, dbl, i32, i32, dbl, dbl, dbl, dbl] + [fp] * 7
                          + [C.POINTER(C.c_int32), fp, C.POINTER(DpdTemplate)], C.c_int),
        "dpd_lipid_template": ([C.POINTER(DpdParams), C.POINTER(DpdTemplate)], C.c_int),
        "dpd_type_clusters": ([vp, i32, i32, dbl, fp], C.c_int),
        "dpd_xoshiro_jump": ([fp, u64, fp], C.c_int),
        "dpd_aggregates": ([vp, i32, dbl, i32, fp, fp], C.c_int),
        "dpd_stats_async": ([vp, i32, fp], C.c_int),
        "dpd_stats_decode": ([vp, i32, fp, fp], C.c_int),
        "dpd_stats_ring": ([vp, i32, fp, i32], C.c_int),
        "dpd_set_rng": ([vp, i32, fp], C.c_int),
        "dpd_get_rng": ([vp, i32, fp], C.c_int),
        "dpd_build_cells": ([vp], C.c_int),
        "dpd_get_cells": ([vp, i32, fp], C.c_int),
        "dpd_forces": ([vp, i64], C.c_int),
        "dpd_pair_forces": ([vp, i32, i64, fp, fp], C.c_int),
        "dpd_bond_forces": ([vp, i32, fp, fp, C.POINTER(C.c_float)], C.c_int),
        "dpd_integrate": ([vp], C.c_int),
        "dpd_chemistry": ([vp, i64], C.c_int),
        "dpd_get_events": ([vp, C.POINTER(DpdEvent), i32, C.POINTER(C.c_int32)], C.c_int),
        "dpd_events_async": ([vp, vp, i32, vp], C.c_int),
        "dpd_observables": ([vp, i32, fp], C.c_int),
        "dpd_stats": ([vp, i32, fp], C.c_int),
        "dpd_set_tuning": ([vp, C.POINTER(DpdTuning)], C.c_int),
        "dpd_get_tuning": ([vp, C.POINTER(DpdTuning)], C.c_int),
        "dpd_sort_cells_noalloc": ([fp, fp, i32, dbl, fp, fp, vp], C.c_int),
        "dpd_set_params": ([vp, i32, C.POINTER(DpdParams)], C.c_int),
        "dpd_window_loss": ([vp, i64, C.POINTER(DpdRdfSpec), fp, fp, fp], C.c_int),
        "dpd_window_adjoint": ([vp, i64, i32, C.POINTER(DpdRdfSpec), fp, fp, fp, fp], C.c_int),
        "dpd_window_adjoint_state": ([vp, i64, i32, C.POINTER(DpdRdfSpec), fp, fp, fp, fp, fp, fp, fp], C.c_int),
        "dpd_fit_graph": ([vp, i64, i32, C.POINTER(DpdRdfSpec), fp, C.POINTER(DpdFitSpec), i32, fp, fp, fp], C.c_int),
        "dpd_force_vjp": ([vp, i32, i64, fp, fp, fp, fp, fp, fp, fp], C.c_int),
        "dpd_pair_hist": ([vp, i32, i32, i32, dbl, i32, fp], C.c_int),
        "dpd_get_stream": ([vp, C.POINTER(vp)], C.c_int),
        "dpd_kernels_per_step": ([vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
        "dpd_step_async": ([vp, i64], C.c_int),
        "dpd_sync": ([vp], C.c_int),
        "dpd_set_graph_steps": ([vp, i32], C.c_int),
        "dpd_profile_step": ([vp, C.POINTER(C.c_float), i32, C.POINTER(C.c_int32)], C.c_int),
        "dpd_cells_default": ([C.POINTER(DpdCellsCfg)], C.c_int),
        "dpd_cells_detect": ([C.POINTER(DpdCellsCfg), dbl, i64, fp, fp, fp, i64, fp, C.POINTER(vp)], C.c_int),
        "dpd_cells_info": ([vp, fp, C.POINTER(C.c_double)], C.c_int),
        "dpd_cells_fetch": ([vp, fp, fp, fp, i32, fp, fp, fp], C.c_int),
        "dpd_cells_free": ([vp], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def check(rc: int):
    if rc != 0:
        raise DpdError(rc, load().dpd_last_error().decode(errors="replace"))
    return rc


def ptr(a) -> int | None:
    """data pointer of a numpy array or torch tensor (None passes NULL)"""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")
