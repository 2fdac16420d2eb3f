"""The C ABI without a GPU: the library loads, exports exactly what include/dpd.h
declares, and its host-only routines behave (no compute call reaches a GPU here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
import oercel_b200 as ob
from oercel_b200 import _capi


def declared():
    src = open(os.path.join(ROOT, "include", "dpd.h")).read()
    return sorted(set(re.findall(r"^DPD_API\s+[\w\s\*]+?\b(dpd_\w+)\s*\(", src, flags=re.M)))


def test_header_and_binding_agree():
    assert declared() == sorted(_capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    for name in declared():
        assert hasattr(lib, name), name
    out = os.popen(f"nm -D --defined-only {_capi.LIB_PATH}").read()
    exported = set(re.findall(r" T (dpd_\w+)", out))
    assert exported == set(declared())


def test_params_default():
    p = _capi.DpdParams()
    assert _capi.load().dpd_params_default(p) == 0
    assert p.dt == 0.03 and p.lam == 0.65 and p.gamma == 4.5 and p.k_bond == 100.0 and p.r0 == 0.5
    assert p.noise == 0 and p.max_chain == 12


def test_host_soup_matches_reference():
    g = golden("soup_L32_seed0.npz")
    s = ob.make_soup(32.0, 4096, 0, nH=1, nT=2, f_lip=0.15, c_N=0.05)
    for k in ("x", "y", "vx", "vy"):
        assert np.array_equal(s[k], g[k]), k
    assert np.array_equal(s["type"], g["type"])
    assert np.array_equal(s["next"], g["nxt"])
    assert s["n_lipid_beads"] == 615


def test_host_soup_rejects_bad_composition():
    with pytest.raises(ob.DpdError):
        ob.make_soup(8.0, 100, 0, f_lip=0.9, c_N=0.5)


def test_errors_are_reported_not_fatal():
    lib = _capi.load()
    h = C.c_void_p()
    p = _capi.DpdParams()
    lib.dpd_params_default(p)
    p.L = 2.0  # too small
    n = (C.c_int32 * 1)(16)
    rc = lib.dpd_create(p, 1, n, C.byref(h))
    assert rc == -1 and b"L must be" in lib.dpd_last_error()
    p.L = 16.0
    p.a[1] = 30.0  # a_01 != a_10
    rc = lib.dpd_create(p, 1, n, C.byref(h))
    assert rc == -1 and b"symmetric" in lib.dpd_last_error()


def test_struct_layouts_agree_with_the_header(tmp_path):
    """the ctypes mirrors of the header's structs (and the numpy record of an
    event) have the C compiler's sizes and field offsets"""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    fields = {"dpd_event": ["step", "kind", "gid", "partner", "x", "y", "replica"],
              "dpd_fit_spec": ["n", "slot", "lr", "beta1", "beta2", "eps"],
              "dpd_rdf_spec": ["ta", "tb", "nbin", "last_steps", "rmax", "sigma", "horizon"],
              "dpd_tuning": ["force_kernel", "tile_w", "tile_h", "graph_steps", "sort_mode", "tile_threads"]}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dpd.h"', "int main(void) {"]
    for st, fs in fields.items():
        lines.append(f'printf("{st} %zu\\n", sizeof({st}));')
        for f in fs:
            lines.append(f'printf("{st}.{f} %zu\\n", offsetof({st}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    mirrors = {"dpd_event": _capi.DpdEvent, "dpd_fit_spec": _capi.DpdFitSpec, "dpd_rdf_spec": _capi.DpdRdfSpec,
               "dpd_tuning": _capi.DpdTuning}
    for st, cls in mirrors.items():
        assert int(got[st]) == C.sizeof(cls), st
        for f in fields[st]:
            assert int(got[f"{st}.{f}"]) == getattr(cls, f).offset, (st, f)
    rec = ob.Engine.EVENT_DTYPE
    assert rec.itemsize == C.sizeof(_capi.DpdEvent)
    for f in fields["dpd_event"]:
        assert rec.fields[f][1] == getattr(_capi.DpdEvent, f).offset, f
