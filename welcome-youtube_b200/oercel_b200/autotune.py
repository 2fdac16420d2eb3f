"""Autotuner of the launch choices of an Engine.

The knobs are those of dpd_tuning (include/dpd.h): which force kernel runs
(cell tiles in shared memory, one pair evaluation per pair, staged by per-bead
loads or by bulk asynchronous copies; or one thread per bead over its 3x3
cells), the tile shape in cells, and the
steps per captured CUDA graph.  Every candidate is timed on the live engine with real steps
(dpd_profile_step: CUDA events around each kernel of one step), so tuning
advances the simulation by a few steps; do it during equilibration.  Results
are cached per system shape in a JSON file.
"""
from __future__ import annotations

import json
import os

import numpy as np

FORCE_CANDIDATES = [
    dict(force_kernel=1),
    dict(force_kernel=0, tile_w=8, tile_h=16, tile_threads=256),
    dict(force_kernel=0, tile_w=14, tile_h=14, tile_threads=256),
    dict(force_kernel=0, tile_w=6, tile_h=30, tile_threads=256),
    dict(force_kernel=0, tile_w=10, tile_h=18, tile_threads=256),
    dict(force_kernel=0, tile_w=12, tile_h=13, tile_threads=256),
    dict(force_kernel=0, tile_w=9, tile_h=17, tile_threads=256),
    dict(force_kernel=0, tile_w=4, tile_h=8, tile_threads=256),
    dict(force_kernel=0, tile_w=2, tile_h=4, tile_threads=256),
    dict(force_kernel=0, tile_w=20, tile_h=20, tile_threads=512),
    dict(force_kernel=0, tile_w=14, tile_h=30, tile_threads=512),
    dict(force_kernel=0, tile_w=10, tile_h=40, tile_threads=512),
    dict(force_kernel=2, tile_w=14, tile_h=14),
    dict(force_kernel=2, tile_w=8, tile_h=16),
    dict(force_kernel=2, tile_w=6, tile_h=30),
    dict(force_kernel=2, tile_w=10, tile_h=18),
    dict(force_kernel=2, tile_w=4, tile_h=8),
]

# 12 x 13 and 9 x 17 cells give 1720 and 1767 tiles on a 512 x 512 grid, just under three full
# rounds of 4 CTAs on 148 SMs (1776)

# the cell sort: 0 two scan passes, 1 one scan pass with decoupled look-back, 2 a block-local
# scan whose block prefixes the placement and fix-up kernels add themselves
SORT_CANDIDATES = [0, 1, 2]


def _key(engine):
    sizes = sorted(engine.n_beads)
    return f"n{len(sizes)}_sum{sum(sizes)}_min{sizes[0]}_max{sizes[-1]}"


def default_cache():
    return os.path.join(os.path.expanduser("~"), ".cache", "oercel_b200", "tune.json")


def autotune(engine, repeats=3, candidates=None, cache_path=None, use_cache=True):
    """pick and apply the fastest force kernel / tile shape; returns the choice"""
    cache_path = cache_path or default_cache()
    key = _key(engine)
    cache = {}
    if use_cache and os.path.exists(cache_path):
        try:
            cache = json.load(open(cache_path))
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        engine.set_tuning(**cache[key]["tuning"])
        return cache[key]
    best, timings = None, []
    for cand in candidates or FORCE_CANDIDATES:
        try:
            engine.set_tuning(**cand)
        except Exception:
            continue
        engine.profile_step()  # first launch of this variant
        ms = float(np.median([engine.profile_step()[-1] for _ in range(repeats)]))
        timings.append(dict(cand, forces_ms=ms))
        if best is None or ms < best[1]:
            best = (cand, ms)
    engine.set_tuning(**best[0])
    # the scan of the cell counts: two passes or one pass with look-back (the
    # first four kernel times of a step: scan1, scan2, place, cellfix)
    sort_best, sort_timings = None, []
    for mode in SORT_CANDIDATES:
        engine.set_tuning(sort_mode=mode)
        engine.profile_step()
        ms = float(np.median([sum(engine.profile_step()[:4]) for _ in range(repeats)]))
        sort_timings.append(dict(sort_mode=mode, sort_ms=ms))
        if sort_best is None or ms < sort_best[1]:
            sort_best = (mode, ms)
    engine.set_tuning(sort_mode=sort_best[0])
    out = {"tuning": engine.tuning(), "forces_ms": best[1], "timings": timings, "sort_ms": sort_best[1],
           "sort_timings": sort_timings}
    if use_cache:
        cache[key] = out
        try:
            os.makedirs(os.path.dirname(cache_path), exist_ok=True)
            json.dump(cache, open(cache_path, "w"), indent=1)
        except OSError:
            pass
    return out
