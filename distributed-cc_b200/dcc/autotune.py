"""Project-written autotuner for the split-precision GEMM tile and pipeline shape.

The kernel's output tile (128 x 256, one CTA per SM, or 128 x 128, two CTAs per
SM), k-block width (128/64/32 bytes of K with the matching swizzle), ring depth
and raster group height are runtime choices (dcc_gemm_set_tile_config).  A
configuration is (k-block bytes, stages, group, tile columns).  `tune(key,
run)` times every candidate on the actual problem with CUDA events, keeps the
fastest, and caches the choice per key (problem shape and precision) for the
process; `use(key)` re-applies it and `applied(key)` applies it around a block.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L

_set = L.bind("dcc_gemm_set_tile_config", [L.c_int, L.c_int, L.c_int, L.c_int])
_get = L.bind("dcc_gemm_get_tile_config", [L.c_vp, L.c_vp, L.c_vp, L.c_vp])

# (k-block bytes, stages) of the 128 x 256 tile; the 128 x 128 tile has one pipeline (64, 2)
PIPELINES = [(128, 2), (64, 4), (64, 3), (32, 8)]
NARROW = (64, 2)
GROUPS = [8, 16, 32]
_cache = {}
_times = {}


def set_config(kb_bytes, stages, group_m, tile_n=256):
    L.check(_set(kb_bytes, stages, group_m, tile_n))


def get_config():
    a, b, c, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.check(_get(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)))
    return a.value, b.value, c.value, d.value


def candidates():
    """Every (k-block bytes, stages, group, tile columns) configuration."""
    return [(kb, st, g, 256) for kb, st in PIPELINES for g in GROUPS] + [NARROW + (g, 128) for g in GROUPS]


def tile_candidates():
    """The configurations that differ for a contraction of K <= 4096 or an FP32 output (on 128 x 256
    tiles those run a fixed pipeline with eight epilogue warps): the tile width and the raster
    group."""
    return [(64, 3, g, 256) for g in GROUPS] + [NARROW + (g, 128) for g in GROUPS]


class applied:
    """Context manager: run a block under the configuration tuned for `key` (when there is one)
    and restore the previous configuration afterwards, so that it does not leak into later
    untuned GEMMs."""

    def __init__(self, key):
        self.key = key

    def __enter__(self):
        self.old = get_config()
        use(self.key)
        return self

    def __exit__(self, *exc):
        set_config(*self.old)
        return False


def tune(key, run, reps=2, cands=None, rounds=3):
    """Time run() under each candidate configuration; keep and return the fastest.

    Every candidate runs once untimed, then `rounds` rounds time each candidate over `reps`
    runs, the order reversed every other round, and a candidate's time is its best round.
    Under the power cap the SM clock drifts during tuning; interleaving the candidates
    spreads that drift over all of them instead of favouring the first ones timed."""
    if key in _cache:
        set_config(*_cache[key])
        return _cache[key]
    cands = list(cands or candidates())
    for cfg in cands:
        set_config(*cfg)
        run()
    best_ms = {cfg: float("inf") for cfg in cands}
    for r in range(rounds):
        for cfg in (cands if r % 2 == 0 else cands[::-1]):
            set_config(*cfg)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            best_ms[cfg] = min(best_ms[cfg], e0.elapsed_time(e1) / reps)
    best = min(cands, key=lambda c: best_ms[c])
    _cache[key], _times[key] = best, best_ms
    set_config(*best)
    return best


def chosen(key):
    """The configuration tuned for `key` (None if it was not)."""
    return _cache.get(key)


def timings(key):
    """{candidate: best ms per run()} measured when `key` was tuned (None if it was not)."""
    return _times.get(key)


def use(key):
    if key in _cache:
        set_config(*_cache[key])
        return _cache[key]
    return None
