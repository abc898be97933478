"""Project-written autotuner for the split-precision GEMM pipeline shape.

The kernel's k-block width (128/64/32 bytes of K with the matching swizzle),
ring depth and raster group height are runtime choices
(dcc_gemm_set_config).  `tune(key, run)` times every candidate on the actual
problem with CUDA events, keeps the fastest, and caches the choice per key
(problem shape and precision) for the process; `use(key)` re-applies it.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L

_set = L.bind("dcc_gemm_set_config", [L.c_int, L.c_int, L.c_int])
_get = L.bind("dcc_gemm_get_config", [L.c_vp, L.c_vp, L.c_vp])

PIPELINES = [(128, 2), (64, 4), (64, 3), (32, 8)]
GROUPS = [8, 16, 32]
_cache = {}


def set_config(kb_bytes, stages, group_m):
    L.check(_set(kb_bytes, stages, group_m))


def get_config():
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.check(_get(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return a.value, b.value, c.value


def candidates():
    return [(kb, st, g) for kb, st in PIPELINES for g in GROUPS]


def tune(key, run, reps=2, cands=None):
    """Time run() under each candidate configuration; keep and return the fastest."""
    if key in _cache:
        set_config(*_cache[key])
        return _cache[key]
    best, best_ms = None, float("inf")
    for cfg in (cands or candidates()):
        set_config(*cfg)
        run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        if ms < best_ms:
            best, best_ms = cfg, ms
    _cache[key] = best
    set_config(*best)
    return best


def use(key):
    if key in _cache:
        set_config(*_cache[key])
        return _cache[key]
    return None
