"""Device DIIS for the unified T1/T2/T3 amplitude vector
(distr_cc/diis.py:25-177, driven as in run_diis_t3, distr_cc/rccsdt.py:1026-1067).

The vector is the concatenation of up to four device amplitude segments,
each starting on a multiple of 32 elements (vector_layout; the gaps are zero,
so the passes move aligned 16-byte pairs) and multiplied by its scale (the reference scales the packed unique T1/T2
by 1/sqrt(nranks) and appends t3_local[:, :nd, :nd, :nd]).  Slots live in
device memory; one update is two single passes over the vector
(dcc_diis_push: error vector, slot copies and the new B-matrix row;
dcc_diis_combine: extrapolation, update norm, and the unpack back into the
segments, divided by their scales) plus the (space+1)^2 host solve the
reference does with numpy.

Out-of-core slots.  The reference can keep the slots from index scratch_start on in .npy
files and read them back each update (distr_cc/diis.py:25-103).  Here those slots live in
pinned host memory instead, and the two passes read and write them in place through their
unified addresses, over the host link: HBM then holds only scratch_start (x, e) slot pairs.
At 180 GB of HBM the slots of a 1.3 GB T3 vector fit on the device, so the default keeps
every slot there."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L

f64 = torch.float64

_push = L.bind("dcc_diis_push", [L.c_vp, L.c_vp, L.c_vp, L.c_int, L.c_vp, L.c_vp, L.c_vp, L.c_vp, L.c_int, L.c_vp,
                                 L.c_vp, ctypes.c_size_t, L.c_vp])
_combine = L.bind("dcc_diis_combine", [L.c_vp, L.c_vp, L.c_int, L.c_vp, L.c_vp, L.c_vp, L.c_vp, L.c_int, L.c_vp,
                                       L.c_vp, ctypes.c_size_t, L.c_vp])
_veclen = L.bind("dcc_diis_vector_length", [L.c_vp, L.c_int, L.c_vp], restype=ctypes.c_int64)


def vector_layout(lengths):
    """(total length, segment offsets) of the DIIS vector for segments of these lengths: each
    segment starts on a multiple of 32 elements, the gaps are zero."""
    n = len(lengths)
    seg_n = (ctypes.c_int64 * n)(*[int(x) for x in lengths])
    off = (ctypes.c_int64 * n)()
    total = int(_veclen(seg_n, n, off))
    if total < 0:
        raise L.DccError(2, L.last_error())
    return total, list(off)


class DIIS:
    """update(segments, scales) extrapolates in place; the first call only records x_prev."""

    def __init__(self, space=6, device="cuda", scratch_start=None):
        self.space = int(space)
        if self.space <= 0 or self.space > 16:
            raise ValueError("DIIS space must be in 1..16")
        self.dev = device
        # Slots with index >= scratch_start in pinned host memory (clamped to 0..space as
        # distr_cc/diis.py:44 does); None keeps every slot in HBM.
        self.scratch_start = self.space if scratch_start is None else max(0, min(int(scratch_start), self.space))
        self.reset()

    def _slot(self, idx, n):
        if idx >= self.scratch_start:
            return torch.empty(n, dtype=f64, pin_memory=True)
        return torch.empty(n, dtype=f64, device=self.dev)

    def reset(self):
        self.xs, self.es = [None] * self.space, [None] * self.space
        self._head, self._H, self._xprev = 0, None, None
        self.last_delta_norm_sq = None
        self._filled = [False] * self.space
        nbytes = int(L.lib().dcc_diis_workspace_bytes())
        self._ws = torch.empty((nbytes + 7) // 8, dtype=f64, device=self.dev)
        self._dots = torch.empty(self.space + 1, dtype=f64, device=self.dev)
        self._delta = torch.empty(1, dtype=f64, device=self.dev)
        return self

    @staticmethod
    def _segs(segments, scales):
        if not 1 <= len(segments) <= 4:
            raise ValueError("1..4 amplitude segments")
        scales = [1.0] * len(segments) if scales is None else [float(s) for s in scales]
        for t in segments:
            L.as_tensor(t, f64, "segment")
        ptr = (ctypes.c_void_p * len(segments))(*[t.data_ptr() for t in segments])
        num = (ctypes.c_int64 * len(segments))(*[t.numel() for t in segments])
        sc = (ctypes.c_double * len(segments))(*scales)
        return ptr, num, sc, scales, sum(t.numel() for t in segments)

    def update(self, segments, scales=None):
        ptr, num, sc, scales, _ = self._segs(segments, scales)
        n, offs = vector_layout([t.numel() for t in segments])
        if self._xprev is None:
            self._xprev = torch.zeros(n, dtype=f64, device=self.dev)
            for t, s, o in zip(segments, scales, offs):
                self._xprev[o:o + t.numel()] = t.reshape(-1) * s
            self.last_delta_norm_sq = None
            return segments
        if self._xprev.numel() != n:
            raise ValueError("DIIS vector length changed")
        h = self._head
        if self.xs[h] is None:
            self.xs[h] = self._slot(h, n)
            self.es[h] = self._slot(h, n)
        others = [i for i in range(self.space) if self._filled[i] and i != h]
        optr = (ctypes.c_void_p * max(1, len(others)))(*[self.es[i].data_ptr() for i in others])
        L.check(_push(ptr, num, sc, len(segments), L.ptr(self._xprev), L.ptr(self.xs[h]), L.ptr(self.es[h]), optr,
                      len(others), L.ptr(self._dots), L.ptr(self._ws), self._ws.numel() * 8, L.stream_ptr()))
        self._filled[h] = True
        nd = sum(self._filled)
        dots = self._dots[:len(others) + 1].cpu().numpy()
        row = np.zeros(nd)
        for j, i in enumerate(others):
            row[i] = dots[j]
        row[h] = dots[len(others)]
        if self._H is None:
            self._H = np.zeros((self.space + 1, self.space + 1))
            self._H[0, 1:] = self._H[1:, 0] = 1
        for i, val in enumerate(row):
            self._H[h + 1, i + 1] = val
            self._H[i + 1, h + 1] = val
        self._head = (h + 1) % self.space
        c = self.coefficients(nd)
        xptr = (ctypes.c_void_p * nd)(*[self.xs[i].data_ptr() for i in range(nd)])
        coef = (ctypes.c_double * nd)(*[float(x) for x in c[1:]])
        L.check(_combine(xptr, coef, nd, L.ptr(self._xprev), ptr, num, sc, len(segments), L.ptr(self._delta),
                         L.ptr(self._ws), self._ws.numel() * 8, L.stream_ptr()))
        self.last_delta_norm_sq = max(float(self._delta.item()), 0.0)
        return segments

    def coefficients(self, nd):
        """The extrapolation coefficients of distr_cc/diis.py:155-170 (eigh with a 1e-14 cut, else solve)."""
        hm = self._H[:nd + 1, :nd + 1]
        g = np.zeros(nd + 1)
        g[0] = 1
        w, v = np.linalg.eigh(hm)
        if np.any(abs(w) < 1e-14):
            idx = abs(w) > 1e-14
            return np.dot(v[:, idx] * (1 / w[idx]), np.dot(v[:, idx].T, g))
        return np.linalg.solve(hm, g)
