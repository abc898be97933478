"""TEST ORACLE ONLY -- numpy restatement of the reference's DIIS update
(distr_cc/diis.py:105-177: circular slots, B-matrix rows of error-vector dot
products, eigh with a 1e-14 cut or solve, x_new = sum_i c_i x_i, and the
|x_new - x_prev|^2 update norm of distr_cc/_runtime.py:90).  One rank, in
memory, no scratch files."""
from __future__ import annotations

import numpy as np


class DIISRef:
    def __init__(self, space=6):
        self.space = int(space)
        self.xs, self.es = [None] * self.space, [None] * self.space
        self._head, self._H, self._xprev = 0, None, None
        self.last_delta_norm_sq = None

    def update(self, x):
        x = np.asarray(x, dtype=np.float64).reshape(-1)
        if self._xprev is None:
            self._xprev = x.copy()
            self.last_delta_norm_sq = None
            return x
        err = x - self._xprev
        self.xs[self._head], self.es[self._head] = x, err
        nd = sum(v is not None for v in self.xs)
        if self._H is None:
            self._H = np.zeros((self.space + 1, self.space + 1))
            self._H[0, 1:] = self._H[1:, 0] = 1
        row = np.array([np.dot(err, err if i == self._head else self.es[i]) for i in range(nd)])
        for i, val in enumerate(row):
            self._H[self._head + 1, i + 1] = val
            self._H[i + 1, self._head + 1] = val
        self._head = (self._head + 1) % self.space
        h = self._H[:nd + 1, :nd + 1]
        g = np.zeros(nd + 1)
        g[0] = 1
        w, v = np.linalg.eigh(h)
        if np.any(abs(w) < 1e-14):
            idx = abs(w) > 1e-14
            c = np.dot(v[:, idx] * (1 / w[idx]), np.dot(v[:, idx].T, g))
        else:
            c = np.linalg.solve(h, g)
        xnew = np.zeros_like(x)
        for i, ci in enumerate(c[1:]):
            xnew += self.xs[i] * ci
        d = xnew - self._xprev
        self.last_delta_norm_sq = max(float(np.dot(d, d)), 0.0)
        self._xprev = xnew.copy()
        return xnew
