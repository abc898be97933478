"""T3 of every ordering, T[a, b, c, i, j, k], read lazily from the canonical i <= j <= k
blocks: the oracle's (Q) task loop (oracle/q_ref.py) only takes slices T[A, B] of two
virtual ranges, so at the benzene shape (nocc=15, nvir=93: 21.7 GB for the full tensor)
each slice is built from the 4.4 GB of canonical blocks when asked for."""
from __future__ import annotations

import itertools

import numpy as np


class LazyT:
    def __init__(self, t3, nocc):
        """t3: host array [n3, nv, nv, nv] of the canonical blocks in lexicographic order."""
        self.t3, self.no = t3, nocc
        nv = t3.shape[1]
        self.shape = (nv, nv, nv, nocc, nocc, nocc)
        trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
        self.index = {t: q for q, t in enumerate(trip)}

    def __getitem__(self, key):
        A, B = key
        no, nv = self.no, self.shape[0]
        na, nb = len(range(nv)[A]), len(range(nv)[B])
        out = np.empty((na, nb, nv, no, no, no))
        for o in itertools.product(range(no), repeat=3):
            # T[o][a0, a1, a2] = C[a_pi(0), a_pi(1), a_pi(2)] for the canonical block C of
            # sorted(o) = (o[pi(0)], o[pi(1)], o[pi(2)]) (the simultaneous permutation symmetry)
            pi = sorted(range(3), key=lambda r: o[r])
            C = self.t3[self.index[tuple(o[p] for p in pi)]]
            out[:, :, :, o[0], o[1], o[2]] = C.transpose(np.argsort(pi))[A, B, :]
        return out
