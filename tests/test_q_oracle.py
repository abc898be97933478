"""The (Q) task-loop oracle on the CPU: its task list is the reference's
(distr_cc/rccsdt_q.py:302-314), it is invariant under the block size (the
factor weights make every a<=b<=c<=d quadruple count once) and the grouped
contraction order of dcc.rccsdt_q matches it (group and task sets agree)."""
import numpy as np
import pytest

from oracle import q_ref
from dcc import rccsdt_q as gq


def _inputs(no, nv, seed):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    g = rng.standard_normal((nmo,) * 4) * 0.1
    perms = [(0, 1, 2, 3), (1, 0, 2, 3), (0, 1, 3, 2), (1, 0, 3, 2), (2, 3, 0, 1), (3, 2, 0, 1), (2, 3, 1, 0),
             (3, 2, 1, 0)]
    g = sum(g.transpose(p) for p in perms) / 8
    phys = g.transpose(0, 2, 1, 3)  # <pq|rs> = (pr|qs)
    o, v = slice(0, no), slice(no, nmo)
    er = {"vvvo": phys[v, v, v, o].copy(), "vooo": phys[v, o, o, o].copy(), "vvoo": phys[v, v, o, o].copy(),
          "ovvo": phys[o, v, v, o].copy(), "ovov": phys[o, v, o, v].copy(), "vvvv": phys[v, v, v, v].copy(),
          "oooo": phys[o, o, o, o].copy()}
    t2 = rng.standard_normal((nv, nv, no, no)) * 0.05
    t2 = 0.5 * (t2 + t2.transpose(1, 0, 3, 2))
    full = rng.standard_normal((nv,) * 3 + (no,) * 3) * 0.01
    import itertools
    T = sum(full.transpose(p + tuple(3 + x for x in p)) for p in itertools.permutations(range(3))) / 6
    e_occ = np.sort(rng.uniform(-1.5, -0.3, no))
    e_vir = np.sort(rng.uniform(0.1, 3.0, nv))
    return er, t2, T, e_occ, e_vir


def test_task_lists_match():
    for nv, blk in [(7, 2), (9, 4), (10, 3)]:
        assert q_ref.task_list(nv, blk) == gq.task_list(nv, blk)
        from_groups = sorted((a0, a1, b0, b1, c0, c1, d0, d1) for (a0, a1, b0, b1, c0, c1) in gq.groups(nv, blk)
                             for d0, d1 in gq.prange(c0, nv, blk))
        ref = sorted((t[0], t[1], t[3], t[4], t[6], t[7], t[9], t[10]) for t in q_ref.task_list(nv, blk))
        assert from_groups == ref


def test_energy_independent_of_block_size(oracle):
    no, nv = 2, 5
    er, t2, T, eo, ev = _inputs(no, nv, 3)
    e1 = q_ref.q_energy_ref(er, t2, T, eo, ev, 1, oracle)
    e2 = q_ref.q_energy_ref(er, t2, T, eo, ev, 2, oracle)
    e3 = q_ref.q_energy_ref(er, t2, T, eo, ev, 3, oracle)
    assert abs(e1[0]) > 0 and abs(e1[1]) > 0
    for a, b in ((e1, e2), (e1, e3)):
        np.testing.assert_allclose(a, b, rtol=1e-11, atol=1e-14)


def test_lazy_t3_slices():
    """tests/lazy_t3.LazyT (used at the benzene shape) gives the same slices as the full T."""
    from lazy_t3 import LazyT
    no, nv = 4, 7
    _, _, T, _, _ = _inputs(no, nv, 3)
    trip = [(i, j, k) for i in range(no) for j in range(i, no) for k in range(j, no)]
    t3 = np.stack([T[:, :, :, i, j, k] for i, j, k in trip])
    L = LazyT(t3, no)
    assert L.shape == T.shape
    for A, B in ((slice(0, 2), slice(2, 4)), (slice(4, 7), slice(0, 3)), (slice(6, 7), slice(6, 7))):
        np.testing.assert_allclose(L[A, B], T[A, B], rtol=0, atol=1e-15)  # T is symmetric to rounding
