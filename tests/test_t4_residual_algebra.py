"""compute_r4_tri without its OO batch: the full-ordered-space formulation of
dcc.t4_residual (every per-block string as one einsum over all orderings of
(i,j,k,l), W_oovvvv kept for every ordered pair) against the oracle's literal
per-block loop (oracle/t4_ref.py), in FP64 on the CPU, relative 1e-12.  The
P3_201 / P4_201 spin summations are the oracle's C restatement here (the GPU
path uses this library's kernels, checked bit for bit elsewhere)."""
import numpy as np
import pytest
import torch

from oracle import t4_ref
from dcc import t4_residual as tr


def _inputs(no, nv, seed):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    r = lambda *s, sc=0.1: rng.standard_normal(s) * sc  # noqa: E731
    return dict(eris=r(nmo, nmo, nmo, nmo), F_vv=r(nv, nv), W_vvvo=r(nv, nv, nv, no), W_vooo=r(nv, no, no, no),
                W_vvvv=r(nv, nv, nv, nv), W_oooo=r(no, no, no, no), W_ovov=r(no, nv, no, nv),
                t2=r(no, no, nv, nv, sc=0.05), t3=r(no, no, no, nv, nv, nv, sc=0.01),
                t4=r(len(t4_ref.stored_quadruples(no)), nv, nv, nv, nv, sc=0.01))


@pytest.mark.parametrize("no,nv", [(4, 3), (5, 4)])
def test_full_space_r4_matches_literal_blocks(oracle, no, nv):
    d = _inputs(no, nv, 3 + no)
    want = t4_ref.compute_r4_tri_ref(d["eris"], d["F_vv"], d["W_vvvo"], d["W_vooo"], d["W_vvvv"], d["W_oooo"],
                                     d["W_ovov"], d["t2"], d["t3"], d["t4"], no, oracle)

    def spin(pattern, n):
        def f(A):
            a = A.numpy()
            if n == 3:
                oracle.t3_spin_sum(a, nv, pattern, 1.0, 0.0)
            else:
                oracle.t4_spin_sum(a, a.size // nv ** 4, nv, pattern, 1.0, 0.0)
            return A
        return f

    t = {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in d.items()}
    r4 = torch.zeros_like(t["t4"])
    tr.compute_r4_tri_(r4, t["eris"], t["F_vv"], t["W_vvvo"], t["W_vooo"], t["W_vvvv"], t["W_oooo"], t["W_ovov"],
                       t["t2"], t["t3"], t["t4"], no, "fp64", spin3=spin("P3_201", 3), spin4=spin("P4_201", 4))
    np.testing.assert_allclose(r4.numpy(), want, rtol=1e-12, atol=1e-14 * np.abs(want).max())


def test_unpack_all_orderings_matches_oracle(oracle):
    no, nv = 4, 3
    quads = tr.stored_quadruples(no)
    assert quads == t4_ref.stored_quadruples(no)
    rng = np.random.default_rng(1)
    t4 = rng.standard_normal((len(quads),) + (nv,) * 4)
    nfull = no * (no + 1) * (no + 2) * (no + 3) // 24
    f2l = np.full(nfull, -1, dtype=np.int64)
    for n, q in enumerate(quads):
        f2l[oracle.ijkl_to_linear(*q, no)] = n
    full = tr.unpack_all_orderings(torch.from_numpy(t4), no).numpy()
    import itertools
    for o in itertools.product(range(no), repeat=4):
        want, rc = oracle.unpack_t4(t4, f2l, *o, no, nv)
        assert np.array_equal(full[o], want), o
