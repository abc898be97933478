"""The batched residual's algebra on the CPU: the full S3 symmetrization of
S - Y (plus F_vv.t3 and W_vvvv.t3) equals the oracle's literal restatement
of compute_r3_tri (distr_cc/rccsdt.py:368-732), with and without the
W_oooo pair symmetry."""
import itertools

import numpy as np
import pytest
import torch

from oracle import einsum_ref as er
from dcc import t3_residual as tr

e = np.einsum


def s3_sum(T):
    return sum(T.transpose(p + tuple(3 + x for x in p)) for p in itertools.permutations(range(3)))


def subset_sum(T, mask):
    perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    out = np.zeros_like(T)
    for b, p in enumerate(perms):
        if mask & (1 << b):
            # out[ijk][abc] += T[p(ijk)][p(abc)], p(x)_m = x[p[m]]
            inv = tuple(np.argsort(p))
            out += T.transpose(inv + tuple(3 + x for x in inv))
    return out


@pytest.mark.parametrize("pair_symmetric", [True, False])
def test_s3_form_matches_oracle(oracle, pair_symmetric):
    no, nv = 4, 5
    rng = np.random.default_rng(11)
    full = rng.standard_normal((no,) * 3 + (nv,) * 3)
    U = s3_sum(full) / 6
    t3 = np.stack([U[i, j, k] for i, j, k in er.ijk_list(no)])
    t2 = rng.standard_normal((no, no, nv, nv))
    t2 = 0.5 * (t2 + t2.transpose(1, 0, 3, 2))
    Wvvvo, Wvooo = rng.standard_normal((nv, nv, nv, no)), rng.standard_normal((nv, no, no, no))
    Wov, Wvo = rng.standard_normal((no, nv, no, nv)), rng.standard_normal((no, nv, nv, no))
    Woo = rng.standard_normal((no,) * 4)
    if pair_symmetric:
        Woo = Woo + Woo.transpose(1, 0, 3, 2)
    Foo, Fvv = rng.standard_normal((no, no)), rng.standard_normal((nv, nv))
    Wvvvv = rng.standard_normal((nv,) * 4)
    imds = er.Imds(Fvv, Foo, Wvvvo, Wvooo, Wvvvv, Wov, Wvo, Woo)
    ref = er.compute_r3_tri_ref(imds, t2, t3, no, with_oo=True)

    A, Wa = tr.woooo_foo_matrix(torch.from_numpy(Woo), torch.from_numpy(Foo))
    assert (Wa is None) == pair_symmetric
    G2 = -0.5 * (Wov + Wvo.transpose(0, 1, 3, 2))
    S = (e('abdj,ikdc->ijkabc', Wvvvo, t2) - e('lbid,jkldca->ijkabc', Wov, U) + e('laid,jkldcb->ijkabc', G2, U)
         + 0.5 * e('ladi,jklbcd->ijkabc', Wvo, U))
    S += (A.numpy() @ U.reshape(no * no, -1)).reshape(S.shape)
    Y = e('alij,lkbc->ijkabc', Wvooo, t2)
    R = s3_sum(S - Y)
    if Wa is not None:
        Ga = e('lmij,lmkabc->ijkabc', Wa.numpy(), U)
        R += subset_sum(Ga, tr.OOOO_SET)
    r3 = np.stack([R[i, j, k] for i, j, k in er.ijk_list(no)])
    r3 += e('ad,qdbc->qabc', Fvv, t3) + e('bd,qadc->qabc', Fvv, t3) + e('cd,qabd->qabc', Fvv, t3)
    r3 += e('abde,qdec->qabc', Wvvvv, t3) + e('acde,qdbe->qabc', Wvvvv, t3) + e('bcde,qade->qabc', Wvvvv, t3)
    np.testing.assert_allclose(r3, ref, rtol=0, atol=1e-10 * np.abs(ref).max())


def test_woooo_k_pieces():
    """K pieces of the K-major U split: one piece while (K - 1) * stride fits in 31 bits, else
    pieces of whole multiples of 8 (the last one the rest) whose offsets all fit."""
    from dcc.t3_residual import woooo_k_pieces
    assert woooo_k_pieces(10, 90) == [100]
    p = woooo_k_pieces(15, 93)
    stride = 15 * 93 ** 3
    assert p == [176, 49] and sum(p) == 225 and all(k % 8 == 0 for k in p[:-1])
    assert all((k - 1) * stride < (1 << 31) - 1 for k in p)
    assert woooo_k_pieces(5, 6, limit=8 * 5 * 6 ** 3 + 1) == [8, 8, 8, 1]
    with pytest.raises(ValueError):
        woooo_k_pieces(4, 10, limit=100)
