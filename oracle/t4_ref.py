"""TEST ORACLE ONLY -- numpy restatement of the dense T4-residual strings of
compute_r4_tri (distr_cc/rccsdtq.py:1039-1055): F_vv.t4 (4 strings) and
W_vvvv.t4 (6 strings) for every stored block (canonical i<=j<=k<=l blocks are
their own unpack).  Literal per-block einsums; small sizes only."""
from __future__ import annotations

import numpy as np


def dense_vvvv_fvv_ref(r4, t4, W_vvvv, F_vv):
    e = np.einsum
    r4 = r4.copy()
    for q in range(t4.shape[0]):
        t = t4[q]
        r = r4[q]
        r += e("ae,ebcd->abcd", F_vv, t)
        r += e("be,aecd->abcd", F_vv, t)
        r += e("ce,abed->abcd", F_vv, t)
        r += e("de,abce->abcd", F_vv, t)
        r += e("abef,efcd->abcd", W_vvvv, t)
        r += e("acef,ebfd->abcd", W_vvvv, t)
        r += e("adef,ebcf->abcd", W_vvvv, t)
        r += e("bcef,aefd->abcd", W_vvvv, t)
        r += e("bdef,aecf->abcd", W_vvvv, t)
        r += e("cdef,abef->abcd", W_vvvv, t)
    return r4
