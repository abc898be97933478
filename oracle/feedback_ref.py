"""TEST ORACLE ONLY -- numpy restatement of the T3 -> lower-order feedback of
the reference, literal per canonical block and per ordering:
  r1r2_add_t3_tri_            distr_cc/rccsdt.py:253-321
  intermediates_t3_add_t3_tri distr_cc/rccsdt.py:323-366
with take_t3 and the P3_422 / P3_201 symmetrizers from the C restatement
(dcc_oracle.c, pinned against the reference's src/rccsdt.c).  One rank.
t1_fock [nmo, nmo], t1_eris [nmo]^4 (the t1-dressed quantities of the
reference's imds), t3 canonical blocks in i<=j<=k order."""
from __future__ import annotations

import numpy as np

from .oracle import Oracle


def ijk_list(nocc):
    return [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]


def _perms(i, j, k):
    if i < j < k:
        return [(i, j, k), (i, k, j), (j, i, k), (j, k, i), (k, i, j), (k, j, i)]
    if i == j < k:
        return [(i, j, k), (i, k, j), (k, i, j)]
    if i < j == k:
        return [(i, j, k), (j, i, k), (j, k, i)]
    return [(i, j, k)]


def _take(orc, t3, nocc, nvir, i, j, k):
    ijk_to_local = np.arange(len(t3), dtype=np.int64)
    out, rc = orc.take_t3(t3, ijk_to_local, i, j, k, nocc, nvir)
    assert rc == 0
    return out


def r1r2_add_t3_ref(t1_fock, t1_eris, r1, r2, t3, nocc, orc=None):
    orc = orc or Oracle()
    nvir = t3.shape[1]
    o, v = slice(0, nocc), slice(nocc, None)
    e = np.einsum
    r1_loc, r2_loc = np.zeros_like(r1), np.zeros_like(r2)
    for i, j, k in ijk_list(nocc):
        x = orc.t3_spin_sum(_take(orc, t3, nocc, nvir, i, j, k), nvir, "P3_422", 1.0, 0.0)
        if i < j < k:
            r1_loc[i] += 0.5 * e('bc,abc->a', t1_eris[j, k, v, v], x) + 0.5 * e('cb,acb->a', t1_eris[j, k, v, v], x)
            r1_loc[j] += 0.5 * e('bc,bac->a', t1_eris[i, k, v, v], x) + 0.5 * e('cb,cab->a', t1_eris[i, k, v, v], x)
            r1_loc[k] += 0.5 * e('bc,bca->a', t1_eris[i, j, v, v], x) + 0.5 * e('cb,cba->a', t1_eris[i, j, v, v], x)
        elif i == j and j < k:
            r1_loc[i] += 0.5 * e('bc,abc->a', t1_eris[j, k, v, v], x) + 0.5 * e('cb,acb->a', t1_eris[j, k, v, v], x)
            r1_loc[k] += 0.5 * e('bc,bca->a', t1_eris[i, j, v, v], x)
        elif i < j and j == k:
            r1_loc[i] += 0.5 * e('bc,abc->a', t1_eris[j, k, v, v], x)
            r1_loc[j] += 0.5 * e('bc,bac->a', t1_eris[i, k, v, v], x) + 0.5 * e('cb,cab->a', t1_eris[i, k, v, v], x)
    r1 = r1 + r1_loc
    for i, j, k in ijk_list(nocc):
        for pi, pj, pk in _perms(i, j, k):
            x = orc.t3_spin_sum(_take(orc, t3, nocc, nvir, pi, pj, pk), nvir, "P3_201", 1.0, 0.0)
            r2_loc[pj, pk] += 0.5 * e("a,abc->bc", t1_fock[pi, v], x)
            r2_loc[pj, pk] += e("cad,dba->bc", t1_eris[v, pi, v, v], x)
            r2_loc[pj] -= e("la,abc->lbc", t1_eris[pk, pi, o, v], x)
    return r1, r2 + r2_loc


def intermediates_t3_add_ref(t1_eris, W_vooo, W_vvvo, t3, nocc, orc=None):
    orc = orc or Oracle()
    nvir = t3.shape[1]
    o, v = slice(0, nocc), slice(nocc, None)
    e = np.einsum
    Wo, Wv = np.zeros_like(W_vooo), np.zeros_like(W_vvvo)
    for i, j, k in ijk_list(nocc):
        for pi, pj, pk in _perms(i, j, k):
            x = orc.t3_spin_sum(_take(orc, t3, nocc, nvir, pi, pj, pk), nvir, "P3_201", 1.0, 0.0)
            Wo[:, :, pj, pk] += e('mde,ead->am', t1_eris[o, pi, v, v], x)
            Wv[:, :, :, pj] -= e('de,eba->abd', t1_eris[pk, pi, v, v], x)
    return W_vooo + Wo, W_vvvo + Wv
