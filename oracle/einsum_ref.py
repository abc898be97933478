"""TEST ORACLE ONLY -- numpy FP64 restatement of the T3 residual of the
reference (distr_cc/rccsdt.py), one rank, canonical blocks in enumeration
order.  It follows the reference's einsum strings and case logic literally
(per block, per batch) so the GPU formulations can be checked against it at
small sizes.  Slow by design; never shipped.

Functions and the reference code they restate:
  compute_r3_tri_ref            distr_cc/rccsdt.py:368-433
  oo_contraction_ref            distr_cc/rccsdt.py:435-614 (one batch = all blocks)
  foo_woooo_ref                 distr_cc/rccsdt.py:616-732
  r3_update_ref                 distr_cc/rccsdt.py:947-971
"""
from __future__ import annotations

import numpy as np

from .oracle import Oracle


def ijk_list(nocc):
    return [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]


class Imds:
    """The T3 intermediates the residual consumes (names of distr_cc/_rccsdtq_core.py:_IMDS)."""

    def __init__(self, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, W_oooo):
        self.F_vv, self.F_oo = F_vv, F_oo
        self.W_vvvo, self.W_vooo, self.W_vvvv = W_vvvo, W_vooo, W_vvvv
        self.W_ovov, self.W_ovvo, self.W_oooo = W_ovov, W_ovvo, W_oooo


def _rows(nocc, targets):
    """(canonical index q, output row) of the blocks to compute: every block, or `targets`."""
    n = len(ijk_list(nocc))
    qs = range(n) if targets is None else targets
    return [(q, r) for r, q in enumerate(qs)]


def _e(*args):
    """numpy einsum contracting through BLAS (the oracle's large-shape cases need it)."""
    return np.einsum(*args, optimize=True)


def vt2_ref(imds, t2, t3, nocc, targets=None):
    """W_vvvo.t2, W_vooo.t2 and F_vv.t3 per block (distr_cc/rccsdt.py:385-402); with `targets`
    (canonical block indices) only those blocks, as rows of the result in that order."""
    W_vvvo, W_vooo, F_vv = imds.W_vvvo, imds.W_vooo, imds.F_vv
    trip = ijk_list(nocc)
    rows = _rows(nocc, targets)
    r3 = np.empty((len(rows),) + t3.shape[1:])
    for q, row in rows:
        i, j, k = trip[q]
        r = np.einsum('abd,dc->abc', W_vvvo[..., j], t2[i, k])
        r += np.einsum('acd,db->abc', W_vvvo[..., k], t2[i, j])
        r += np.einsum('bad,dc->abc', W_vvvo[..., i], t2[j, k])
        r += np.einsum('bcd,da->abc', W_vvvo[..., k], t2[j, i])
        r += np.einsum('cad,db->abc', W_vvvo[..., i], t2[k, j])
        r += np.einsum('cbd,da->abc', W_vvvo[..., j], t2[k, i])
        r -= np.einsum('al,lbc->abc', W_vooo[:, :, i, j], t2[:, k])
        r -= np.einsum('al,lcb->abc', W_vooo[:, :, i, k], t2[:, j])
        r -= np.einsum('bl,lac->abc', W_vooo[:, :, j, i], t2[:, k])
        r -= np.einsum('bl,lca->abc', W_vooo[:, :, j, k], t2[:, i])
        r -= np.einsum('cl,lab->abc', W_vooo[:, :, k, i], t2[:, j])
        r -= np.einsum('cl,lba->abc', W_vooo[:, :, k, j], t2[:, i])
        r += np.einsum('ad,dbc->abc', F_vv, t3[q])
        r += np.einsum('bd,adc->abc', F_vv, t3[q])
        r += np.einsum('cd,abd->abc', F_vv, t3[q])
        r3[row] = r
    return r3


def wvvvv_ref(imds, t3, r3, targets=None):
    """W_vvvv.t3 (distr_cc/rccsdt.py:421-427); rows of r3 as in vt2_ref."""
    W = imds.W_vvvv
    qs = range(t3.shape[0]) if targets is None else targets
    for row, q in enumerate(qs):
        r3[row] += _e('abde,dec->abc', W, t3[q])
        r3[row] += _e('acde,dbe->abc', W, t3[q])
        r3[row] += _e('bcde,ade->abc', W, t3[q])
    return r3


def foo_woooo_ref(imds, t3, r3, nocc, targets=None):
    """Prefactor-matrix form of the F_oo / W_oooo terms (distr_cc/rccsdt.py:616-732),
    one batch holding every canonical block; rows of r3 as in vt2_ref."""
    F_oo, W_oooo = imds.F_oo, imds.W_oooo
    trip = ijk_list(nocc)
    n = len(trip)
    rows = _rows(nocc, targets)
    pfs = np.zeros((6, n, len(rows)))
    for idx, (o00, o10, o20) in enumerate(trip):
        for q, (i, j, k) in [(row, trip[qq]) for qq, row in rows]:
            if k == o20:
                pfs[0, idx, q] += W_oooo[o00, o10, i, j]
            if o10 != o20 and k == o10:
                pfs[1, idx, q] += W_oooo[o00, o20, i, j]
            if o00 != o10 and k == o20:
                pfs[2, idx, q] += W_oooo[o10, o00, i, j]
            if o10 != o20 and k == o10:
                pfs[3, idx, q] += W_oooo[o20, o00, i, j]
            if o00 != o10 and k == o00:
                pfs[4, idx, q] += W_oooo[o10, o20, i, j]
            if o00 != o10 and o10 != o20 and k == o00:
                pfs[5, idx, q] += W_oooo[o20, o10, i, j]
            if j == o20:
                pfs[1, idx, q] += W_oooo[o00, o10, i, k]
            if o10 != o20 and j == o10:
                pfs[0, idx, q] += W_oooo[o00, o20, i, k]
            if o00 != o10 and j == o20:
                pfs[4, idx, q] += W_oooo[o10, o00, i, k]
            if o10 != o20 and j == o10:
                pfs[5, idx, q] += W_oooo[o20, o00, i, k]
            if o00 != o10 and j == o00:
                pfs[2, idx, q] += W_oooo[o10, o20, i, k]
            if o00 != o10 and o10 != o20 and j == o00:
                pfs[3, idx, q] += W_oooo[o20, o10, i, k]
            if i == o20:
                pfs[3, idx, q] += W_oooo[o00, o10, j, k]
            if o10 != o20 and i == o10:
                pfs[2, idx, q] += W_oooo[o00, o20, j, k]
            if o00 != o10 and i == o20:
                pfs[5, idx, q] += W_oooo[o10, o00, j, k]
            if o10 != o20 and i == o10:
                pfs[4, idx, q] += W_oooo[o20, o00, j, k]
            if o00 != o10 and i == o00:
                pfs[0, idx, q] += W_oooo[o10, o20, j, k]
            if o00 != o10 and o10 != o20 and i == o00:
                pfs[1, idx, q] += W_oooo[o20, o10, j, k]
            if j == o00 and k == o10:
                pfs[3, idx, q] -= F_oo[o20, i]
            if o10 != o20 and j == o00 and k == o20:
                pfs[2, idx, q] -= F_oo[o10, i]
            if o00 != o10 and j == o10 and k == o20:
                pfs[0, idx, q] -= F_oo[o00, i]
            if i == o00 and k == o10:
                pfs[1, idx, q] -= F_oo[o20, j]
            if o10 != o20 and i == o00 and k == o20:
                pfs[0, idx, q] -= F_oo[o10, j]
            if o00 != o10 and i == o10 and k == o20:
                pfs[2, idx, q] -= F_oo[o00, j]
            if i == o00 and j == o10:
                pfs[0, idx, q] -= F_oo[o20, k]
            if o10 != o20 and i == o00 and j == o20:
                pfs[1, idx, q] -= F_oo[o10, k]
            if o00 != o10 and i == o10 and j == o20:
                pfs[4, idx, q] -= F_oo[o00, k]
    r3 += _e('pq,pabc->qabc', pfs[0], t3)
    r3 += _e('pq,pacb->qabc', pfs[1], t3)
    r3 += _e('pq,pbac->qabc', pfs[2], t3)
    r3 += _e('pq,pabc->qcab', pfs[3], t3)
    r3 += _e('pq,pabc->qbca', pfs[4], t3)
    r3 += _e('pq,pabc->qcba', pfs[5], t3)
    return r3


def oo_ovov_ref(imds, t3, r3, nocc, orc=None, targets=None):
    """Masked W_ovov / W_ovvo terms (distr_cc/rccsdt.py:532-596) with the
    transpose-add and triple-sym variants of every batch block; rows of r3 as in
    vt2_ref.  A batch block's variants are made only when some target uses them."""
    orc = orc or Oracle()
    Wov, Wvo = imds.W_ovov, imds.W_ovvo
    nvir = t3.shape[1]
    trip = ijk_list(nocc)
    rows = [(row, trip[qq]) for qq, row in _rows(nocc, targets)]
    e = _e
    for idx, (o00, o10, o20) in enumerate(trip):
        used = [(row, (i, j, k)) for row, (i, j, k) in rows
                if (j == o00 and k == o10) or (o10 != o20 and j == o00 and k == o20)
                or (o00 != o10 and j == o10 and k == o20) or (i == o00 and k == o10)
                or (o10 != o20 and i == o00 and k == o20) or (o00 != o10 and i == o10 and k == o20)
                or (i == o00 and j == o10) or (o10 != o20 and i == o00 and j == o20)
                or (o00 != o10 and i == o10 and j == o20)]
        if not used:
            continue
        T = np.ascontiguousarray(t3[idx])
        T2 = orc.t3_transpose_add(T, nvir)
        V0, V1, V2 = orc.t3_triple_sym(T, nvir)
        for q, (i, j, k) in used:
            r = r3[q]
            if j == o00 and k == o10:
                r -= e('bd,dca->abc', Wov[o20, :, i, :], T)
                r -= 0.5 * e('ad,dcb->abc', Wov[o20, :, i, :], T2)
                r -= e('cd,bda->abc', Wov[o20, :, i, :], T)
                r += 0.5 * e('ad,bcd->abc', Wvo[o20, :, :, i], V0)
            if o10 != o20 and j == o00 and k == o20:
                r -= e('bd,dac->abc', Wov[o10, :, i, :], T)
                r -= e('cd,bad->abc', Wov[o10, :, i, :], T)
                r -= 0.5 * e('ad,bcd->abc', Wov[o10, :, i, :], T2)
                r += 0.5 * e('ad,bdc->abc', Wvo[o10, :, :, i], V1)
            if o00 != o10 and j == o10 and k == o20:
                r -= e('bd,adc->abc', Wov[o00, :, i, :], T)
                r -= 0.5 * e('ad,bdc->abc', Wov[o00, :, i, :], T2)
                r -= e('cd,abd->abc', Wov[o00, :, i, :], T)
                r += 0.5 * e('ad,dbc->abc', Wvo[o00, :, :, i], V2)
            if i == o00 and k == o10:
                r -= e('ad,dcb->abc', Wov[o20, :, j, :], T)
                r -= 0.5 * e('bd,dca->abc', Wov[o20, :, j, :], T2)
                r -= e('cd,adb->abc', Wov[o20, :, j, :], T)
                r += 0.5 * e('bd,acd->abc', Wvo[o20, :, :, j], V0)
            if o10 != o20 and i == o00 and k == o20:
                r -= e('ad,dbc->abc', Wov[o10, :, j, :], T)
                r -= e('cd,abd->abc', Wov[o10, :, j, :], T)
                r -= 0.5 * e('bd,acd->abc', Wov[o10, :, j, :], T2)
                r += 0.5 * e('bd,adc->abc', Wvo[o10, :, :, j], V1)
            if o00 != o10 and i == o10 and k == o20:
                r -= e('ad,bdc->abc', Wov[o00, :, j, :], T)
                r -= 0.5 * e('bd,adc->abc', Wov[o00, :, j, :], T2)
                r -= e('cd,bad->abc', Wov[o00, :, j, :], T)
                r += 0.5 * e('bd,dac->abc', Wvo[o00, :, :, j], V2)
            if i == o00 and j == o10:
                r -= e('bd,adc->abc', Wov[o20, :, k, :], T)
                r -= e('ad,dbc->abc', Wov[o20, :, k, :], T)
                r -= 0.5 * e('cd,dba->abc', Wov[o20, :, k, :], T2)
                r += 0.5 * e('cd,abd->abc', Wvo[o20, :, :, k], V0)
            if o10 != o20 and i == o00 and j == o20:
                r -= 0.5 * e('cd,abd->abc', Wov[o10, :, k, :], T2)
                r -= e('bd,acd->abc', Wov[o10, :, k, :], T)
                r -= e('ad,dcb->abc', Wov[o10, :, k, :], T)
                r += 0.5 * e('cd,adb->abc', Wvo[o10, :, :, k], V1)
            if o00 != o10 and i == o10 and j == o20:
                r -= e('bd,cad->abc', Wov[o00, :, k, :], T)
                r -= e('ad,cdb->abc', Wov[o00, :, k, :], T)
                r -= 0.5 * e('cd,adb->abc', Wov[o00, :, k, :], T2)
                r += 0.5 * e('cd,dab->abc', Wvo[o00, :, :, k], V2)
    return r3


def compute_r3_tri_ref(imds, t2, t3, nocc, with_oo=True, targets=None):
    """The whole compute_r3_tri at one rank (distr_cc/rccsdt.py:368-433); with `targets`
    (canonical block indices) the r3 of those blocks only, in that order."""
    r3 = vt2_ref(imds, t2, t3, nocc, targets)
    if with_oo:
        foo_woooo_ref(imds, t3, r3, nocc, targets)
        oo_ovov_ref(imds, t3, r3, nocc, targets=targets)
    wvvvv_ref(imds, t3, r3, targets)
    return r3


def r3_update_ref(t3, r3, eia, nocc, nvir_active=None, orc=None):
    """P3_full symmetrize (-1/6, 1), divide by D, norms, t3 += r3 (distr_cc/rccsdt.py:947-971)."""
    orc = orc or Oracle()
    nvir = t3.shape[1]
    r3 = orc.t3_spin_sum(np.ascontiguousarray(r3), nvir, "P3_full", -1.0 / 6.0, 1.0)
    ijk = np.asarray(ijk_list(nocc), dtype=np.int32)
    orc.r3_divide(r3, eia, ijk)
    na = nvir if nvir_active is None else nvir_active
    norms = (float(np.sum(r3 ** 2)), float(np.sum(r3[:, :na, :na, :na] ** 2)))
    return t3 + r3, r3, norms
