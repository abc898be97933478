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


# ----------------------------------------------------------------------------
# compute_r4_tri without its OO batch (distr_cc/rccsdtq.py:700-1060), literal:
# the W builders (:700-833) and the per-block strings of :862-1055, on blocks
# i<=j<=k<=l stored in lexicographic order without the zero blocks
# (distr_cc/distribute_t4.py:68-70, three equal occupied indices).
# ----------------------------------------------------------------------------

def stored_quadruples(nocc):
    out = []
    for i in range(nocc):
        for j in range(i, nocc):
            for k in range(j, nocc):
                for l in range(k, nocc):
                    if not (i == j == k or j == k == l):
                        out.append((i, j, k, l))
    return out


def _pair_index(i, j, nocc):
    if i > j:
        i, j = j, i
    return i * nocc - i * (i - 1) // 2 + (j - i)


def build_w_oovvvo(eris, t2, c_t3, nocc):
    """distr_cc/rccsdtq.py:700-714 (c_t3 = P3_201 of the full t3)."""
    e = np.einsum
    o, v = slice(0, nocc), slice(nocc, None)
    W = 2.0 * e('maef,jibf->ijeabm', eris[o, v, v, v], t2)
    W -= e('mafe,jibf->ijeabm', eris[o, v, v, v], t2)
    W -= 2.0 * e('mnei,njab->ijeabm', eris[o, o, v, o], t2)
    W += e('nmei,njab->ijeabm', eris[o, o, v, o], t2)
    W += 0.5 * e('nmfe,nijfab->ijeabm', eris[o, o, v, v], c_t3)
    W -= 0.25 * e('mnfe,nijfab->ijeabm', eris[o, o, v, v], c_t3)
    return W + W.transpose(1, 0, 2, 4, 3, 5)


def build_w_ovovvo(eris, t2, t3, nocc):
    """distr_cc/rccsdtq.py:716-727."""
    e = np.einsum
    o, v = slice(0, nocc), slice(nocc, None)
    W = e('mafe,jibf->iejabm', eris[o, v, v, v], t2)
    W -= e('mnie,njab->iejabm', eris[o, o, o, v], t2)
    W -= 0.5 * e('nmef,injfab->iejabm', eris[o, o, v, v], t3)
    return W


def build_w_ooooov(eris, t2, t3, nocc):
    """distr_cc/rccsdtq.py:729-738."""
    e = np.einsum
    o, v = slice(0, nocc), slice(nocc, None)
    W = e('mnek,ijae->kjinma', eris[o, o, v, o], t2)
    W += 0.5 * e('mnef,ijkaef->kjinma', eris[o, o, v, v], t3)
    return W + W.transpose(1, 0, 2, 4, 3, 5)


def build_w_oooovv_oovvvv(eris, t2, t3, t4, quads, W_oooo, W_ovov, W_vvvv, nocc, orc):
    """distr_cc/rccsdtq.py:740-833: the T4 loop over the distinct orderings of every
    stored block (P4_201 applied to each unpacked ordering), then the replicated terms."""
    import itertools
    e = np.einsum
    o, v = slice(0, nocc), slice(nocc, None)
    nvir = t2.shape[2]
    nfull = nocc * (nocc + 1) * (nocc + 2) * (nocc + 3) // 24
    f2l = np.full(nfull, -1, dtype=np.int64)  # full triangular index -> stored block
    for n, qd in enumerate(quads):
        f2l[orc.ijkl_to_linear(*qd, nocc)] = n
    W_oooovv = np.zeros((nocc,) * 4 + (nvir,) * 2)
    W_oovvvv = np.zeros((nocc * (nocc + 1) // 2,) + (nvir,) * 4)
    for inds in quads:
        if max(inds.count(x) for x in inds) >= 3:
            continue
        for (pi, pj, pk, pl) in dict.fromkeys(itertools.permutations(inds)):
            t, _ = orc.unpack_t4(np.ascontiguousarray(t4), f2l, pi, pj, pk, pl, nocc, nvir)
            orc.t4_spin_sum(t, 1, nvir, "P4_201", 1.0, 0.0)
            W_oooovv[pj, pk, pl] += 0.5 * e('mef,fabe->mab', eris[o, pi, v, v], t)
            p = _pair_index(pk, pl, nocc)
            if pk < pl:
                W_oovvvv[p] -= 0.5 * e('ef,fabc->abce', eris[pj, pi, v, v], t)
            elif pk > pl:
                W_oovvvv[p] -= 0.5 * e('ef,fabc->acbe', eris[pj, pi, v, v], t)
            else:
                W_oovvvv[p] -= 0.5 * e('ef,fabc->abce', eris[pj, pi, v, v], t)
                W_oovvvv[p] -= 0.5 * e('ef,fabc->acbe', eris[pj, pi, v, v], t)
    W_oooovv += e('amef,ijkebf->ijkmab', eris[v, o, v, v], t3)
    tmp = eris[o, v, v, o].copy()
    c_t2 = 2.0 * t2 - t2.transpose(0, 1, 3, 2)
    tmp += e('nmfe,nifa->maei', eris[o, o, v, v], c_t2)
    tmp -= 0.5 * e('mnfe,nifa->maei', eris[o, o, v, v], c_t2)
    tmp -= 0.5 * e('nmef,infa->maei', eris[o, o, v, v], t2)
    W_oooovv += e('maei,jkbe->ijkmab', tmp, t2)
    W_oooovv += e('make,jibe->ijkmab', W_ovov, t2)
    W_oooovv -= 0.5 * e('mnki,njab->ijkmab', W_oooo, t2)
    for j in range(nocc):
        for k in range(j, nocc):
            p = _pair_index(j, k, nocc)
            W_oovvvv[p] += 0.5 * e('abef,fc->abce', W_vvvv, t2[j, k])
            W_oovvvv[p] += 0.5 * e('acef,fb->abce', W_vvvv, t2[k, j])
    W_oooovv = W_oooovv + W_oooovv.transpose(1, 0, 2, 3, 5, 4)
    return W_oooovv, W_oovvvv


def compute_r4_tri_ref(eris, F_vv, W_vvvo, W_vooo, W_vvvv, W_oooo, W_ovov, t2, t3, t4, nocc, orc, F_oo=None,
                       W_ovvo=None):
    """r4 of every stored block (distr_cc/rccsdtq.py:834-1060), with the OO batch when F_oo and
    W_ovvo are given (oo_batch_ref).
    eris: t1-dressed ERIs [nmo]^4 (physicist slices as the reference cuts them);
    t2 [i,j,a,b]; t3 full [i,j,k,a,b,c]; t4 [nstored, nvir^4]."""
    e = np.einsum
    nvir = t2.shape[2]
    quads = stored_quadruples(nocc)
    t3_tmp = np.ascontiguousarray(t3).copy()
    orc.t3_spin_sum(t3_tmp, nvir, "P3_201", 1.0, 0.0)
    W_oovvvo = build_w_oovvvo(eris, t2, t3_tmp, nocc)
    r4 = np.zeros_like(t4)
    for q, (i, j, k, l) in enumerate(quads):
        r = r4[q]
        r += e("abe,ecd->abcd", W_vvvo[..., j], t3[i, k, l])
        r += e("ace,ebd->abcd", W_vvvo[..., k], t3[i, j, l])
        r += e("ade,ebc->abcd", W_vvvo[..., l], t3[i, j, k])
        r += e("bae,ecd->abcd", W_vvvo[..., i], t3[j, k, l])
        r += e("cae,ebd->abcd", W_vvvo[..., i], t3[k, j, l])
        r += e("dae,ebc->abcd", W_vvvo[..., i], t3[l, j, k])
        r += e("bce,ead->abcd", W_vvvo[..., k], t3[j, i, l])
        r += e("bde,eac->abcd", W_vvvo[..., l], t3[j, i, k])
        r += e("cbe,ead->abcd", W_vvvo[..., j], t3[k, i, l])
        r += e("dbe,eac->abcd", W_vvvo[..., j], t3[l, i, k])
        r += e("cde,eab->abcd", W_vvvo[..., l], t3[k, i, j])
        r += e("dce,eab->abcd", W_vvvo[..., k], t3[l, i, j])
        r -= e("am,mbcd->abcd", W_vooo[:, :, i, j], t3[:, k, l])
        r -= e("am,mcbd->abcd", W_vooo[:, :, i, k], t3[:, j, l])
        r -= e("am,mdbc->abcd", W_vooo[:, :, i, l], t3[:, j, k])
        r -= e("bm,macd->abcd", W_vooo[:, :, j, i], t3[:, k, l])
        r -= e("cm,mabd->abcd", W_vooo[:, :, k, i], t3[:, j, l])
        r -= e("dm,mabc->abcd", W_vooo[:, :, l, i], t3[:, j, k])
        r -= e("bm,mcad->abcd", W_vooo[:, :, j, k], t3[:, i, l])
        r -= e("bm,mdac->abcd", W_vooo[:, :, j, l], t3[:, i, k])
        r -= e("cm,mbad->abcd", W_vooo[:, :, k, j], t3[:, i, l])
        r -= e("dm,mbac->abcd", W_vooo[:, :, l, j], t3[:, i, k])
        r -= e("cm,mdab->abcd", W_vooo[:, :, k, l], t3[:, i, j])
        r -= e("dm,mcab->abcd", W_vooo[:, :, l, k], t3[:, i, j])
        r += 0.5 * e("eabm,mecd->abcd", W_oovvvo[i, j], t3_tmp[:, k, l])
        r += 0.5 * e("eacm,mebd->abcd", W_oovvvo[i, k], t3_tmp[:, j, l])
        r += 0.5 * e("eadm,mebc->abcd", W_oovvvo[i, l], t3_tmp[:, j, k])
        r += 0.5 * e("ebcm,mead->abcd", W_oovvvo[j, k], t3_tmp[:, i, l])
        r += 0.5 * e("ebdm,meac->abcd", W_oovvvo[j, l], t3_tmp[:, i, k])
        r += 0.5 * e("ecdm,meab->abcd", W_oovvvo[k, l], t3_tmp[:, i, j])
    W_ovovvo = build_w_ovovvo(eris, t2, t3, nocc)
    for q, (i, j, k, l) in enumerate(quads):
        r = r4[q]
        for s, (x, y), (p, s2) in _OVOV_T3:
            occ = {"i": i, "j": j, "k": k, "l": l}
            r -= e(s, W_ovovvo[occ[x], :, occ[y]], t3[:, occ[p], occ[s2]])
    t3_tmp = t3 + t3.transpose(0, 1, 2, 4, 5, 3)
    W_ovovvo = W_ovovvo + W_ovovvo.transpose(2, 1, 0, 4, 3, 5)
    W_ooooov = build_w_ooooov(eris, t2, t3, nocc)
    for q, (i, j, k, l) in enumerate(quads):
        r = r4[q]
        r -= 0.5 * e("eabm,mced->abcd", W_ovovvo[i, :, j], t3_tmp[:, k, l])
        r -= 0.5 * e("eacm,mbed->abcd", W_ovovvo[i, :, k], t3_tmp[:, j, l])
        r -= 0.5 * e("eadm,mbec->abcd", W_ovovvo[i, :, l], t3_tmp[:, j, k])
        r -= 0.5 * e("ebcm,maed->abcd", W_ovovvo[j, :, k], t3_tmp[:, i, l])
        r -= 0.5 * e("ebdm,maec->abcd", W_ovovvo[j, :, l], t3_tmp[:, i, k])
        r -= 0.5 * e("ecdm,maeb->abcd", W_ovovvo[k, :, l], t3_tmp[:, i, j])
        r += e("nma,mnbcd->abcd", W_ooooov[k, j, i], t3[:, :, l])
        r += e("nma,mnbdc->abcd", W_ooooov[l, j, i], t3[:, :, k])
        r += e("nma,mncdb->abcd", W_ooooov[l, k, i], t3[:, :, j])
        r += e("nmb,mnacd->abcd", W_ooooov[k, i, j], t3[:, :, l])
        r += e("nmb,mnadc->abcd", W_ooooov[l, i, j], t3[:, :, k])
        r += e("nmb,mncda->abcd", W_ooooov[l, k, j], t3[:, :, i])
        r += e("nmc,mnabd->abcd", W_ooooov[j, i, k], t3[:, :, l])
        r += e("nmc,mnadb->abcd", W_ooooov[l, i, k], t3[:, :, j])
        r += e("nmc,mnbda->abcd", W_ooooov[l, j, k], t3[:, :, i])
        r += e("nmd,mnabc->abcd", W_ooooov[j, i, l], t3[:, :, k])
        r += e("nmd,mnacb->abcd", W_ooooov[k, i, l], t3[:, :, j])
        r += e("nmd,mnbca->abcd", W_ooooov[k, j, l], t3[:, :, i])
    W_oooovv, W_oovvvv = build_w_oooovv_oovvvv(eris, t2, t3, t4, quads, W_oooo, W_ovov, W_vvvv, nocc, orc)
    for q, (i, j, k, l) in enumerate(quads):
        r = r4[q]
        r -= e("mab,mcd->abcd", W_oooovv[i, j, k], t2[:, l])
        r -= e("mab,mdc->abcd", W_oooovv[i, j, l], t2[:, k])
        r -= e("mac,mbd->abcd", W_oooovv[i, k, j], t2[:, l])
        r -= e("mad,mbc->abcd", W_oooovv[i, l, j], t2[:, k])
        r -= e("mac,mdb->abcd", W_oooovv[i, k, l], t2[:, j])
        r -= e("mad,mcb->abcd", W_oooovv[i, l, k], t2[:, j])
        r -= e("mbc,mad->abcd", W_oooovv[j, k, i], t2[:, l])
        r -= e("mbd,mac->abcd", W_oooovv[j, l, i], t2[:, k])
        r -= e("mcd,mab->abcd", W_oooovv[k, l, i], t2[:, j])
        r -= e("mbc,mda->abcd", W_oooovv[j, k, l], t2[:, i])
        r -= e("mbd,mca->abcd", W_oooovv[j, l, k], t2[:, i])
        r -= e("mcd,mba->abcd", W_oooovv[k, l, j], t2[:, i])
        P = lambda x, y: W_oovvvv[_pair_index(x, y, nocc)]  # noqa: E731 (x <= y here)
        r += e("abce,ed->abcd", P(j, k), t2[i, l])
        r += e("abde,ec->abcd", P(j, l), t2[i, k])
        r += e("acde,eb->abcd", P(k, l), t2[i, j])
        r += e("bace,ed->abcd", P(i, k), t2[j, l])
        r += e("bade,ec->abcd", P(i, l), t2[j, k])
        r += e("cabe,ed->abcd", P(i, j), t2[k, l])
        r += e("dabe,ec->abcd", P(i, j), t2[l, k])
        r += e("cade,eb->abcd", P(i, l), t2[k, j])
        r += e("dace,eb->abcd", P(i, k), t2[l, j])
        r += e("bcde,ea->abcd", P(k, l), t2[j, i])
        r += e("cbde,ea->abcd", P(j, l), t2[k, i])
        r += e("dbce,ea->abcd", P(j, k), t2[l, i])
    r4 = dense_vvvv_fvv_ref(r4, t4, W_vvvv, F_vv)
    if F_oo is not None:
        r4 = oo_batch_ref(r4, t4, F_oo, W_oooo, W_ovvo, W_ovov, nocc, orc)
    return r4


# (string, W_ovovvo occupied slots, t3 occupied slots) of distr_cc/rccsdtq.py:913-938
_OVOV_T3 = [
    ("ecbm,maed->abcd", ("i", "j"), ("k", "l")), ("edbm,maec->abcd", ("i", "j"), ("l", "k")),
    ("ebcm,maed->abcd", ("i", "k"), ("j", "l")), ("ebdm,maec->abcd", ("i", "l"), ("j", "k")),
    ("edcm,maeb->abcd", ("i", "k"), ("l", "j")), ("ecdm,maeb->abcd", ("i", "l"), ("k", "j")),
    ("ecam,mbed->abcd", ("j", "i"), ("k", "l")), ("edam,mbec->abcd", ("j", "i"), ("l", "k")),
    ("ebam,mced->abcd", ("k", "i"), ("j", "l")), ("ebam,mdec->abcd", ("l", "i"), ("j", "k")),
    ("edam,mceb->abcd", ("k", "i"), ("l", "j")), ("ecam,mdeb->abcd", ("l", "i"), ("k", "j")),
    ("eacm,mbed->abcd", ("j", "k"), ("i", "l")), ("eadm,mbec->abcd", ("j", "l"), ("i", "k")),
    ("eabm,mced->abcd", ("k", "j"), ("i", "l")), ("eabm,mdec->abcd", ("l", "j"), ("i", "k")),
    ("eadm,mceb->abcd", ("k", "l"), ("i", "j")), ("eacm,mdeb->abcd", ("l", "k"), ("i", "j")),
    ("edcm,mbea->abcd", ("j", "k"), ("l", "i")), ("ecdm,mbea->abcd", ("j", "l"), ("k", "i")),
    ("edbm,mcea->abcd", ("k", "j"), ("l", "i")), ("ecbm,mdea->abcd", ("l", "j"), ("k", "i")),
    ("ebdm,mcea->abcd", ("k", "l"), ("j", "i")), ("ebcm,mdea->abcd", ("l", "k"), ("j", "i")),
]


# ----------------------------------------------------------------------------
# The OO batch of the T4 residual (distr_cc/rccsdtq.py:1062-1349), literal:
# the F_oo / W_oooo prefactor slots (:140-237) and, per stored source block and
# stored output block, the W_ovov / W_voov strings of the four placements of m.
# ----------------------------------------------------------------------------

def _canon_perm(v):
    order = sorted(range(4), key=lambda p: (v[p], p))
    return tuple(v[p] for p in order), tuple(order.index(p) for p in range(4))


def _foo_terms(can, target):
    """(p, m, output axes of the canonical block) of distr_cc/rccsdtq.py:198-227."""
    import itertools
    out = []
    for p in range(4):
        comp = tuple(x for x in range(4) if x != p)
        tail = tuple(target[x] for x in comp)
        to_out = (p,) + comp
        tr = tuple(to_out.index(x) for x in range(4))
        seen = set()
        for req in itertools.permutations(can):
            if req in seen:
                continue
            seen.add(req)
            if req[1:] != tail:
                continue
            c, perm = _canon_perm(req)
            if c != can:
                continue
            out.append((p, req[0], ''.join("abcd"[perm[x]] for x in tr)))
    return out


def _woooo_terms(can, target):
    """(p, q, m, n, output axes of the canonical block) of distr_cc/rccsdtq.py:166-196."""
    import itertools
    out = []
    for p, q in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
        comp = tuple(x for x in range(4) if x not in (p, q))
        head = (target[comp[0]], target[comp[1]])
        to_out = comp + (p, q)
        tr = tuple(to_out.index(x) for x in range(4))
        seen = set()
        for req in itertools.permutations(can):
            if req in seen:
                continue
            seen.add(req)
            if req[:2] != head:
                continue
            c, perm = _canon_perm(req)
            if c != can:
                continue
            out.append((p, q, req[2], req[3], ''.join("abcd"[perm[x]] for x in tr)))
    return out


def oo_batch_ref(r4, t4, F_oo, W_oooo, W_ovvo, W_ovov, nocc, orc):
    """r4 += the OO batch for every stored output block (one batch of all blocks)."""
    import itertools
    e = np.einsum
    nvir = t4.shape[1]
    quads = stored_quadruples(nocc)
    W_voov = np.ascontiguousarray(W_ovvo.transpose(1, 0, 3, 2))
    slots = {''.join(p): s for s, p in enumerate(itertools.permutations("abcd"))}
    pfs = np.zeros((24, len(quads), len(quads)))
    for s_idx, can in enumerate(quads):
        for o_idx, tgt in enumerate(quads):
            for p, m, ax in _foo_terms(can, tgt):
                pfs[slots[ax], s_idx, o_idx] -= F_oo[m, tgt[p]]
            for p, q, m, n, ax in _woooo_terms(can, tgt):
                pfs[slots[ax], s_idx, o_idx] += W_oooo[m, n, tgt[p], tgt[q]]
    for ax, s in slots.items():
        r4 += e("pq,pabcd->q" + ax, pfs[s], t4)
    W = W_ovov
    for s_idx, (o0, o1, o2, o3) in enumerate(quads):
        T = t4[s_idx]
        T3 = orc.t4_transpose_add(np.ascontiguousarray(T), nvir)
        V0, V1, V2, V3 = orc.t4_quadruple_sym(np.ascontiguousarray(T), nvir)
        for o_idx, (i, j, k, l) in enumerate(quads):
            r = r4[o_idx]
            # j k l (W at i)
            if j == o1 and k == o2 and l == o3:
                r -= e("be,aecd->abcd", W[o0, :, i, :], T) + e("ce,abed->abcd", W[o0, :, i, :], T)
                r -= e("de,abce->abcd", W[o0, :, i, :], T)
                r += 0.5 * e("ae,ebcd->abcd", W_voov[:, o0, i, :], V3)
                r -= 0.5 * e("ae,becd->abcd", W[o0, :, i, :], T3)
            if o0 != o1 and j == o0 and k == o2 and l == o3:
                r -= e("be,eacd->abcd", W[o1, :, i, :], T) + e("ce,baed->abcd", W[o1, :, i, :], T)
                r -= e("de,bace->abcd", W[o1, :, i, :], T)
                r += 0.5 * e("ae,becd->abcd", W_voov[:, o1, i, :], V2)
                r -= 0.5 * (e("ae,ebcd->abcd", W[o1, :, i, :], T) + e("ae,bced->abcd", W[o1, :, i, :], T)
                            + e("ae,bdce->abcd", W[o1, :, i, :], T))
            if o1 != o2 and j == o0 and k == o1 and l == o3:
                r -= e("be,ecad->abcd", W[o2, :, i, :], T) + e("ce,bead->abcd", W[o2, :, i, :], T)
                r -= e("de,bcae->abcd", W[o2, :, i, :], T)
                r += 0.5 * e("ae,bced->abcd", W_voov[:, o2, i, :], V1)
                r -= 0.5 * (e("ae,ecbd->abcd", W[o2, :, i, :], T) + e("ae,becd->abcd", W[o2, :, i, :], T)
                            + e("ae,bcde->abcd", W[o2, :, i, :], T))
            if o2 != o3 and j == o0 and k == o1 and l == o2:
                r -= e("be,ecda->abcd", W[o3, :, i, :], T) + e("ce,beda->abcd", W[o3, :, i, :], T)
                r -= e("de,bcea->abcd", W[o3, :, i, :], T)
                r += 0.5 * e("ae,bcde->abcd", W_voov[:, o3, i, :], V0)
                r -= 0.5 * (e("ae,ecdb->abcd", W[o3, :, i, :], T) + e("ae,bedc->abcd", W[o3, :, i, :], T)
                            + e("ae,bced->abcd", W[o3, :, i, :], T))
            # i k l (W at j)
            if i == o1 and k == o2 and l == o3:
                r -= e("ae,becd->abcd", W[o0, :, j, :], T) + e("ce,baed->abcd", W[o0, :, j, :], T)
                r -= e("de,bace->abcd", W[o0, :, j, :], T)
                r += 0.5 * e("be,eacd->abcd", W_voov[:, o0, j, :], V3)
                r -= 0.5 * e("be,aecd->abcd", W[o0, :, j, :], T3)
            if o0 != o1 and i == o0 and k == o2 and l == o3:
                r -= e("ae,ebcd->abcd", W[o1, :, j, :], T) + e("ce,abed->abcd", W[o1, :, j, :], T)
                r -= e("de,abce->abcd", W[o1, :, j, :], T)
                r += 0.5 * e("be,aecd->abcd", W_voov[:, o1, j, :], V2)
                r -= 0.5 * (e("be,eacd->abcd", W[o1, :, j, :], T) + e("be,aced->abcd", W[o1, :, j, :], T)
                            + e("be,adce->abcd", W[o1, :, j, :], T))
            if o1 != o2 and i == o0 and k == o1 and l == o3:
                r -= e("ae,ecbd->abcd", W[o2, :, j, :], T) + e("ce,aebd->abcd", W[o2, :, j, :], T)
                r -= e("de,acbe->abcd", W[o2, :, j, :], T)
                r += 0.5 * e("be,aced->abcd", W_voov[:, o2, j, :], V1)
                r -= 0.5 * (e("be,ecad->abcd", W[o2, :, j, :], T) + e("be,aecd->abcd", W[o2, :, j, :], T)
                            + e("be,acde->abcd", W[o2, :, j, :], T))
            if o2 != o3 and i == o0 and k == o1 and l == o2:
                r -= e("ae,ecdb->abcd", W[o3, :, j, :], T) + e("ce,aedb->abcd", W[o3, :, j, :], T)
                r -= e("de,aceb->abcd", W[o3, :, j, :], T)
                r += 0.5 * e("be,acde->abcd", W_voov[:, o3, j, :], V0)
                r -= 0.5 * (e("be,ecda->abcd", W[o3, :, j, :], T) + e("be,aedc->abcd", W[o3, :, j, :], T)
                            + e("be,aced->abcd", W[o3, :, j, :], T))
            # i j l (W at k)
            if i == o1 and j == o2 and l == o3:
                r -= e("ae,cebd->abcd", W[o0, :, k, :], T) + e("be,caed->abcd", W[o0, :, k, :], T)
                r -= e("de,cabe->abcd", W[o0, :, k, :], T)
                r += 0.5 * e("ce,eabd->abcd", W_voov[:, o0, k, :], V3)
                r -= 0.5 * e("ce,aebd->abcd", W[o0, :, k, :], T3)
            if o0 != o1 and i == o0 and j == o2 and l == o3:
                r -= e("ae,ecbd->abcd", W[o1, :, k, :], T) + e("be,aced->abcd", W[o1, :, k, :], T)
                r -= e("de,acbe->abcd", W[o1, :, k, :], T)
                r += 0.5 * e("ce,aebd->abcd", W_voov[:, o1, k, :], V2)
                r -= 0.5 * (e("ce,eabd->abcd", W[o1, :, k, :], T) + e("ce,abed->abcd", W[o1, :, k, :], T)
                            + e("ce,adbe->abcd", W[o1, :, k, :], T))
            if o1 != o2 and i == o0 and j == o1 and l == o3:
                r -= e("ae,ebcd->abcd", W[o2, :, k, :], T) + e("be,aecd->abcd", W[o2, :, k, :], T)
                r -= e("de,abce->abcd", W[o2, :, k, :], T)
                r += 0.5 * e("ce,abed->abcd", W_voov[:, o2, k, :], V1)
                r -= 0.5 * (e("ce,ebad->abcd", W[o2, :, k, :], T) + e("ce,aebd->abcd", W[o2, :, k, :], T)
                            + e("ce,abde->abcd", W[o2, :, k, :], T))
            if o2 != o3 and i == o0 and j == o1 and l == o2:
                r -= e("ae,ebdc->abcd", W[o3, :, k, :], T) + e("be,aedc->abcd", W[o3, :, k, :], T)
                r -= e("de,abec->abcd", W[o3, :, k, :], T)
                r += 0.5 * e("ce,abde->abcd", W_voov[:, o3, k, :], V0)
                r -= 0.5 * (e("ce,ebda->abcd", W[o3, :, k, :], T) + e("ce,aedb->abcd", W[o3, :, k, :], T)
                            + e("ce,abed->abcd", W[o3, :, k, :], T))
            # i j k (W at l)
            if i == o1 and j == o2 and k == o3:
                r -= e("ae,debc->abcd", W[o0, :, l, :], T) + e("be,daec->abcd", W[o0, :, l, :], T)
                r -= e("ce,dabe->abcd", W[o0, :, l, :], T)
                r += 0.5 * e("de,eabc->abcd", W_voov[:, o0, l, :], V3)
                r -= 0.5 * e("de,aebc->abcd", W[o0, :, l, :], T3)
            if o0 != o1 and i == o0 and j == o2 and k == o3:
                r -= e("ae,edbc->abcd", W[o1, :, l, :], T) + e("be,adec->abcd", W[o1, :, l, :], T)
                r -= e("ce,adbe->abcd", W[o1, :, l, :], T)
                r += 0.5 * e("de,aebc->abcd", W_voov[:, o1, l, :], V2)
                r -= 0.5 * (e("de,eabc->abcd", W[o1, :, l, :], T) + e("de,abec->abcd", W[o1, :, l, :], T)
                            + e("de,acbe->abcd", W[o1, :, l, :], T))
            if o1 != o2 and i == o0 and j == o1 and k == o3:
                r -= e("ae,ebdc->abcd", W[o2, :, l, :], T) + e("be,aedc->abcd", W[o2, :, l, :], T)
                r -= e("ce,abde->abcd", W[o2, :, l, :], T)
                r += 0.5 * e("de,abec->abcd", W_voov[:, o2, l, :], V1)
                r -= 0.5 * (e("de,ebac->abcd", W[o2, :, l, :], T) + e("de,aebc->abcd", W[o2, :, l, :], T)
                            + e("de,abce->abcd", W[o2, :, l, :], T))
            if o2 != o3 and i == o0 and j == o1 and k == o2:
                r -= e("ae,ebcd->abcd", W[o3, :, l, :], T) + e("be,aecd->abcd", W[o3, :, l, :], T)
                r -= e("ce,abed->abcd", W[o3, :, l, :], T)
                r += 0.5 * e("de,abce->abcd", W_voov[:, o3, l, :], V0)
                r -= 0.5 * (e("de,ebca->abcd", W[o3, :, l, :], T) + e("de,aecb->abcd", W[o3, :, l, :], T)
                            + e("de,abec->abcd", W[o3, :, l, :], T))
    return r4


# ----------------------------------------------------------------------------
# T4 -> r2 and T4 -> r3 feedback of RCCSDTQ, literal per stored block:
# r2_add_t4_tri_ (distr_cc/rccsdtq.py:471-575) and r3_add_t4_tri_ (:577-683).
# ----------------------------------------------------------------------------

# (unpacked ordering as positions of (i, j, k, l), alpha) per case of r2_add_t4_tri_
# (:489-556); the term is r2[o[2], o[3]] += alpha eris[o[0], o[1], e, f] P4_442(T[o])[e,f,a,b]
_R2_CASES = {
    "ijkl": [((0, 1, 2, 3), 1.0), ((0, 2, 1, 3), 1.0), ((0, 3, 1, 2), 1.0), ((1, 2, 0, 3), 1.0),
             ((1, 3, 0, 2), 1.0), ((2, 3, 0, 1), 1.0)],
    "iikl": [((0, 1, 2, 3), 0.5), ((0, 2, 1, 3), 1.0), ((0, 3, 1, 2), 1.0), ((2, 3, 0, 1), 0.5)],
    "ijjl": [((0, 1, 2, 3), 1.0), ((0, 3, 1, 2), 0.5), ((1, 2, 0, 3), 0.5), ((1, 3, 0, 2), 1.0)],
    "ijkk": [((0, 1, 2, 3), 0.5), ((0, 2, 1, 3), 1.0), ((1, 2, 0, 3), 1.0), ((2, 3, 0, 1), 0.5)],
    "iikk": [((0, 1, 2, 3), 0.25), ((0, 2, 1, 3), 1.0), ((2, 3, 0, 1), 0.25)],
}
# the same for the T1-Fock part of r3_add_t4_tri_ (:598-647): r3[o[1], o[2], o[3]] +=
# alpha fock[o[0], e] P4_201(T[o])[e,a,b,c]
_R3_CASES = {
    "ijkl": [((0, 1, 2, 3), 1.0), ((1, 0, 2, 3), 1.0), ((2, 0, 1, 3), 1.0), ((3, 0, 1, 2), 1.0)],
    "iikl": [((0, 1, 2, 3), 1.0), ((2, 0, 1, 3), 0.5), ((3, 0, 1, 2), 0.5)],
    "ijjl": [((0, 1, 2, 3), 0.5), ((1, 0, 2, 3), 1.0), ((3, 0, 1, 2), 0.5)],
    "ijkk": [((0, 1, 2, 3), 0.5), ((1, 0, 2, 3), 0.5), ((2, 0, 1, 3), 1.0)],
    "iikk": [((0, 1, 2, 3), 0.5), ((2, 0, 1, 3), 0.5)],
}


def _case(q):
    i, j, k, l = q
    if i < j < k < l:
        return "ijkl"
    if i == j < k < l:
        return "iikl"
    if i < j == k < l:
        return "ijjl"
    if i < j < k == l:
        return "ijkk"
    if i == j < k == l:
        return "iikk"
    return None


def _unpacked(t4, f2l, o, nocc, nvir, orc, pattern):
    t, _ = orc.unpack_t4(np.ascontiguousarray(t4), f2l, o[0], o[1], o[2], o[3], nocc, nvir)
    return orc.t4_spin_sum(t, 1, nvir, pattern, 1.0, 0.0)


def _f2l(quads, nocc, orc):
    nfull = nocc * (nocc + 1) * (nocc + 2) * (nocc + 3) // 24
    f2l = np.full(nfull, -1, dtype=np.int64)
    for n, qd in enumerate(quads):
        f2l[orc.ijkl_to_linear(*qd, nocc)] = n
    return f2l


def r2_add_t4_tri_ref(r2, t4, t1_eris, nocc, orc):
    """r2 + the T4 contributions of r2_add_t4_tri_ (t4 the stored blocks, t1_eris [nmo]^4)."""
    e = np.einsum
    nvir = t4.shape[1]
    v = slice(nocc, None)
    quads = stored_quadruples(nocc)
    f2l = _f2l(quads, nocc, orc)
    r2_loc = np.zeros_like(r2)
    for q in quads:
        for pos, alpha in _R2_CASES[_case(q)]:
            o = tuple(q[p] for p in pos)
            t = _unpacked(t4, f2l, o, nocc, nvir, orc, "P4_442")
            r2_loc[o[2], o[3]] += alpha * e('ef,efab->ab', t1_eris[o[0], o[1], v, v], t)
    return r2 + r2_loc


def r3_add_t4_tri_ref(r3, t4, t1_fock, t1_eris, nocc, orc):
    """r3 (full [no]^3 [nv]^3) + the T4 contributions of r3_add_t4_tri_."""
    import itertools
    e = np.einsum
    nvir = t4.shape[1]
    o_, v = slice(0, nocc), slice(nocc, None)
    quads = stored_quadruples(nocc)
    f2l = _f2l(quads, nocc, orc)
    r3_loc = np.zeros_like(r3)
    for q in quads:
        for pos, alpha in _R3_CASES[_case(q)]:
            o = tuple(q[p] for p in pos)
            t = _unpacked(t4, f2l, o, nocc, nvir, orc, "P4_201")
            r3_loc[o[1], o[2], o[3]] += alpha * e('e,eabc->abc', t1_fock[o[0], v], t)
    for q in quads:
        if max(q.count(x) for x in q) >= 3:
            continue
        for (pi, pj, pk, pl) in dict.fromkeys(itertools.permutations(q)):
            t = _unpacked(t4, f2l, (pi, pj, pk, pl), nocc, nvir, orc, "P4_201")
            r3_loc[pj, pk, pl] += 0.5 * e('aef,febc->abc', t1_eris[v, pi, v, v], t)
            r3_loc[pj, :, pl] += -0.5 * e('en,eabc->nabc', t1_eris[pi, pk, v, o_], t)
    return r3 + r3_loc
