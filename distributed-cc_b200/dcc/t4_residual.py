"""Dense part of the T4 residual on the GPU (distr_cc/rccsdtq.py:1039-1055).

For every stored T4 block (a canonical i<=j<=k<=l block is its own unpack)
the reference adds four F_vv.t4 and six W_vvvv.t4 strings.  Here each
W_vvvv string is ONE GEMM over all stored blocks (M = nblocks nvir^2, N = K =
nvir^2), run as a split-precision tcgen05 GEMM that reads t4 in place and
accumulates into r4 through its address maps (contract.einsum_into); the F_vv
strings ride in the first and last W strings as extra terms of their W
operand, as for T3:
    'ae,ebcd' + 'be,aecd' = (F[a,e] delta(b,f) + delta(a,e) F[b,f]) t4[e,f,c,d]   ('abef,efcd')
    'ce,abed' + 'de,abce' = (F[c,e] delta(d,f) + delta(c,e) F[d,f]) t4[a,b,e,f]   ('cdef,abef')
precision "fp64" runs the same strings through torch (cuBLAS DGEMM)."""
from __future__ import annotations

import torch

from . import contract

f64 = torch.float64

STRINGS = ("abef,qefcd->qabcd", "acef,qebfd->qabcd", "adef,qebcf->qabcd", "bcef,qaefd->qabcd",
           "bdef,qaecf->qabcd", "cdef,qabef->qabcd")


def w_with_f(W, F):
    """W + F[x,e] delta(y,f) + delta(x,e) F[y,f] over W's index pairs (x, y) and (e, f)."""
    Wf = W.clone()
    Wf.diagonal(0, 1, 3).add_(F.unsqueeze(2))  # F[x,e] delta(y,f)
    Wf.diagonal(0, 0, 2).add_(F.unsqueeze(2))  # delta(x,e) F[y,f]
    return Wf


def dense_vvvv_fvv_(r4, t4, W_vvvv, F_vv, precision="fp64"):
    """r4 += F_vv.t4 + W_vvvv.t4 over all stored blocks (r4, t4: [nblocks, nvir^4])."""
    kind = None if precision == "fp64" else contract.KIND[precision]
    Wf = w_with_f(W_vvvv, F_vv)
    for n, s in enumerate(STRINGS):
        W = Wf if n in (0, 5) else W_vvvv
        contract.einsum_into(s, W, t4, r4, 1.0, 1.0, kind)
    return r4


# ----------------------------------------------------------------------------
# compute_r4_tri without its OO batch (distr_cc/rccsdtq.py:700-1058).
#
# The reference adds, per stored block (i<=j<=k<=l), about a hundred strings
# "W[occupied slots of (i,j,k,l)] . T[other slots]" over the block's virtual
# indices.  Here each string is ONE contraction batched over the stored blocks:
# both operands are cut at every block's occupied slots at once (a gather by
# the blocks' index columns) and contracted over the rest with the block as the
# batch index, straight into r4.  The W builders are full-tensor einsums (the
# T4 part of W_oooovv / W_oovvvv sums over every ordering of the stored blocks,
# P4_201 applied, exactly the reference's loop over distinct permutations).
# W_oovvvv is kept for every ordered pair (x, y) with W[x, y] = W_pair(min, max):
# the strings only read x <= y.
# ----------------------------------------------------------------------------

import itertools  # noqa: E402
import struct  # noqa: E402

import numpy as np  # noqa: E402


def stored_quadruples(nocc):
    """Stored T4 blocks: i<=j<=k<=l in lexicographic order without three equal indices
    (distr_cc/distribute_t4.py:68-70)."""
    return [(i, j, k, l) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)
            for l in range(k, nocc) if not (i == j == k or j == k == l)]


_DEV_CACHE = {}


def _cached(key, device, build):
    """Index tensors built once per (key, device) and kept on the device, so that a step
    makes no host-to-device copy (a requirement of CUDA-graph capture)."""
    k = key + (str(torch.device(device)),)
    if k not in _DEV_CACHE:
        _DEV_CACHE[k] = build()
    return _DEV_CACHE[k]


def _unpack_groups(nocc, device):
    """[(axis ranks, ordered-tuple rows, stored-block rows)] grouped by the virtual-axis
    permutation that takes the stored block to the ordering."""
    def build():
        index = {q: n for n, q in enumerate(stored_quadruples(nocc))}
        groups = {}
        for o in itertools.product(range(nocc), repeat=4):
            order = sorted(range(4), key=lambda p: (o[p], p))
            can = tuple(o[p] for p in order)
            if can not in index:
                continue
            rank = tuple(order.index(p) for p in range(4))
            flat = ((o[0] * nocc + o[1]) * nocc + o[2]) * nocc + o[3]
            groups.setdefault(rank, ([], []))
            groups[rank][0].append(flat)
            groups[rank][1].append(index[can])
        return [(rank, torch.tensor(d, device=device), torch.tensor(s, device=device))
                for rank, (d, s) in groups.items()]
    return _cached(("unpack", nocc), device, build)


def _stored_rows(nocc, device):
    """Row of each stored block in the [nocc^4] ordered space."""
    return _cached(("stored", nocc), device, lambda: torch.tensor(
        [((i * nocc + j) * nocc + k) * nocc + l for i, j, k, l in stored_quadruples(nocc)], device=device))


def unpack_all_orderings(t4, nocc):
    """T[o] for every ordered quadruple o: the stored canonical block with its virtual
    axes permuted (axis p of the ordering is axis rank(p) of the canonical block, stable
    sort of the occupied values); zero where the canonical block is not stored."""
    nv = t4.shape[1]
    out = torch.zeros((nocc ** 4,) + (nv,) * 4, dtype=t4.dtype, device=t4.device)
    for rank, d, s in _unpack_groups(nocc, t4.device):
        out[d] = t4[s].permute(0, *(1 + r for r in rank))
    return out.view((nocc,) * 4 + (nv,) * 4)


def _slots(tensor, slots, sub):
    """Subscripts of a full tensor cut as the reference cuts it per block: `sub` are the
    block-level subscripts, `slots` the occupied letters the reference fixes."""
    if tensor in ("W_vvvo",):
        return sub + slots
    if tensor == "W_vooo":
        return sub + slots
    if tensor in ("W_oovvvo", "W_ooooov", "W_oooovv", "W_oovvvv", "t3", "t3p", "t3s"):
        return slots + sub
    if tensor in ("W_ovovvo", "W_ovovvo_s"):
        return slots[0] + sub[0] + slots[1] + sub[1:]
    if tensor in ("t3_m", "t3p_m", "t3s_m"):  # t3[:, x, y]
        return sub[0] + slots + sub[1:]
    if tensor == "t3_mn":  # t3[:, :, x]
        return sub[:2] + slots + sub[2:]
    if tensor == "t2_m":  # t2[:, x]
        return sub[0] + slots + sub[1:]
    if tensor == "t2":  # t2[x, y]
        return slots + sub
    raise ValueError(tensor)


# (block string, W tensor, W slots, T tensor, T slots, alpha) of distr_cc/rccsdtq.py:862-1033
_R4_STRINGS = [
    ("abe,ecd", "W_vvvo", "j", "t3", "ikl", 1.0), ("ace,ebd", "W_vvvo", "k", "t3", "ijl", 1.0),
    ("ade,ebc", "W_vvvo", "l", "t3", "ijk", 1.0), ("bae,ecd", "W_vvvo", "i", "t3", "jkl", 1.0),
    ("cae,ebd", "W_vvvo", "i", "t3", "kjl", 1.0), ("dae,ebc", "W_vvvo", "i", "t3", "ljk", 1.0),
    ("bce,ead", "W_vvvo", "k", "t3", "jil", 1.0), ("bde,eac", "W_vvvo", "l", "t3", "jik", 1.0),
    ("cbe,ead", "W_vvvo", "j", "t3", "kil", 1.0), ("dbe,eac", "W_vvvo", "j", "t3", "lik", 1.0),
    ("cde,eab", "W_vvvo", "l", "t3", "kij", 1.0), ("dce,eab", "W_vvvo", "k", "t3", "lij", 1.0),
    ("am,mbcd", "W_vooo", "ij", "t3_m", "kl", -1.0), ("am,mcbd", "W_vooo", "ik", "t3_m", "jl", -1.0),
    ("am,mdbc", "W_vooo", "il", "t3_m", "jk", -1.0), ("bm,macd", "W_vooo", "ji", "t3_m", "kl", -1.0),
    ("cm,mabd", "W_vooo", "ki", "t3_m", "jl", -1.0), ("dm,mabc", "W_vooo", "li", "t3_m", "jk", -1.0),
    ("bm,mcad", "W_vooo", "jk", "t3_m", "il", -1.0), ("bm,mdac", "W_vooo", "jl", "t3_m", "ik", -1.0),
    ("cm,mbad", "W_vooo", "kj", "t3_m", "il", -1.0), ("dm,mbac", "W_vooo", "lj", "t3_m", "ik", -1.0),
    ("cm,mdab", "W_vooo", "kl", "t3_m", "ij", -1.0), ("dm,mcab", "W_vooo", "lk", "t3_m", "ij", -1.0),
    ("eabm,mecd", "W_oovvvo", "ij", "t3p_m", "kl", 0.5), ("eacm,mebd", "W_oovvvo", "ik", "t3p_m", "jl", 0.5),
    ("eadm,mebc", "W_oovvvo", "il", "t3p_m", "jk", 0.5), ("ebcm,mead", "W_oovvvo", "jk", "t3p_m", "il", 0.5),
    ("ebdm,meac", "W_oovvvo", "jl", "t3p_m", "ik", 0.5), ("ecdm,meab", "W_oovvvo", "kl", "t3p_m", "ij", 0.5),
    ("ecbm,maed", "W_ovovvo", "ij", "t3_m", "kl", -1.0), ("edbm,maec", "W_ovovvo", "ij", "t3_m", "lk", -1.0),
    ("ebcm,maed", "W_ovovvo", "ik", "t3_m", "jl", -1.0), ("ebdm,maec", "W_ovovvo", "il", "t3_m", "jk", -1.0),
    ("edcm,maeb", "W_ovovvo", "ik", "t3_m", "lj", -1.0), ("ecdm,maeb", "W_ovovvo", "il", "t3_m", "kj", -1.0),
    ("ecam,mbed", "W_ovovvo", "ji", "t3_m", "kl", -1.0), ("edam,mbec", "W_ovovvo", "ji", "t3_m", "lk", -1.0),
    ("ebam,mced", "W_ovovvo", "ki", "t3_m", "jl", -1.0), ("ebam,mdec", "W_ovovvo", "li", "t3_m", "jk", -1.0),
    ("edam,mceb", "W_ovovvo", "ki", "t3_m", "lj", -1.0), ("ecam,mdeb", "W_ovovvo", "li", "t3_m", "kj", -1.0),
    ("eacm,mbed", "W_ovovvo", "jk", "t3_m", "il", -1.0), ("eadm,mbec", "W_ovovvo", "jl", "t3_m", "ik", -1.0),
    ("eabm,mced", "W_ovovvo", "kj", "t3_m", "il", -1.0), ("eabm,mdec", "W_ovovvo", "lj", "t3_m", "ik", -1.0),
    ("eadm,mceb", "W_ovovvo", "kl", "t3_m", "ij", -1.0), ("eacm,mdeb", "W_ovovvo", "lk", "t3_m", "ij", -1.0),
    ("edcm,mbea", "W_ovovvo", "jk", "t3_m", "li", -1.0), ("ecdm,mbea", "W_ovovvo", "jl", "t3_m", "ki", -1.0),
    ("edbm,mcea", "W_ovovvo", "kj", "t3_m", "li", -1.0), ("ecbm,mdea", "W_ovovvo", "lj", "t3_m", "ki", -1.0),
    ("ebdm,mcea", "W_ovovvo", "kl", "t3_m", "ji", -1.0), ("ebcm,mdea", "W_ovovvo", "lk", "t3_m", "ji", -1.0),
    ("eabm,mced", "W_ovovvo_s", "ij", "t3s_m", "kl", -0.5), ("eacm,mbed", "W_ovovvo_s", "ik", "t3s_m", "jl", -0.5),
    ("eadm,mbec", "W_ovovvo_s", "il", "t3s_m", "jk", -0.5), ("ebcm,maed", "W_ovovvo_s", "jk", "t3s_m", "il", -0.5),
    ("ebdm,maec", "W_ovovvo_s", "jl", "t3s_m", "ik", -0.5), ("ecdm,maeb", "W_ovovvo_s", "kl", "t3s_m", "ij", -0.5),
    ("nma,mnbcd", "W_ooooov", "kji", "t3_mn", "l", 1.0), ("nma,mnbdc", "W_ooooov", "lji", "t3_mn", "k", 1.0),
    ("nma,mncdb", "W_ooooov", "lki", "t3_mn", "j", 1.0), ("nmb,mnacd", "W_ooooov", "kij", "t3_mn", "l", 1.0),
    ("nmb,mnadc", "W_ooooov", "lij", "t3_mn", "k", 1.0), ("nmb,mncda", "W_ooooov", "lkj", "t3_mn", "i", 1.0),
    ("nmc,mnabd", "W_ooooov", "jik", "t3_mn", "l", 1.0), ("nmc,mnadb", "W_ooooov", "lik", "t3_mn", "j", 1.0),
    ("nmc,mnbda", "W_ooooov", "ljk", "t3_mn", "i", 1.0), ("nmd,mnabc", "W_ooooov", "jil", "t3_mn", "k", 1.0),
    ("nmd,mnacb", "W_ooooov", "kil", "t3_mn", "j", 1.0), ("nmd,mnbca", "W_ooooov", "kjl", "t3_mn", "i", 1.0),
    ("mab,mcd", "W_oooovv", "ijk", "t2_m", "l", -1.0), ("mab,mdc", "W_oooovv", "ijl", "t2_m", "k", -1.0),
    ("mac,mbd", "W_oooovv", "ikj", "t2_m", "l", -1.0), ("mad,mbc", "W_oooovv", "ilj", "t2_m", "k", -1.0),
    ("mac,mdb", "W_oooovv", "ikl", "t2_m", "j", -1.0), ("mad,mcb", "W_oooovv", "ilk", "t2_m", "j", -1.0),
    ("mbc,mad", "W_oooovv", "jki", "t2_m", "l", -1.0), ("mbd,mac", "W_oooovv", "jli", "t2_m", "k", -1.0),
    ("mcd,mab", "W_oooovv", "kli", "t2_m", "j", -1.0), ("mbc,mda", "W_oooovv", "jkl", "t2_m", "i", -1.0),
    ("mbd,mca", "W_oooovv", "jlk", "t2_m", "i", -1.0), ("mcd,mba", "W_oooovv", "klj", "t2_m", "i", -1.0),
    ("abce,ed", "W_oovvvv", "jk", "t2", "il", 1.0), ("abde,ec", "W_oovvvv", "jl", "t2", "ik", 1.0),
    ("acde,eb", "W_oovvvv", "kl", "t2", "ij", 1.0), ("bace,ed", "W_oovvvv", "ik", "t2", "jl", 1.0),
    ("bade,ec", "W_oovvvv", "il", "t2", "jk", 1.0), ("cabe,ed", "W_oovvvv", "ij", "t2", "kl", 1.0),
    ("dabe,ec", "W_oovvvv", "ij", "t2", "lk", 1.0), ("cade,eb", "W_oovvvv", "il", "t2", "kj", 1.0),
    ("dace,eb", "W_oovvvv", "ik", "t2", "lj", 1.0), ("bcde,ea", "W_oovvvv", "kl", "t2", "ji", 1.0),
    ("cbde,ea", "W_oovvvv", "jl", "t2", "ki", 1.0), ("dbce,ea", "W_oovvvv", "jk", "t2", "li", 1.0),
]


def _einsum(kind, subs, X, Y, out, alpha):
    if kind is None:
        ins, o = subs.split("->")
        out.add_(torch.einsum(subs, X, Y), alpha=alpha)
    else:
        contract.einsum_into(subs, X, Y, out, alpha, 1.0, kind)


def build_intermediates(eris, W_oooo, W_ovov, W_vvvv, t2, t3, t3p, t4, nocc, spin4, T4full=None):
    """The W builders of distr_cc/rccsdtq.py:700-833 as full tensors (FP64, torch).  T4full:
    unpack_all_orderings(t4) when the caller has it already."""
    e = torch.einsum
    o, v = slice(0, nocc), slice(nocc, None)
    W = {}
    X = 2.0 * e('maef,jibf->ijeabm', eris[o, v, v, v], t2) - e('mafe,jibf->ijeabm', eris[o, v, v, v], t2)
    X = X - 2.0 * e('mnei,njab->ijeabm', eris[o, o, v, o], t2) + e('nmei,njab->ijeabm', eris[o, o, v, o], t2)
    X = X + 0.5 * e('nmfe,nijfab->ijeabm', eris[o, o, v, v], t3p) - 0.25 * e('mnfe,nijfab->ijeabm', eris[o, o, v, v], t3p)
    W["W_oovvvo"] = X + X.permute(1, 0, 2, 4, 3, 5)
    X = e('mafe,jibf->iejabm', eris[o, v, v, v], t2) - e('mnie,njab->iejabm', eris[o, o, o, v], t2)
    W["W_ovovvo"] = X - 0.5 * e('nmef,injfab->iejabm', eris[o, o, v, v], t3)
    W["W_ovovvo_s"] = W["W_ovovvo"] + W["W_ovovvo"].permute(2, 1, 0, 4, 3, 5)
    X = e('mnek,ijae->kjinma', eris[o, o, v, o], t2) + 0.5 * e('mnef,ijkaef->kjinma', eris[o, o, v, v], t3)
    W["W_ooooov"] = X + X.permute(1, 0, 2, 4, 3, 5)
    # W_oooovv / W_oovvvv: the T4 sums over every ordering (P4_201 applied per ordering)
    T4s = unpack_all_orderings(t4, nocc) if T4full is None else T4full.clone()
    spin4(T4s)
    Woo = 0.5 * e('mief,ijklfabe->jklmab', eris[o, o, v, v], T4s)
    Word = -0.5 * e('jief,ijklfabc->klabce', eris[o, o, v, v], T4s)
    del T4s
    Woo = Woo + e('amef,ijkebf->ijkmab', eris[v, o, v, v], t3)
    c_t2 = 2.0 * t2 - t2.permute(0, 1, 3, 2)
    tmp = (eris[o, v, v, o] + e('nmfe,nifa->maei', eris[o, o, v, v], c_t2)
           - 0.5 * e('mnfe,nifa->maei', eris[o, o, v, v], c_t2) - 0.5 * e('nmef,infa->maei', eris[o, o, v, v], t2))
    Woo = Woo + e('maei,jkbe->ijkmab', tmp, t2) + e('make,jibe->ijkmab', W_ovov, t2)
    Woo = Woo - 0.5 * e('mnki,njab->ijkmab', W_oooo, t2)
    W["W_oooovv"] = Woo + Woo.permute(1, 0, 2, 3, 5, 4)
    # pair (x <= y): T4 part of orderings (x, y) plus (y, x) with b, c swapped, then the replicated terms
    Wp = Word + Word.permute(1, 0, 2, 4, 3, 5)
    Wp = Wp + 0.5 * e('abef,xyfc->xyabce', W_vvvv, t2) + 0.5 * e('acef,yxfb->xyabce', W_vvvv, t2)
    lo, hi = _cached(("pair", nocc), t2.device, lambda: (
        torch.tensor([min(x, y) for x in range(nocc) for y in range(nocc)], device=t2.device),
        torch.tensor([max(x, y) for x in range(nocc) for y in range(nocc)], device=t2.device)))
    W["W_oovvvv"] = Wp[lo, hi].view(Wp.shape)
    return W


def _gather_slots(X, subs, nocc, cache, name):
    """X cut at the occupied slots of every stored block: for X with einsum subscripts `subs`
    whose letters among i, j, k, l are the block's fixed occupied indices, the batch
    [n_stored, ...other dims] of X[those indices of block q] and the subscripts of the other
    dims.  Cached per (tensor, slot letters) for one compute_r4_tri call."""
    slots = [c for c in subs if c in "ijkl"]
    rest = "".join(c for c in subs if c not in "ijkl")
    key = (name, tuple(subs.index(c) for c in slots), tuple(slots))
    if key not in cache:
        dev = X.device
        cols = _cached(("quad_cols", nocc), dev, lambda: torch.tensor(stored_quadruples(nocc), device=dev).t().contiguous())
        order = [subs.index(c) for c in slots] + [n for n, c in enumerate(subs) if c not in "ijkl"]
        Xp = X.permute(*order)
        cache[key] = Xp[tuple(cols["ijkl".index(c)] for c in slots)]
    return cache[key], rest


# The operands of the fused strings kernel (dcc_t4_strings), in its operand-table order, and
# the tensor each T name of _R4_STRINGS reads.  The dense strings add Wf, W_vvvv and t4; the
# OO batch adds t4, its block forms, the unpacked T4 of every ordering and its W tensors.
_FUSED_OPS = ("W_vvvo", "W_vooo", "W_oovvvo", "W_ovovvo", "W_ovovvo_s", "W_ooooov", "W_oooovv", "W_oovvvv",
              "t3", "t3p", "t3s", "t2")
_DENSE_OPS = ("Wf", "W_vvvv")
_OO_OPS = ("F_oo", "W_oooo", "T4full", "W_ovov", "W_voov", "T3", "V0", "V1", "V2", "V3")
# the F_oo / W_oooo prefactor slots of the OO batch as strings over every ordering (subscripts, alpha)
_OO_PLAIN = (("F_oo", "mi", "mjklabcd", -1.0), ("F_oo", "mj", "imklabcd", -1.0), ("F_oo", "mk", "ijmlabcd", -1.0),
             ("F_oo", "ml", "ijkmabcd", -1.0), ("W_oooo", "mnij", "mnklabcd", 1.0),
             ("W_oooo", "mnik", "mjnlabcd", 1.0), ("W_oooo", "mnil", "mjknabcd", 1.0),
             ("W_oooo", "mnjk", "imnlabcd", 1.0), ("W_oooo", "mnjl", "imknabcd", 1.0),
             ("W_oooo", "mnkl", "ijmnabcd", 1.0))
_T_OPERAND = {"t3": "t3", "t3_m": "t3", "t3_mn": "t3", "t3p_m": "t3p", "t3s_m": "t3s", "t2_m": "t2", "t2": "t2"}


def _operand_shapes(nocc, nv, nq):
    o, v = nocc, nv
    return {"W_vvvo": (v, v, v, o), "W_vooo": (v, o, o, o), "W_oovvvo": (o, o, v, v, v, o),
            "W_ovovvo": (o, v, o, v, v, o), "W_ovovvo_s": (o, v, o, v, v, o), "W_ooooov": (o, o, o, o, o, v),
            "W_oooovv": (o, o, o, o, v, v), "W_oovvvv": (o, o, v, v, v, v), "t3": (o, o, o, v, v, v),
            "t3p": (o, o, o, v, v, v), "t3s": (o, o, o, v, v, v), "t2": (o, o, v, v), "Wf": (v, v, v, v),
            "W_vvvv": (v, v, v, v), "t4": (nq, v, v, v, v), "F_oo": (o, o), "W_oooo": (o, o, o, o),
            "T4full": (o, o, o, o, v, v, v, v), "W_ovov": (o, v, o, v), "W_voov": (v, o, o, v),
            "T3": (nq, v, v, v, v), "V0": (nq, v, v, v, v), "V1": (nq, v, v, v, v), "V2": (nq, v, v, v, v),
            "V3": (nq, v, v, v, v)}


def string_descriptor(wsubs, wshape, wop, tsubs, tshape, top, alpha, mode=0):
    """The 32-int64 descriptor of dcc_t4_strings for r4[q][abcd] += alpha W[wsubs] T[tsubs]:
    i, j, k, l are the block's occupied indices, q the block index, a..d the output, every
    other letter (at most two) is summed.  mode g+1: a pair-mode string of group g, where W's
    letter M is the pair's occupied index and T's letter Q its source block.  Operands are
    C-contiguous of the given shapes."""
    def strides(shape):
        st = [1] * len(shape)
        for p in range(len(shape) - 2, -1, -1):
            st[p] = st[p + 1] * shape[p + 1]
        return st

    if len(wsubs) != len(wshape) or len(tsubs) != len(tshape):
        raise ValueError("subscripts do not match the operand ranks")
    ws, ts = strides(wshape), strides(tshape)
    d = [0] * 32
    d[0], d[1] = wop, top
    for n, c in enumerate("ijkl"):
        d[2 + n] = ws[wsubs.index(c)] if c in wsubs else 0
        d[6 + n] = ts[tsubs.index(c)] if c in tsubs else 0
    d[10] = ws[wsubs.index("q")] if "q" in wsubs else 0
    d[11] = ts[tsubs.index("q")] if "q" in tsubs else 0
    if mode:
        if "Q" not in tsubs or "M" not in wsubs or "q" in tsubs:
            raise ValueError("a pair-mode string reads W at M and T at Q")
        d[11] = ts[tsubs.index("Q")]
        d[30] = ws[wsubs.index("M")]
        d[31] = mode
    mask = 0
    for n, c in enumerate("abcd"):
        if (c in wsubs) == (c in tsubs):
            raise ValueError("output letter %s must be in exactly one operand" % c)
        if c in wsubs:
            d[12 + n] = ws[wsubs.index(c)]
            mask |= 1 << n
        else:
            d[16 + n] = ts[tsubs.index(c)]
    d[20] = mask
    # iteration orders: W's output letters (rows) and T's (columns), slowest first, the
    # letter with the smallest stride last; nibble p holds letter + 1 of position p
    rows = sorted((n for n in range(4) if mask >> n & 1), key=lambda n: -d[12 + n])
    cols = sorted((n for n in range(4) if not mask >> n & 1), key=lambda n: -d[16 + n])
    d[28] = sum((n + 1) << (4 * p) for p, n in enumerate(rows))
    d[29] = sum((n + 1) << (4 * p) for p, n in enumerate(cols))
    summed = [c for c in wsubs if c not in "ijklqabcdMQ"]
    if sorted(summed) != sorted(c for c in tsubs if c not in "ijklqabcdMQ") or len(summed) > 2:
        raise ValueError("at most two summed letters, each in both operands")
    ks = []
    for c in summed:
        if wshape[wsubs.index(c)] != tshape[tsubs.index(c)]:
            raise ValueError("extents of %s differ" % c)
        ks.append((wshape[wsubs.index(c)], ws[wsubs.index(c)], ts[tsubs.index(c)]))
    ks += [(1, 0, 0)] * (2 - len(ks))
    d[21:24], d[24:27] = ks[0], ks[1]
    d[27] = struct.unpack("<q", struct.pack("<d", float(alpha)))[0]
    return d


def fused_plan(nocc, nv, dense, device, oo=False):
    """(descriptor table [nstr, 32] int64, quads [nq, 4] int32, operand names, pair lists) of
    the fused strings kernel: the strings of _R4_STRINGS; with `dense` the F_vv / W_vvvv
    strings of dense_vvvv_fvv_ (W_vvvv with F_vv folded into its first and last string); with
    `oo` the OO batch: the F_oo / W_oooo strings over the unpacked T4 of every ordering and
    every W_ovov / W_voov string of _OO_TABLE in pair mode over oo_pairs (pair lists
    (pair_off [nq, 17], pair_sm [npairs, 2]), None without `oo`)."""
    def build():
        quads = stored_quadruples(nocc)
        nq = len(quads)
        shp = _operand_shapes(nocc, nv, nq)
        names = list(_FUSED_OPS) + (["t4"] if dense or oo else []) + (list(_DENSE_OPS) if dense else []) + \
            (list(_OO_OPS) if oo else [])
        rows = []
        for sub, wn, ws, tn, ts, al in _R4_STRINGS:
            sw, st = sub.split(",")
            tname = _T_OPERAND[tn]
            rows.append(string_descriptor(_slots(wn, ws, sw), shp[wn], names.index(wn),
                                          _slots(tn, ts, st), shp[tname], names.index(tname), al))
        if dense:
            for n, s in enumerate(STRINGS):
                wsubs, rest = s.split(",")
                wn = "Wf" if n in (0, 5) else "W_vvvv"
                rows.append(string_descriptor(wsubs, shp[wn], names.index(wn), rest.split("->")[0], shp["t4"],
                                              names.index("t4"), 1.0))
        pairs = None
        if oo:
            for wn, ws, ts, al in _OO_PLAIN:
                rows.append(string_descriptor(ws, shp[wn], names.index(wn), ts, shp["T4full"],
                                              names.index("T4full"), al))
            groups = sorted(oo_pairs(nocc))
            for gid, (g, c) in enumerate(groups):
                x = "ijkl"[g]
                for wn, sub, al, form in _OO_TABLE[g][c]:
                    ws, ts = sub.split(",")
                    if wn == "ovov":  # W_ovov[m, a, x, e]
                        wsubs, wname = "M" + ws[0] + x + ws[1], "W_ovov"
                    else:  # W_voov[a, m, x, e] = W_ovvo[m, a, e, x]
                        wsubs, wname = ws[0] + "M" + x + ws[1], "W_voov"
                    tname = "t4" if form == "T" else form
                    rows.append(string_descriptor(wsubs, shp[wname], names.index(wname), "Q" + ts, shp[tname],
                                                  names.index(tname), al, mode=gid + 1))
            lists = oo_pairs(nocc)
            per = [[[] for _ in groups] for _ in range(nq)]
            for gid, gc in enumerate(groups):
                si, ti, m, _x = lists[gc]
                for a, b, mm in zip(si, ti, m):
                    per[b][gid].append((a, mm))
            off, sm = [], []
            for q in range(nq):
                row = [len(sm)]
                for gid in range(len(groups)):
                    sm.extend(per[q][gid])
                    row.append(len(sm))
                off.append(row)
            pairs = (torch.tensor(off, dtype=torch.int32, device=device),
                     torch.tensor(sm, dtype=torch.int32, device=device).view(-1, 2))
        return (torch.tensor(rows, dtype=torch.int64, device=device),
                torch.tensor(quads, dtype=torch.int32, device=device), names, pairs)
    return _cached(("fused", nocc, nv, bool(dense), bool(oo)), device, build)


def fused_status(device):
    """The int32 status word of the fused strings kernel on `device` (0: every string ran)."""
    return _cached(("fused_status",), device, lambda: torch.zeros(1, dtype=torch.int32, device=device))


def compute_r4_tri_(r4, eris, F_vv, W_vvvo, W_vooo, W_vvvv, W_oooo, W_ovov, t2, t3, t4, nocc, precision="fp64",
                    spin3=None, spin4=None, F_oo=None, W_ovvo=None, forms=None):
    """r4[stored blocks] = compute_r4_tri (distr_cc/rccsdtq.py:834-1060); with F_oo and W_ovvo
    given it includes the OO batch (oo_batch_, :1062-1349), else it stops before it.

    eris: t1-dressed ERIs [nmo]^4 (the reference's imds.t1_eris); t2 [i,j,a,b]; t3 full
    [i,j,k,a,b,c]; t4 and r4 [nstored, nvir^4] in stored_quadruples order.  spin3 / spin4
    apply P3_201 / P4_201 in place to [n, nvir^3] / [n, nvir^4] blocks (default: this
    library's kernels).

    On a CUDA device the ~100 per-block strings of distr_cc/rccsdtq.py:862-1033 run in ONE
    launch of the fused strings kernel (dcc_t4_strings: a CTA per stored block and row range
    holds its r4 rows in shared memory and runs every string over them, operands read in
    place through the descriptors of fused_plan), and with F_oo given the OO batch joins
    the same launch (its F_oo / W_oooo slots as strings over the unpacked T4, its W_ovov /
    W_voov strings in pair mode over the sparse (source, output) pair lists).  Their
    contractions are short (K = nvir, nocc, nocc^2 or nocc nvir), so they are FP64 in every
    precision; in FP64 the F_vv / W_vvvv strings join the same launch, and precision
    "bf16x3"/"tf32x3" runs those (K = nvir^2) as split GEMMs.  The builders stay FP64.  On the CPU (the formulation
    tests) each string is one einsum batched over the stored blocks, its operands cut at
    every block's occupied slots (_gather_slots)."""
    from . import _c_rccsdt, _c_rccsdt_q, _c_rccsdtq
    kind = None if precision == "fp64" else contract.KIND[precision]
    nv = t2.shape[2]
    if spin3 is None:
        spin3 = lambda A: _c_rccsdt.t3_spin_summation_inplace_(A, A.numel() // nv ** 3, nv, "P3_201", 1.0, 0.0)  # noqa: E731
    if spin4 is None:
        spin4 = lambda A: _c_rccsdt_q.t4_spin_summation_inplace_(A, A.numel() // nv ** 4, nv, "P4_201", 1.0, 0.0)  # noqa: E731
    t3 = t3.contiguous()
    t3p = t3.clone()
    spin3(t3p)
    nq = r4.shape[0]
    if t3.is_cuda and _c_rccsdtq.t4_strings_rows_per_cta(nq, nv) >= 1:
        # every string of every stored block in one launch (FP64), the OO batch included when
        # F_oo is given; the W_vvvv strings join it in FP64 and run as split GEMMs otherwise
        dense, oo = kind is None, F_oo is not None
        T4full = unpack_all_orderings(t4, nocc)
        W = build_intermediates(eris, W_oooo, W_ovov, W_vvvv, t2, t3, t3p, t4, nocc, spin4, T4full=T4full)
        W["W_vvvo"], W["W_vooo"] = W_vvvo, W_vooo
        desc, quads, names, pairs = fused_plan(nocc, nv, dense, t3.device, oo=oo)
        ops = dict(W, t3=t3, t3p=t3p, t3s=t3 + t3.permute(0, 1, 2, 4, 5, 3), t2=t2, t4=t4)
        if dense:
            ops.update(Wf=w_with_f(W_vvvv, F_vv), W_vvvv=W_vvvv)
        if oo:
            if forms is None:
                forms = lambda t: _c_rccsdtq.t4_forms_batched(t, nv)  # noqa: E731
            T3f, V = forms(t4)
            ops.update(F_oo=F_oo, W_oooo=W_oooo, T4full=T4full, W_ovov=W_ovov,
                       W_voov=W_ovvo.permute(1, 0, 3, 2), T3=T3f, V0=V[0], V1=V[1], V2=V[2], V3=V[3])
        _c_rccsdtq.t4_strings([ops[n].contiguous() for n in names], desc, quads, nocc, nv, r4.view(nq, -1),
                              0.0, fused_status(t3.device), pairs=pairs)
        if not dense:
            dense_vvvv_fvv_(r4, t4, W_vvvv, F_vv, precision)
        return r4
    W = build_intermediates(eris, W_oooo, W_ovov, W_vvvv, t2, t3, t3p, t4, nocc, spin4)
    W["W_vvvo"], W["W_vooo"] = W_vvvo, W_vooo
    T = {"t3": t3, "t3_m": t3, "t3_mn": t3, "t3p_m": t3p, "t3s_m": t3 + t3.permute(0, 1, 2, 4, 5, 3),
         "t2_m": t2, "t2": t2}
    r4.zero_()
    gathered = {}
    for sub, wn, ws, tn, ts, al in _R4_STRINGS:
        sw, st = sub.split(",")
        gw, lw = _gather_slots(W[wn], _slots(wn, ws, sw), nocc, gathered, wn)
        gt, lt = _gather_slots(T[tn], _slots(tn, ts, st), nocc, gathered, tn)
        r4.view((-1,) + (nv,) * 4).add_(torch.einsum("q" + lw + ",q" + lt + "->qabcd", gw, gt), alpha=al)
    del gathered
    dense_vvvv_fvv_(r4, t4, W_vvvv, F_vv, precision)
    if F_oo is not None:
        oo_batch_(r4, t4, F_oo, W_oooo, W_ovvo, W_ovov, nocc, forms)
    return r4


# ----------------------------------------------------------------------------
# The OO batch (distr_cc/rccsdtq.py:1062-1349).
#
# F_oo and W_oooo: the reference's 24 prefactor slots sum, for each output
# block, every ordering of the stored blocks that places m (and n) at output
# positions; over the full ordered space these are the plain strings
#   R[ijkl] -= F_oo[m,i] T[mjkl] + ... (4),   R[ijkl] += W_oooo[m,n,i,j] T[mnkl] + ... (6).
# W_ovov / W_voov: for each output block, group g (the position whose index
# enters W) and case c (where m sits in the stored source block), a fixed set
# of strings on the source block, its transpose-add or one of its four
# quadruple-symmetrized forms.  The (source, output, m) pairs of each (g, c)
# are listed once per nocc and every string runs as one batched einsum over
# its pairs, scattered into r4.
# ----------------------------------------------------------------------------

# (W tensor, string, alpha, source form) for group g (W at output position g) and case c;
# forms: "T" the block, "T3" its transpose-add, "V0".."V3" its quadruple-symmetrized forms
_OO_TABLE = {
    0: [[("ovov", "be,aecd", -1.0, "T"), ("ovov", "ce,abed", -1.0, "T"), ("ovov", "de,abce", -1.0, "T"),
         ("voov", "ae,ebcd", 0.5, "V3"), ("ovov", "ae,becd", -0.5, "T3")],
        [("ovov", "be,eacd", -1.0, "T"), ("ovov", "ce,baed", -1.0, "T"), ("ovov", "de,bace", -1.0, "T"),
         ("voov", "ae,becd", 0.5, "V2"), ("ovov", "ae,ebcd", -0.5, "T"), ("ovov", "ae,bced", -0.5, "T"),
         ("ovov", "ae,bdce", -0.5, "T")],
        [("ovov", "be,ecad", -1.0, "T"), ("ovov", "ce,bead", -1.0, "T"), ("ovov", "de,bcae", -1.0, "T"),
         ("voov", "ae,bced", 0.5, "V1"), ("ovov", "ae,ecbd", -0.5, "T"), ("ovov", "ae,becd", -0.5, "T"),
         ("ovov", "ae,bcde", -0.5, "T")],
        [("ovov", "be,ecda", -1.0, "T"), ("ovov", "ce,beda", -1.0, "T"), ("ovov", "de,bcea", -1.0, "T"),
         ("voov", "ae,bcde", 0.5, "V0"), ("ovov", "ae,ecdb", -0.5, "T"), ("ovov", "ae,bedc", -0.5, "T"),
         ("ovov", "ae,bced", -0.5, "T")]],
    1: [[("ovov", "ae,becd", -1.0, "T"), ("ovov", "ce,baed", -1.0, "T"), ("ovov", "de,bace", -1.0, "T"),
         ("voov", "be,eacd", 0.5, "V3"), ("ovov", "be,aecd", -0.5, "T3")],
        [("ovov", "ae,ebcd", -1.0, "T"), ("ovov", "ce,abed", -1.0, "T"), ("ovov", "de,abce", -1.0, "T"),
         ("voov", "be,aecd", 0.5, "V2"), ("ovov", "be,eacd", -0.5, "T"), ("ovov", "be,aced", -0.5, "T"),
         ("ovov", "be,adce", -0.5, "T")],
        [("ovov", "ae,ecbd", -1.0, "T"), ("ovov", "ce,aebd", -1.0, "T"), ("ovov", "de,acbe", -1.0, "T"),
         ("voov", "be,aced", 0.5, "V1"), ("ovov", "be,ecad", -0.5, "T"), ("ovov", "be,aecd", -0.5, "T"),
         ("ovov", "be,acde", -0.5, "T")],
        [("ovov", "ae,ecdb", -1.0, "T"), ("ovov", "ce,aedb", -1.0, "T"), ("ovov", "de,aceb", -1.0, "T"),
         ("voov", "be,acde", 0.5, "V0"), ("ovov", "be,ecda", -0.5, "T"), ("ovov", "be,aedc", -0.5, "T"),
         ("ovov", "be,aced", -0.5, "T")]],
    2: [[("ovov", "ae,cebd", -1.0, "T"), ("ovov", "be,caed", -1.0, "T"), ("ovov", "de,cabe", -1.0, "T"),
         ("voov", "ce,eabd", 0.5, "V3"), ("ovov", "ce,aebd", -0.5, "T3")],
        [("ovov", "ae,ecbd", -1.0, "T"), ("ovov", "be,aced", -1.0, "T"), ("ovov", "de,acbe", -1.0, "T"),
         ("voov", "ce,aebd", 0.5, "V2"), ("ovov", "ce,eabd", -0.5, "T"), ("ovov", "ce,abed", -0.5, "T"),
         ("ovov", "ce,adbe", -0.5, "T")],
        [("ovov", "ae,ebcd", -1.0, "T"), ("ovov", "be,aecd", -1.0, "T"), ("ovov", "de,abce", -1.0, "T"),
         ("voov", "ce,abed", 0.5, "V1"), ("ovov", "ce,ebad", -0.5, "T"), ("ovov", "ce,aebd", -0.5, "T"),
         ("ovov", "ce,abde", -0.5, "T")],
        [("ovov", "ae,ebdc", -1.0, "T"), ("ovov", "be,aedc", -1.0, "T"), ("ovov", "de,abec", -1.0, "T"),
         ("voov", "ce,abde", 0.5, "V0"), ("ovov", "ce,ebda", -0.5, "T"), ("ovov", "ce,aedb", -0.5, "T"),
         ("ovov", "ce,abed", -0.5, "T")]],
    3: [[("ovov", "ae,debc", -1.0, "T"), ("ovov", "be,daec", -1.0, "T"), ("ovov", "ce,dabe", -1.0, "T"),
         ("voov", "de,eabc", 0.5, "V3"), ("ovov", "de,aebc", -0.5, "T3")],
        [("ovov", "ae,edbc", -1.0, "T"), ("ovov", "be,adec", -1.0, "T"), ("ovov", "ce,adbe", -1.0, "T"),
         ("voov", "de,aebc", 0.5, "V2"), ("ovov", "de,eabc", -0.5, "T"), ("ovov", "de,abec", -0.5, "T"),
         ("ovov", "de,acbe", -0.5, "T")],
        [("ovov", "ae,ebdc", -1.0, "T"), ("ovov", "be,aedc", -1.0, "T"), ("ovov", "ce,abde", -1.0, "T"),
         ("voov", "de,abec", 0.5, "V1"), ("ovov", "de,ebac", -0.5, "T"), ("ovov", "de,aebc", -0.5, "T"),
         ("ovov", "de,abce", -0.5, "T")],
        [("ovov", "ae,ebcd", -1.0, "T"), ("ovov", "be,aecd", -1.0, "T"), ("ovov", "ce,abed", -1.0, "T"),
         ("voov", "de,abce", 0.5, "V0"), ("ovov", "de,ebca", -0.5, "T"), ("ovov", "de,aecb", -0.5, "T"),
         ("ovov", "de,abec", -0.5, "T")]],
}

_OO_PAIRS = {}


def oo_pairs(nocc):
    """{(g, c): (source blocks, output blocks, m, W index)} of the OO batch: output block t
    with t[g] = x and the other three positions equal to the source block s without its
    position c (m = s[c]; for c > 0 the source's s[c-1] != s[c])."""
    if nocc in _OO_PAIRS:
        return _OO_PAIRS[nocc]
    quads = stored_quadruples(nocc)
    index = {q: n for n, q in enumerate(quads)}
    out = {}
    for si, s in enumerate(quads):
        for c in range(4):
            if c > 0 and s[c - 1] == s[c]:
                continue
            rest = s[:c] + s[c + 1:]
            for g in range(4):
                for x in range(nocc):
                    t = rest[:g] + (x,) + rest[g:]
                    ti = index.get(t)
                    if ti is None:
                        continue
                    lst = out.setdefault((g, c), ([], [], [], []))
                    lst[0].append(si)
                    lst[1].append(ti)
                    lst[2].append(s[c])
                    lst[3].append(x)
    _OO_PAIRS[nocc] = out
    return out


def oo_batch_(r4, t4, F_oo, W_oooo, W_ovvo, W_ovov, nocc, forms=None):
    """r4 += the OO batch of compute_r4_tri (distr_cc/rccsdtq.py:1062-1349), FP64.

    forms(t4) -> (T3, [V0, V1, V2, V3]) per stored block (default: this library's batched
    t4_transpose_add and quadruple-sym kernels, all blocks in one launch each)."""
    e = torch.einsum
    nv = t4.shape[1]
    dev = t4.device
    if forms is None:
        from . import _c_rccsdtq

        def forms(t):  # every stored block's transpose-add and quadruple-sym forms, two launches
            return _c_rccsdtq.t4_forms_batched(t, nv)
    # F_oo and W_oooo over the full ordered space
    T = unpack_all_orderings(t4, nocc)
    R = torch.zeros_like(T)
    R -= (e('mi,mjklabcd->ijklabcd', F_oo, T) + e('mj,imklabcd->ijklabcd', F_oo, T)
          + e('mk,ijmlabcd->ijklabcd', F_oo, T) + e('ml,ijkmabcd->ijklabcd', F_oo, T))
    R += (e('mnij,mnklabcd->ijklabcd', W_oooo, T) + e('mnik,mjnlabcd->ijklabcd', W_oooo, T)
          + e('mnil,mjknabcd->ijklabcd', W_oooo, T) + e('mnjk,imnlabcd->ijklabcd', W_oooo, T)
          + e('mnjl,imknabcd->ijklabcd', W_oooo, T) + e('mnkl,ijmnabcd->ijklabcd', W_oooo, T))
    del T
    r4 += R.view(nocc ** 4, -1)[_stored_rows(nocc, dev)].view(r4.shape)
    del R
    # W_ovov / W_voov strings, batched over the (source, output) pairs of each group and case
    T3, V = forms(t4)
    src = {"T": t4, "T3": T3, "V0": V[0], "V1": V[1], "V2": V[2], "V3": V[3]}
    W_voov = W_ovvo.permute(1, 0, 3, 2).contiguous()
    pairs = _cached(("oo_pairs", nocc), dev, lambda: [
        (gc, tuple(torch.tensor(v, device=dev) for v in lists)) for gc, lists in oo_pairs(nocc).items()])
    for (g, c), (si, ti, m, x) in pairs:
        Wo = W_ovov[m, :, x, :]   # [P, a, e] = W_ovov[m, :, x, :]
        Wv = W_voov[:, m, x, :].permute(1, 0, 2)  # [P, a, e] = W_voov[:, m, x, :]
        cut, acc = {}, None  # each source form gathered once per (g, c); one scatter per (g, c)
        for wn, s, al, form in _OO_TABLE[g][c]:
            ws, ts = s.split(",")
            if form not in cut:
                cut[form] = src[form][si]
            upd = e("p" + ws + ",p" + ts + "->pabcd", Wo if wn == "ovov" else Wv, cut[form])
            acc = upd.mul_(al) if acc is None else acc.add_(upd, alpha=al)
        r4.view(r4.shape[0], -1).index_add_(0, ti, acc.reshape(acc.shape[0], -1))
    return r4


# ----------------------------------------------------------------------------
# T4 -> r2 and T4 -> r3 feedback (r2_add_t4_tri_, distr_cc/rccsdtq.py:471-575;
# r3_add_t4_tri_, :577-683) over the full ordered occupied space.
#
# The reference walks the stored blocks and, per block, the distinct ways to pull
# a pair (r2) or one index (r3, T1-Fock part) out of its occupied multiset, with
# weights 1/2 (1/4) where pulled or remaining indices coincide.  Over every ordered
# tuple of T4s = P4(T[ordering]) this is one string each:
#   r2[z,w] += W2[x,y] W2[z,w] sum_{x,y,e,f} eris[x,y,e,f] T4s_442[x,y,z,w][e,f,a,b]
#   r3[x,y,z] += W3[x,y,z] sum_{m,e} fock[m,e] T4s_201[m,x,y,z][e,a,b,c]
# with W2 = 1 (x < y), 1/2 (x = y), 0 (x > y) and W3 = 1 (x < y < z), 1/2 (sorted, two
# equal), 0 otherwise; the T1-ERI part of r3 (:649-667) already runs over every
# distinct ordering and becomes two plain strings.
# ----------------------------------------------------------------------------

def _w2(nocc, device):
    return _cached(("w2", nocc), device, lambda: torch.tensor(
        [[1.0 if x < y else (0.5 if x == y else 0.0) for y in range(nocc)] for x in range(nocc)],
        dtype=torch.float64, device=device))


def _w3(nocc, device):
    def w(x, y, z):
        if not x <= y <= z or x == z:
            return 0.0
        return 1.0 if x < y < z else 0.5
    return _cached(("w3", nocc), device, lambda: torch.tensor(
        [[[w(x, y, z) for z in range(nocc)] for y in range(nocc)] for x in range(nocc)],
        dtype=torch.float64, device=device))


def _spin4_default(nv):
    from . import _c_rccsdt_q
    return lambda A, pattern: _c_rccsdt_q.t4_spin_summation_inplace_(A, A.numel() // nv ** 4, nv, pattern, 1.0, 0.0)


def r2_add_t4_(r2, t4, eris, nocc, precision="fp64", spin4=None):
    """r2 += the T4 part of r2_add_t4_tri_ (distr_cc/rccsdtq.py:471-575).  r2 [i,j,a,b];
    t4 the stored blocks [n4, nv^4]; eris the t1-dressed ERIs [nmo]^4.  spin4(A, pattern)
    applies a P4 pattern in place to [n, nv^4] blocks (default: this library's kernel)."""
    kind = None if precision == "fp64" else contract.KIND[precision]
    nv = t4.shape[1]
    spin4 = _spin4_default(nv) if spin4 is None else spin4
    T = unpack_all_orderings(t4, nocc).contiguous()
    spin4(T.view(-1, nv, nv, nv, nv), "P4_442")
    w2 = _w2(nocc, t4.device)
    o, v = slice(0, nocc), slice(nocc, None)
    Ew = (eris[o, o, v, v] * w2[:, :, None, None]).contiguous()
    R = torch.zeros((nocc, nocc, nv, nv), dtype=t4.dtype, device=t4.device)
    _einsum(kind, "xyef,xyzwefab->zwab", Ew, T, R, 1.0)
    r2 += R * w2[:, :, None, None]
    return r2


def r3_add_t4_(r3, t4, fock, eris, nocc, precision="fp64", spin4=None):
    """r3 += the T4 part of r3_add_t4_tri_ (distr_cc/rccsdtq.py:577-683).  r3 the full
    [i,j,k,a,b,c]; fock the t1-dressed Fock matrix [nmo, nmo]; other arguments as
    r2_add_t4_."""
    kind = None if precision == "fp64" else contract.KIND[precision]
    nv = t4.shape[1]
    spin4 = _spin4_default(nv) if spin4 is None else spin4
    T = unpack_all_orderings(t4, nocc).contiguous()
    spin4(T.view(-1, nv, nv, nv, nv), "P4_201")
    o, v = slice(0, nocc), slice(nocc, None)
    R = torch.zeros((nocc,) * 3 + (nv,) * 3, dtype=t4.dtype, device=t4.device)
    _einsum(kind, "me,mxyzeabc->xyzabc", fock[o, v].contiguous(), T, R, 1.0)
    R *= _w3(nocc, t4.device)[:, :, :, None, None, None]
    _einsum(kind, "amef,mxyzfebc->xyzabc", eris[v, o, v, v].contiguous(), T, R, 0.5)
    _einsum(kind, "myen,mxyzeabc->xnzabc", eris[o, o, v, o].contiguous(), T, R, -0.5)
    r3 += R
    return r3
