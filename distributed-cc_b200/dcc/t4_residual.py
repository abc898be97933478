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


def build_intermediates(eris, W_oooo, W_ovov, W_vvvv, t2, t3, t3p, t4, nocc, spin4):
    """The W builders of distr_cc/rccsdtq.py:700-833 as full tensors (FP64, torch)."""
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
    T4s = unpack_all_orderings(t4, nocc)
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


def compute_r4_tri_(r4, eris, F_vv, W_vvvo, W_vooo, W_vvvv, W_oooo, W_ovov, t2, t3, t4, nocc, precision="fp64",
                    spin3=None, spin4=None, F_oo=None, W_ovvo=None, forms=None):
    """r4[stored blocks] = compute_r4_tri (distr_cc/rccsdtq.py:834-1060); with F_oo and W_ovvo
    given it includes the OO batch (oo_batch_, :1062-1349), else it stops before it.

    eris: t1-dressed ERIs [nmo]^4 (the reference's imds.t1_eris); t2 [i,j,a,b]; t3 full
    [i,j,k,a,b,c]; t4 and r4 [nstored, nvir^4] in stored_quadruples order.  spin3 / spin4
    apply P3_201 / P4_201 in place to [n, nvir^3] / [n, nvir^4] blocks (default: this
    library's kernels).

    The ~100 per-block strings of distr_cc/rccsdtq.py:862-1033 each run as ONE batched
    contraction over the stored blocks: every operand is cut at the block's occupied slots
    for all blocks at once (_gather_slots) and the strings contract over the remaining
    virtual (and summed occupied) indices with the block as the batch index, straight into
    r4 -- the work and memory of the stored blocks only.  Their contractions are short
    (K = nvir or nocc), so they stay FP64 in every precision; precision "bf16x3"/"tf32x3"
    runs the W_vvvv.t4 strings (K = nvir^2) as split GEMMs; the builders stay FP64."""
    from . import _c_rccsdt, _c_rccsdt_q
    kind = None if precision == "fp64" else contract.KIND[precision]
    nv = t2.shape[2]
    if spin3 is None:
        spin3 = lambda A: _c_rccsdt.t3_spin_summation_inplace_(A, A.numel() // nv ** 3, nv, "P3_201", 1.0, 0.0)  # noqa: E731
    if spin4 is None:
        spin4 = lambda A: _c_rccsdt_q.t4_spin_summation_inplace_(A, A.numel() // nv ** 4, nv, "P4_201", 1.0, 0.0)  # noqa: E731
    t3 = t3.contiguous()
    t3p = t3.clone()
    spin3(t3p)
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
