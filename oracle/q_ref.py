"""TEST ORACLE ONLY -- numpy FP64 restatement of the RCCSDT(Q) energy task
loop of the reference (distr_cc/rccsdt_q.py:302-314 task list, :390-428 W
builders and factor, :976-1160 task body), one rank, all tasks.  The einsum
strings are the reference's, applied to slices of a full T3[a,b,c,i,j,k]
(the reference reads the same values from its ABC-ordered T3 through
fill_t3_from_ptr_array).  The division, P4_444 and factor steps call the C
restatement in dcc_oracle.c (pinned bit for bit against the reference's
src/rccsdt_q.c).  Slow by design: small sizes only; never shipped.

Tensors (physicist ERI slices as the reference's eris.pppp[...] cuts):
  eris_vvvo[a,b,c,i], eris_vooo[a,i,j,k], eris_vvoo[a,b,i,j], eris_ovvo[i,a,b,j],
  eris_ovov[i,a,j,b], eris_vvvv[a,b,c,d], eris_oooo[i,j,k,l], t2[a,b,i,j] (vvoo order),
  T[a,b,c,i,j,k] full T3.
"""
from __future__ import annotations

import numpy as np

from .oracle import Oracle


def prange(start, stop, step):
    return [(i, min(i + step, stop)) for i in range(start, stop, step)]


def task_list(nvir, blksize):
    """The reference's canonical task order (distr_cc/rccsdt_q.py:302-314)."""
    tasks = []
    for d0, d1 in prange(0, nvir, blksize):
        for c0, c1 in prange(0, d1, blksize):
            for b0, b1 in prange(0, c1, blksize):
                for a0, a1 in prange(0, b1, blksize):
                    tasks.append((a0, a1, a1 - a0, b0, b1, b1 - b0, c0, c1, c1 - c0, d0, d1, d1 - d0))
    return tasks


def task_blocks(er, t2, T, task, blksize):
    """z4 (T3-connected) and t4 (T2-connected) of one task (a0, a1, ba, b0, b1, bb,
    c0, c1, bc, d0, d1, bd), [blk]^4 x [nocc]^4 (distr_cc/rccsdt_q.py:1014-1129)."""
    e = np.einsum
    blk = blksize
    nocc = T.shape[3]
    vvvo, vooo = er["vvvo"], er["vooo"]
    ovvo, ovov, vvvv, oooo = er["ovvo"], er["ovov"], er["vvvv"], er["oooo"]

    def W_vvvvoo(a0, a1, b0, b1, c0, c1):
        W = 0.5 * e('abef,fcjk->abcejk', vvvv[a0:a1, b0:b1], t2[:, c0:c1])
        W += 0.5 * e('acef,fbkj->abcejk', vvvv[a0:a1, c0:c1], t2[:, b0:b1])
        W -= e('mbej,acmk->abcejk', ovvo[:, b0:b1], t2[a0:a1, c0:c1])
        W -= e('mcek,abmj->abcejk', ovvo[:, c0:c1], t2[a0:a1, b0:b1])
        W -= e('maje,bcmk->abcejk', ovov[:, a0:a1], t2[b0:b1, c0:c1])
        W -= e('make,cbmj->abcejk', ovov[:, a0:a1], t2[c0:c1, b0:b1])
        return W

    def W_vvoooo(a0, a1, b0, b1):
        W = -0.5 * e('mnki,abnj->abmijk', oooo, t2[a0:a1, b0:b1])
        W -= 0.5 * e('mnkj,bani->abmijk', oooo, t2[b0:b1, a0:a1])
        return W

    (a0, a1, ba, b0, b1, bb, c0, c1, bc, d0, d1, bd) = task
    A, B, C, D = slice(a0, a1), slice(b0, b1), slice(c0, c1), slice(d0, d1)
    z4 = np.zeros((blk,) * 4 + (nocc,) * 4)
    t4 = np.zeros_like(z4)
    z = z4[:ba, :bb, :bc, :bd]
    t = T[A, B]
    z += e('cdel,abeijk->abcdijkl', vvvo[C, D], t)
    z += e('dcek,abeijl->abcdijkl', vvvo[D, C], t)
    z -= e('dmli,abcmjk->abcdijkl', vooo[D], t[:, :, C])
    z -= e('dmlj,abcimk->abcdijkl', vooo[D], t[:, :, C])
    z -= e('cmki,abdmjl->abcdijkl', vooo[C], t[:, :, D])
    z -= e('cmkj,abdiml->abcdijkl', vooo[C], t[:, :, D])
    t = T[A, C]
    z += e('bdel,aceikj->abcdijkl', vvvo[B, D], t)
    z += e('dbej,aceikl->abcdijkl', vvvo[D, B], t)
    z -= e('bmji,acdmkl->abcdijkl', vooo[B], t[:, :, D])
    z -= e('bmjk,acdiml->abcdijkl', vooo[B], t[:, :, D])
    z -= e('dmlk,acbimj->abcdijkl', vooo[D], t[:, :, B])
    t = T[A, D]
    z += e('bcek,adeilj->abcdijkl', vvvo[B, C], t)
    z += e('cbej,adeilk->abcdijkl', vvvo[C, B], t)
    z -= e('bmjl,adcimk->abcdijkl', vooo[B], t[:, :, C])
    z -= e('cmkl,adbimj->abcdijkl', vooo[C], t[:, :, B])
    t = T[B, C]
    z += e('adel,bcejki->abcdijkl', vvvo[A, D], t)
    z += e('daei,bcejkl->abcdijkl', vvvo[D, A], t)
    z -= e('amij,bcdmkl->abcdijkl', vooo[A], t[:, :, D])
    z -= e('amik,bcdjml->abcdijkl', vooo[A], t[:, :, D])
    t = T[B, D]
    z += e('acek,bdejli->abcdijkl', vvvo[A, C], t)
    z += e('caei,bdejlk->abcdijkl', vvvo[C, A], t)
    z -= e('amil,bdcjmk->abcdijkl', vooo[A], t[:, :, C])
    t = T[C, D]
    z += e('abej,cdekli->abcdijkl', vvvo[A, B], t)
    z += e('baei,cdeklj->abcdijkl', vvvo[B, A], t)

    x = t4[:ba, :bb, :bc, :bd]
    x += e('abcejk,edil->abcdijkl', W_vvvvoo(a0, a1, b0, b1, c0, c1), t2[:, D])
    x += e('abdejl,ecik->abcdijkl', W_vvvvoo(a0, a1, b0, b1, d0, d1), t2[:, C])
    x += e('acdekl,ebij->abcdijkl', W_vvvvoo(a0, a1, c0, c1, d0, d1), t2[:, B])
    x += e('baceik,edjl->abcdijkl', W_vvvvoo(b0, b1, a0, a1, c0, c1), t2[:, D])
    x += e('badeil,ecjk->abcdijkl', W_vvvvoo(b0, b1, a0, a1, d0, d1), t2[:, C])
    x += e('bcdekl,eaji->abcdijkl', W_vvvvoo(b0, b1, c0, c1, d0, d1), t2[:, A])
    x += e('cabeij,edkl->abcdijkl', W_vvvvoo(c0, c1, a0, a1, b0, b1), t2[:, D])
    x += e('cadeil,ebkj->abcdijkl', W_vvvvoo(c0, c1, a0, a1, d0, d1), t2[:, B])
    x += e('cbdejl,eaki->abcdijkl', W_vvvvoo(c0, c1, b0, b1, d0, d1), t2[:, A])
    x += e('dabeij,eclk->abcdijkl', W_vvvvoo(d0, d1, a0, a1, b0, b1), t2[:, C])
    x += e('daceik,eblj->abcdijkl', W_vvvvoo(d0, d1, a0, a1, c0, c1), t2[:, B])
    x += e('dbcejk,eali->abcdijkl', W_vvvvoo(d0, d1, b0, b1, c0, c1), t2[:, A])
    W = W_vvoooo(a0, a1, b0, b1)
    x -= e('abmijk,cdml->abcdijkl', W, t2[C, D])
    x -= e('abmijl,dcmk->abcdijkl', W, t2[D, C])
    W = W_vvoooo(a0, a1, c0, c1)
    x -= e('acmikj,bdml->abcdijkl', W, t2[B, D])
    x -= e('acmikl,dbmj->abcdijkl', W, t2[D, B])
    W = W_vvoooo(a0, a1, d0, d1)
    x -= e('admilj,bcmk->abcdijkl', W, t2[B, C])
    x -= e('admilk,cbmj->abcdijkl', W, t2[C, B])
    W = W_vvoooo(b0, b1, c0, c1)
    x -= e('bcmjki,adml->abcdijkl', W, t2[A, D])
    x -= e('bcmjkl,dami->abcdijkl', W, t2[D, A])
    W = W_vvoooo(b0, b1, d0, d1)
    x -= e('bdmjli,acmk->abcdijkl', W, t2[A, C])
    x -= e('bdmjlk,cami->abcdijkl', W, t2[C, A])
    W = W_vvoooo(c0, c1, d0, d1)
    x -= e('cdmkli,abmj->abcdijkl', W, t2[A, B])
    x -= e('cdmklj,bami->abcdijkl', W, t2[B, A])
    return z4, t4


def q_energy_ref(er, t2, T, e_occ, e_vir, blksize, orc=None, tasks=None):
    """(e_bracket, e_paren) summed over `tasks` (default: all) in task order."""
    orc = orc or Oracle()
    e = np.einsum
    nvir = e_vir.size
    nocc = e_occ.size
    blk = blksize
    vvoo = er["vvoo"]

    def factor(a0, a1, b0, b1, c0, c1, d0, d1):
        f = np.zeros((blk,) * 4)
        for a in range(a0, a1):
            for b in range(b0, b1):
                for c in range(c0, c1):
                    for d in range(d0, d1):
                        f[a - a0, b - b0, c - c0, d - d0] = orc.q_factor(a, b, c, d)
        return f

    eb = ep = 0.0
    for task in (tasks if tasks is not None else task_list(nvir, blk)):
        (a0, a1, ba, b0, b1, bb, c0, c1, bc, d0, d1, bd) = task
        A, B, C, D = slice(a0, a1), slice(b0, b1), slice(c0, c1), slice(d0, d1)
        z4, t4 = task_blocks(er, t2, T, task, blk)
        # epilogue (distr_cc/rccsdt_q.py:1131-1154)
        t4 += z4
        orc.e_abcdijkl_division(t4, e_occ, e_vir, a0, a1, b0, b1, c0, c1, d0, d1, blk, blk, blk, nocc)
        orc.t4_spin_sum(t4, blk ** 4, nocc, "P4_444", 1.0, 0.0)
        orc.t4_multiply_factor(t4, factor(a0, a1, b0, b1, c0, c1, d0, d1), blk, blk, blk, blk, nocc)
        paren = float(np.dot(t4.ravel(), z4.ravel())) / 12.0
        zs = z4[:ba, :bb, :bc, :bd]
        zs[...] = e('abij,cdkl->abcdijkl', vvoo[A, B], t2[C, D])
        zs += e('acik,bdjl->abcdijkl', vvoo[A, C], t2[B, D])
        zs += e('adil,bcjk->abcdijkl', vvoo[A, D], t2[B, C])
        zs += e('bcjk,adil->abcdijkl', vvoo[B, C], t2[A, D])
        zs += e('bdjl,acik->abcdijkl', vvoo[B, D], t2[A, C])
        zs += e('cdkl,abij->abcdijkl', vvoo[C, D], t2[A, B])
        bracket = float(np.dot(t4.ravel(), z4.ravel())) / 12.0
        eb += bracket
        ep += paren + bracket
    return eb, ep
