"""Plain FP64 torch formulation of the (Q) task loop (the oracle's restatement of
distr_cc/rccsdt_q.py:976-1160 in torch ops: task blocks by einsum, the masked
division, P4_444 as its three transposition stages, the factor and the two dot
products), differentiable by autograd: the reference the hand-written (Q)
adjoint is checked against.  Small sizes only."""
import torch

from adjoint_ref import unpack_torch


def _factor(a, b, c, d):
    if a < b < c < d:
        return 24.0
    if (a == b < c < d) or (a < b == c < d) or (a < b < c == d):
        return 12.0
    if a == b < c == d:
        return 6.0
    return 0.0


def _p4_444(x):
    """P4_444 over the last four (occupied) axes of x: T1 = 2A - A(ab) - A(ac) - A(ad),
    T2 = 2T1 - T1(bc) - T1(bd), R = 2T2 - T2(cd)."""
    n = x.dim()
    i, j, k, l = n - 4, n - 3, n - 2, n - 1
    t1 = 2 * x - x.transpose(i, j) - x.transpose(i, k) - x.transpose(i, l)
    t2 = 2 * t1 - t1.transpose(j, k) - t1.transpose(j, l)
    return 2 * t2 - t2.transpose(k, l)


def q_energy_torch(er, t2, t3, eo, ev, blk):
    """(e_bracket, e_paren) of canonical t3 blocks (torch, differentiable)."""
    e = torch.einsum
    nocc, nvir = eo.numel(), ev.numel()
    T = unpack_torch(t3, nocc).permute(3, 4, 5, 0, 1, 2)  # T[a,b,c,i,j,k]
    vvvo, vooo, vvoo = er["vvvo"], er["vooo"], er["vvoo"]
    ovvo, ovov, vvvv, oooo = er["ovvo"], er["ovov"], er["vvvv"], er["oooo"]

    def Wv(X, Y, Z):
        W = 0.5 * e('abef,fcjk->abcejk', vvvv[X, Y], t2[:, Z])
        W = W + 0.5 * e('acef,fbkj->abcejk', vvvv[X, Z], t2[:, Y])
        W = W - e('mbej,acmk->abcejk', ovvo[:, Y], t2[X, Z]) - e('mcek,abmj->abcejk', ovvo[:, Z], t2[X, Y])
        W = W - e('maje,bcmk->abcejk', ovov[:, X], t2[Y, Z]) - e('make,cbmj->abcejk', ovov[:, X], t2[Z, Y])
        return W

    def Vo(X, Y):
        return -0.5 * e('mnki,abnj->abmijk', oooo, t2[X, Y]) - 0.5 * e('mnkj,bani->abmijk', oooo, t2[Y, X])

    pr = lambda n: [(i, min(i + blk, n)) for i in range(0, n, blk)]  # noqa: E731
    eb = ep = 0.0
    for d0, d1 in pr(nvir):
        for c0, c1 in pr(d1):
            for b0, b1 in pr(c1):
                for a0, a1 in pr(b1):
                    A, B, C, D = slice(a0, a1), slice(b0, b1), slice(c0, c1), slice(d0, d1)
                    t = T[A, B]
                    z = (e('cdel,abeijk->abcdijkl', vvvo[C, D], t) + e('dcek,abeijl->abcdijkl', vvvo[D, C], t)
                         - e('dmli,abcmjk->abcdijkl', vooo[D], t[:, :, C]) - e('dmlj,abcimk->abcdijkl', vooo[D], t[:, :, C])
                         - e('cmki,abdmjl->abcdijkl', vooo[C], t[:, :, D]) - e('cmkj,abdiml->abcdijkl', vooo[C], t[:, :, D]))
                    t = T[A, C]
                    z = z + e('bdel,aceikj->abcdijkl', vvvo[B, D], t) + e('dbej,aceikl->abcdijkl', vvvo[D, B], t)
                    z = z - e('bmji,acdmkl->abcdijkl', vooo[B], t[:, :, D]) - e('bmjk,acdiml->abcdijkl', vooo[B], t[:, :, D])
                    z = z - e('dmlk,acbimj->abcdijkl', vooo[D], t[:, :, B])
                    t = T[A, D]
                    z = z + e('bcek,adeilj->abcdijkl', vvvo[B, C], t) + e('cbej,adeilk->abcdijkl', vvvo[C, B], t)
                    z = z - e('bmjl,adcimk->abcdijkl', vooo[B], t[:, :, C]) - e('cmkl,adbimj->abcdijkl', vooo[C], t[:, :, B])
                    t = T[B, C]
                    z = z + e('adel,bcejki->abcdijkl', vvvo[A, D], t) + e('daei,bcejkl->abcdijkl', vvvo[D, A], t)
                    z = z - e('amij,bcdmkl->abcdijkl', vooo[A], t[:, :, D]) - e('amik,bcdjml->abcdijkl', vooo[A], t[:, :, D])
                    t = T[B, D]
                    z = z + e('acek,bdejli->abcdijkl', vvvo[A, C], t) + e('caei,bdejlk->abcdijkl', vvvo[C, A], t)
                    z = z - e('amil,bdcjmk->abcdijkl', vooo[A], t[:, :, C])
                    t = T[C, D]
                    z = z + e('abej,cdekli->abcdijkl', vvvo[A, B], t) + e('baei,cdeklj->abcdijkl', vvvo[B, A], t)
                    x = (e('abcejk,edil->abcdijkl', Wv(A, B, C), t2[:, D]) + e('abdejl,ecik->abcdijkl', Wv(A, B, D), t2[:, C])
                         + e('acdekl,ebij->abcdijkl', Wv(A, C, D), t2[:, B]) + e('baceik,edjl->abcdijkl', Wv(B, A, C), t2[:, D])
                         + e('badeil,ecjk->abcdijkl', Wv(B, A, D), t2[:, C]) + e('bcdekl,eaji->abcdijkl', Wv(B, C, D), t2[:, A])
                         + e('cabeij,edkl->abcdijkl', Wv(C, A, B), t2[:, D]) + e('cadeil,ebkj->abcdijkl', Wv(C, A, D), t2[:, B])
                         + e('cbdejl,eaki->abcdijkl', Wv(C, B, D), t2[:, A]) + e('dabeij,eclk->abcdijkl', Wv(D, A, B), t2[:, C])
                         + e('daceik,eblj->abcdijkl', Wv(D, A, C), t2[:, B]) + e('dbcejk,eali->abcdijkl', Wv(D, B, C), t2[:, A]))
                    x = x - e('abmijk,cdml->abcdijkl', Vo(A, B), t2[C, D]) - e('abmijl,dcmk->abcdijkl', Vo(A, B), t2[D, C])
                    x = x - e('acmikj,bdml->abcdijkl', Vo(A, C), t2[B, D]) - e('acmikl,dbmj->abcdijkl', Vo(A, C), t2[D, B])
                    x = x - e('admilj,bcmk->abcdijkl', Vo(A, D), t2[B, C]) - e('admilk,cbmj->abcdijkl', Vo(A, D), t2[C, B])
                    x = x - e('bcmjki,adml->abcdijkl', Vo(B, C), t2[A, D]) - e('bcmjkl,dami->abcdijkl', Vo(B, C), t2[D, A])
                    x = x - e('bdmjli,acmk->abcdijkl', Vo(B, D), t2[A, C]) - e('bdmjlk,cami->abcdijkl', Vo(B, D), t2[C, A])
                    x = x - e('cdmkli,abmj->abcdijkl', Vo(C, D), t2[A, B]) - e('cdmklj,bami->abcdijkl', Vo(C, D), t2[B, A])
                    den = (eo[:, None, None, None] + eo[None, :, None, None] + eo[None, None, :, None]
                           + eo[None, None, None, :])
                    vsum = (ev[A][:, None, None, None] + ev[B][None, :, None, None] + ev[C][None, None, :, None]
                            + ev[D][None, None, None, :])
                    D8 = den[None, None, None, None] - vsum[..., None, None, None, None]
                    X = torch.where(D8.abs() > 1e-15, (x + z) / D8, torch.zeros_like(D8))
                    f = torch.tensor([[[[_factor(a, b, c, d) for d in range(d0, d1)] for c in range(c0, c1)]
                                       for b in range(b0, b1)] for a in range(a0, a1)], dtype=x.dtype, device=x.device)
                    Y = f[..., None, None, None, None] * _p4_444(X)
                    zsq = (e('abij,cdkl->abcdijkl', vvoo[A, B], t2[C, D]) + e('acik,bdjl->abcdijkl', vvoo[A, C], t2[B, D])
                           + e('adil,bcjk->abcdijkl', vvoo[A, D], t2[B, C]) + e('bcjk,adil->abcdijkl', vvoo[B, C], t2[A, D])
                           + e('bdjl,acik->abcdijkl', vvoo[B, D], t2[A, C]) + e('cdkl,abij->abcdijkl', vvoo[C, D], t2[A, B]))
                    br = (Y * zsq).sum() / 12.0
                    eb = eb + br
                    ep = ep + (Y * z).sum() / 12.0 + br
    return eb, ep
