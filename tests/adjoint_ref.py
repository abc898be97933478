"""Plain FP64 torch.einsum formulation of compute_r3_tri (the reformulated,
all-ordered-block form whose equality with the reference's literal per-block
einsums is checked in tests/test_residual_algebra.py), differentiable by
autograd: the reference the hand-written adjoint is checked against."""
import itertools

import torch


def unpack_torch(t3, nocc):
    """U[x,y,z] = t3[canonical(x,y,z)] with (a,b,c) permuted along (autograd-friendly)."""
    trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
    index = {t: q for q, t in enumerate(trip)}
    blocks = []
    for x, y, z in itertools.product(range(nocc), repeat=3):
        o = (x, y, z)
        srt = sorted(range(3), key=lambda m: (o[m], m))  # positions of the sorted entries
        q = index[tuple(o[m] for m in srt)]
        # U[o][v] = t3[q][w] with v[m] = w[rank of m]: axis m of U is axis rank(m) of t3
        rank = [srt.index(m) for m in range(3)]
        blocks.append(t3[q].permute(*rank))
    nv = t3.shape[1]
    return torch.stack(blocks).view((nocc,) * 3 + (nv,) * 3)


def r3_torch(t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, W_oooo):
    nocc = t2.shape[0]
    e = torch.einsum
    U = unpack_torch(t3, nocc)
    G2 = -0.5 * (W_ovov + W_ovvo.permute(0, 1, 3, 2))
    Ws = 0.5 * (W_oooo + W_oooo.permute(1, 0, 3, 2))
    S = (e('abdj,ikdc->ijkabc', W_vvvo, t2) - e('lbid,jkldca->ijkabc', W_ovov, U)
         + e('laid,jkldcb->ijkabc', G2, U) + 0.5 * e('ladi,jklbcd->ijkabc', W_ovvo, U)
         + 0.5 * e('lmij,lmkabc->ijkabc', Ws, U) - 0.5 * e('li,ljkabc->ijkabc', F_oo, U))
    S = S - e('alij,lkbc->ijkabc', W_vooo, t2)
    R = sum(S.permute(*(p + tuple(3 + x for x in p))) for p in itertools.permutations(range(3)))
    trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
    r3 = torch.stack([R[i, j, k] for i, j, k in trip])
    r3 = r3 + e('ad,qdbc->qabc', F_vv, t3) + e('bd,qadc->qabc', F_vv, t3) + e('cd,qabd->qabc', F_vv, t3)
    r3 = r3 + e('abde,qdec->qabc', W_vvvv, t3) + e('acde,qdbe->qabc', W_vvvv, t3) + e('bcde,qade->qabc', W_vvvv, t3)
    return r3
