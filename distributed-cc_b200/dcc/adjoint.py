"""Hand-written adjoint (VJP) of the batched T3 residual behind
torch.autograd.Function (the product the Lambda equations need).

Forward: r3 = compute_r3_tri(t2, t3; F_vv, F_oo, W_vvvo, W_vooo, W_vvvv,
W_ovov, W_ovvo, W_oooo) for canonical t3 blocks (distr_cc/rccsdt.py:368-732)
in the reformulated form of dcc.t3_residual,

    r3 = G(S - Y) + Wv(t3),   G: sum over the simultaneous permutations
    S = X + T1 + T2 + T5/2 + (Ws.U - F_oo.U)/2,   U = unpack(t3),

with W_oooo entering through its pair-symmetric part Ws (the form the
residual takes for the pair-symmetric W_oooo of RHF; W_oooo's antisymmetric
part is not differentiated).  Backward, for the cotangent lam of r3:

    Lam = G^T(lam) = unpack(lam_sym)      lam_sym: lam summed over each block's
                                          stabilizer (i=j, j=k, i=j=k)
    g(W, t2) from X, Y, T1, T2, T5, Ws, F_oo   contractions of Lam with U, t2, W
    gU  = the transposed T1, T2, T5, Ws, F_oo contractions of Lam
    gt3 = unpack^T(gU) + Wv^T(lam)

Gradients with respect to t3 are returned projected onto blocks symmetric
under their stabilizer (the subspace canonical T3 lives in); U is recomputed
from t3 in the backward pass instead of being stored.  Every contraction is
FP64 (torch/cuBLAS), or with precision "bf16x3"/"tf32x3" a split-precision
tcgen05 GEMM (contract.einsum_into); the forward is dcc.t3_residual.
"""
from __future__ import annotations

import torch

from . import contract, t3_residual
from .synthetic import canonical_ijk

f64 = torch.float64

NAMES = ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo")
MAX_SPLIT_K = 16384  # longer contractions of the backward accumulate in FP64


class _D:
    pass


def _stab_masks(ijk):
    i, j, k = ijk[:, 0], ijk[:, 1], ijk[:, 2]
    m = lambda c: c.to(f64)[:, None, None, None]  # noqa: E731
    return m(i == j), m(j == k), m((i == j) & (j == k))


def stab_sum(lam, ijk):
    """lam summed over each canonical block's stabilizer in S3 (acting on a, b, c)."""
    ab, bc, al = _stab_masks(ijk)
    out = lam + ab * lam.transpose(1, 2) + bc * lam.transpose(2, 3)
    out = out + al * (lam.permute(0, 3, 2, 1) + lam.permute(0, 2, 3, 1) + lam.permute(0, 3, 1, 2))
    return out


def stab_project(g, ijk):
    """Projection onto blocks symmetric under their stabilizer: stab_sum / |stabilizer|."""
    ab, bc, al = _stab_masks(ijk)
    order = 1.0 + ab + bc + 3.0 * al  # 1, 2, 2 or 6 elements
    return stab_sum(g, ijk) / order


class T3ResidualFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, W_oooo, precision):
        nocc, nvir = t2.shape[0], t2.shape[2]
        d = _D()
        for n, v in zip(NAMES, (F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, W_oooo)):
            setattr(d, n, v.contiguous())
        d.W_oooo = 0.5 * (d.W_oooo + d.W_oooo.permute(1, 0, 3, 2))  # pair-symmetric part
        d.t2 = t2.contiguous()
        d.ijk = torch.tensor(canonical_ijk(nocc), dtype=torch.int32, device=t3.device)
        res = t3_residual.T3Residual(nocc, nvir, precision, t3.device, with_oo=True)
        r3 = res.compute(d, t3.contiguous())
        if not res.status_ok():
            raise RuntimeError("a bounded wait in a GPU kernel gave up (timeout)")
        ctx.precision = precision
        ctx.save_for_backward(t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, d.W_oooo)
        return r3

    @staticmethod
    def backward(ctx, lam):
        t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, Ws = ctx.saved_tensors
        return vjp(lam, t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, Ws, ctx.precision) + (None,)


def vjp(lam, t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, Ws, precision="fp64"):
    """Gradients of <lam, r3> with respect to (t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv,
    W_ovov, W_ovvo, W_oooo)."""
    kind = None if precision == "fp64" else contract.KIND[precision]
    nocc, nvir = t2.shape[0], t2.shape[2]
    dev = t3.device
    lam = lam.contiguous()
    ijk = torch.tensor(canonical_ijk(nocc), dtype=torch.int32, device=dev)
    full = (nocc,) * 3 + (nvir,) * 3
    # Lam = G^T(lam), U = unpack(t3) (recomputed, not stored)
    Lam = torch.empty(full, dtype=f64, device=dev)
    t3_residual.unpack_all_(stab_sum(lam, ijk).contiguous(), Lam.view(nocc ** 3, nvir, nvir, nvir), nocc, nvir)
    U = torch.empty(full, dtype=f64, device=dev)
    t3_residual.unpack_all_(t3.contiguous(), U.view(nocc ** 3, nvir, nvir, nvir), nocc, nvir)

    def E(subs, X, Y, out, alpha=1.0, beta=1.0):
        # the long reductions onto the integrals (K up to nocc nvir^3) stay FP64
        return contract.einsum_into(subs, X, Y, out, alpha, beta, kind, max_k=MAX_SPLIT_K)

    z = lambda *s: torch.zeros(s, dtype=f64, device=dev)  # noqa: E731
    G2 = -0.5 * (W_ovov + W_ovvo.permute(0, 1, 3, 2))
    # X = W_vvvo.t2, Y = W_vooo.t2
    gWvvvo = E('ijkabc,ikdc->abdj', Lam, t2, z(*W_vvvo.shape), 1.0, 0.0)
    gt2 = E('ijkabc,abdj->ikdc', Lam, W_vvvo, z(*t2.shape), 1.0, 0.0)
    gWvooo = E('ijkabc,lkbc->alij', Lam, t2, z(*W_vooo.shape), -1.0, 0.0)
    E('ijkabc,alij->lkbc', Lam, W_vooo, gt2, -1.0)
    # T1, T2, T5/2 (W_ovov, W_ovvo through G2)
    gWovov = E('ijkabc,jkldca->lbid', Lam, U, z(*W_ovov.shape), -1.0, 0.0)
    gG2 = E('ijkabc,jkldcb->laid', Lam, U, z(*W_ovov.shape), 1.0, 0.0)
    gWovvo = E('ijkabc,jklbcd->ladi', Lam, U, z(*W_ovvo.shape), 0.5, 0.0)
    gWovov.add_(gG2, alpha=-0.5)
    gWovvo.add_(gG2.permute(0, 1, 3, 2), alpha=-0.5)
    # (Ws.U - F_oo.U) / 2
    gWs = E('ijkabc,lmkabc->lmij', Lam, U, z(*Ws.shape), 0.5, 0.0)
    gWoooo = 0.5 * (gWs + gWs.permute(1, 0, 3, 2))
    gFoo = E('ijkabc,ljkabc->li', Lam, U, z(*F_oo.shape), -0.5, 0.0)
    del U
    gU = torch.empty(full, dtype=f64, device=dev)
    E('ijkabc,lbid->jkldca', Lam, W_ovov, gU, -1.0, 0.0)
    E('ijkabc,laid->jkldcb', Lam, G2, gU)
    E('ijkabc,ladi->jklbcd', Lam, W_ovvo, gU, 0.5)
    E('ijkabc,lmij->lmkabc', Lam, Ws, gU, 0.5)
    E('ijkabc,li->ljkabc', Lam, F_oo, gU, -0.5)
    del Lam
    # unpack^T then the projection: (1/|stab|) * sum over all six permutations
    gt3 = torch.empty_like(t3)
    t3_residual.perm_gather_(gt3, ijk, nvir, 0.0, [(gU.view(nocc ** 3, nvir, nvir, nvir), 1.0,
                                                     t3_residual.full_strides(nocc, nvir), t3_residual.ALL_S3)])
    ab, bc, al = _stab_masks(ijk)
    gt3.div_(1.0 + ab + bc + 3.0 * al)
    del gU
    # W_vvvv.t3 and F_vv.t3 (distr_cc/rccsdt.py:400-427) on canonical t3
    gWvvvv = E('qabc,qdec->abde', lam, t3, z(*W_vvvv.shape), 1.0, 0.0)
    E('qabc,qdbe->acde', lam, t3, gWvvvv)
    E('qabc,qade->bcde', lam, t3, gWvvvv)
    gFvv = E('qabc,qdbc->ad', lam, t3, z(*F_vv.shape), 1.0, 0.0)
    E('qabc,qadc->bd', lam, t3, gFvv)
    E('qabc,qabd->cd', lam, t3, gFvv)
    gd = z(*t3.shape)
    E('qabc,abde->qdec', lam, W_vvvv, gd)
    E('qabc,acde->qdbe', lam, W_vvvv, gd)
    E('qabc,bcde->qade', lam, W_vvvv, gd)
    E('qabc,ad->qdbc', lam, F_vv, gd)
    E('qabc,bd->qadc', lam, F_vv, gd)
    E('qabc,cd->qabd', lam, F_vv, gd)
    gt3.add_(stab_project(gd, ijk))
    return gt2, gt3, gFvv, gFoo, gWvvvo, gWvooo, gWvvvv, gWovov, gWovvo, gWoooo


def t3_residual_fn(t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, W_oooo, precision="fp64"):
    """Differentiable r3 (canonical blocks) with the hand-written backward above."""
    return T3ResidualFunction.apply(t2, t3, F_vv, F_oo, W_vvvo, W_vooo, W_vvvv, W_ovov, W_ovvo, W_oooo, precision)
