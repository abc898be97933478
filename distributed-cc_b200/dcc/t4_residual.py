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
