"""Dense T3 residual contractions on the tensor cores (split-BF16x3 / TF32x3
with FP32 accumulation, FP64 results) and their plain FP64 counterparts.

The reference evaluates these as per-block `_einsum` calls with
out=..., alpha, beta (distr_cc/rccsdt.py:385-427).  Here the whole batch of
canonical blocks is one GEMM per einsum string: the FP64 operands are split
once into two pieces (x = hi + lo), the GEMM accumulates
A_hi B_hi + A_hi B_lo + A_lo B_hi in tensor memory, and the epilogue adds the
result straight into the FP64 r3 with the einsum's output permutation.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L

f64 = torch.float64

KIND = {"bf16x3": 0, "tf32x3": 1}
_KBLK = {0: 64, 1: 32}

_split = L.bind("dcc_split_operand_at", [L.c_vp, L.c_vp, L.c_vp] + [L.c_i64] * 5 + [L.c_vp, L.c_int, L.c_vp])
_gemm = L.bind("dcc_gemm_split3_ld", [L.c_vp, L.c_vp, L.c_i64, L.c_vp, L.c_vp] + [L.c_i64] * 4 +
               [L.c_vp, L.c_vp, L.c_dbl, L.c_dbl, L.c_int, L.c_vp, L.c_vp])

BIG = 1 << 30  # radix that makes a digit of a map a plain stride (< 2^31)


def lin(s):
    """m -> m * s."""
    return (1, BIG, 0, 0, s)


def two(d, s1, s2):
    """m -> (m / d) * s1 + (m % d) * s2."""
    return (1, d, s1, 0, s2)


def three(R1, R2, S0, S1, S2):
    """m -> (m / (R1 R2)) * S0 + ((m / R2) % R1) * S1 + (m % R2) * S2."""
    return (R1, R2, S0, S1, S2)


def _i64x10(f, g):
    """Two three-digit maps as the HOST int64[10] the C ABI takes."""
    v = tuple(f) + tuple(g)
    if len(v) != 10:
        raise ValueError("a map pair needs 2 x 5 values")
    return (ctypes.c_int64 * 10)(*[int(x) for x in v])


def padded_k(K, kind):
    b = _KBLK[kind]
    return (K + b - 1) // b * b


class Split:
    """Two-piece K-major copy of an FP64 operand: rows M, contraction K padded to Kp.

    With pieces=[K0, K1, ...] the contraction is the concatenation of several
    operands (each piece starts on a multiple of 8 columns; the gaps and the
    tail are zero), filled one by one with fill_piece."""

    def __init__(self, M, K=None, kind=0, device="cuda", buffers=None, pieces=None):
        self.M, self.kind = int(M), int(kind)
        if pieces is None:
            pieces = [int(K)]
        offs, o = [], 0
        for k in pieces:
            offs.append(o)
            o += (int(k) + 7) // 8 * 8
        self.K = o if len(pieces) > 1 else int(pieces[0])
        self.Kp = padded_k(self.K, self.kind)
        ends = offs[1:] + [self.Kp]
        self.pieces = [(off, int(k), end - off) for off, k, end in zip(offs, pieces, ends)]
        dt = torch.bfloat16 if self.kind == 0 else torch.float32
        if buffers is None:
            self.hi = torch.empty((self.M, self.Kp), dtype=dt, device=device)
            self.lo = torch.empty((self.M, self.Kp), dtype=dt, device=device)
        else:
            self.hi, self.lo = buffers

    def fill_piece(self, i, src, fm, fk):
        """Columns of piece i: dst[m][off + k] = src[fm(m) + fk(k)] (zero past the piece's K)."""
        L.as_tensor(src, f64, "src")
        off, k, w = self.pieces[i]
        L.check(_split(L.ptr(src), L.ptr(self.hi), L.ptr(self.lo), self.M, k, w, self.Kp, off, _i64x10(fm, fk),
                       self.kind, L.stream_ptr()))
        return self

    def fill(self, src, fm, fk):
        """dst[m][k] = src[fm(m) + fk(k)] for three-digit maps fm, fk."""
        if len(self.pieces) != 1:
            raise ValueError("a K-concatenated operand is filled with fill_piece")
        return self.fill_piece(0, src, fm, fk)


def gemm_(A, B, C, frow, fcol, alpha=1.0, beta=1.0, status=None, Kp=None):
    """C[frow(m) + fcol(n)] = alpha * A B^T + beta * C (A: Split [M,K], B: Split [N,K]).

    Kp (default: both operands' padded K) contracts only the leading Kp columns."""
    if A.kind != B.kind:
        raise ValueError("A and B must be split with the same kind")
    if Kp is None:
        if A.Kp != B.Kp:
            raise ValueError("A and B must have the same padded K (or pass Kp)")
        Kp = A.Kp
    if Kp > A.Kp or Kp > B.Kp:
        raise ValueError("Kp exceeds an operand's columns")
    L.as_tensor(C, f64, "C")
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=C.device)
    L.check(_gemm(L.ptr(A.hi), L.ptr(A.lo), A.Kp, L.ptr(B.hi), L.ptr(B.lo), B.Kp, A.M, B.M, int(Kp), L.ptr(C),
                  _i64x10(frow, fcol), float(alpha), float(beta), A.kind, L.ptr(status), L.stream_ptr()))
    return status


def matmul_split3(A, B, kind="bf16x3"):
    """A @ B^T in split precision (test helper): A [M,K], B [N,K] FP64 CUDA tensors."""
    k = KIND[kind]
    M, K = A.shape
    N = B.shape[0]
    a = Split(M, K, k).fill(A.contiguous(), lin(K), lin(1))
    b = Split(N, K, k).fill(B.contiguous(), lin(K), lin(1))
    C = torch.zeros((M, N), dtype=f64, device=A.device)
    st = gemm_(a, b, C, lin(N), lin(1), 1.0, 0.0)
    return C, st


# ----------------------------------------------------------------------------
# W_vvvv . t3 (distr_cc/rccsdt.py:421-427), all canonical blocks at once
#   r3[q,a,b,c] += sum_de W[a,b,d,e] t3[q,d,e,c]     'abde,dec->abc'
#   r3[q,a,b,c] += sum_de W[a,c,d,e] t3[q,d,b,e]     'acde,dbe->abc'
#   r3[q,a,b,c] += sum_de W[b,c,d,e] t3[q,a,d,e]     'bcde,ade->abc'
# ----------------------------------------------------------------------------

def wvvvv_maps(nv):
    """(A row map, A k map, out row map, out col map) of the three einsum strings
    for blocks of nv^3 (A rows and out rows run over (q, free index))."""
    n2, n3 = nv * nv, nv ** 3
    return [
        # 'abde,dec->abc': rows (q,c), K (d,e): t3[q][d][e][c]; out r3[q][a][b][c] = (q,c) x (a,b)
        (two(nv, n3, 1), lin(nv), two(nv, n3, 1), lin(nv)),
        # 'acde,dbe->abc': rows (q,b), K (d,e): t3[q][d][b][e]; out (q,b) x (a,c)
        (two(nv, n3, nv), two(nv, n2, 1), two(nv, n3, nv), two(nv, n2, 1)),
        # 'bcde,ade->abc': rows (q,a), K (d,e): t3[q][a][d][e]; out (q,a) x (b,c)
        (lin(n2), lin(1), two(nv, n3, n2), lin(1)),
    ]


class WvvvvT3:
    """Split-precision W_vvvv . t3 for a fixed (nblocks, nvir); buffers are reused across calls.

    With F given, the three F_vv . t3 strings (distr_cc/rccsdt.py:400-402) ride
    along in the same GEMMs: over the contraction pair (d,e),
      'ad,dbc' + 'bd,adc' = (F[a,d] delta(b,e) + delta(a,d) F[b,e]) t3[q,d,e,c]   (first GEMM)
      'cd,abd'            = delta(b,d) F[c,e] t3[q,a,d,e]                          (third GEMM)
    so the first and third GEMMs take W plus those rank-deficient terms."""

    def __init__(self, nblocks, nvir, kind="bf16x3", device="cuda"):
        self.n, self.nv, self.kind = int(nblocks), int(nvir), KIND[kind]
        K = nvir * nvir
        self.W = Split(K, K, self.kind, device)
        self.A = Split(self.n * nvir, K, self.kind, device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.maps = wvvvv_maps(nvir)
        self.WF = None

    def __call__(self, r3, W, t3, alpha=1.0, F=None):
        nv = self.nv
        L.as_tensor(r3, f64, "r3")
        L.as_tensor(t3, f64, "t3")
        if F is None:
            ws = [self.W.fill(W.reshape(nv * nv, nv * nv), lin(nv * nv), lin(1))] * 3
        else:
            if self.WF is None:
                self.WF = [Split(nv * nv, nv * nv, self.kind, r3.device) for _ in range(2)]
            W1 = W.clone()
            W1.diagonal(0, 1, 3).add_(F.unsqueeze(2))  # F[a,d] delta(b,e)
            W1.diagonal(0, 0, 2).add_(F.unsqueeze(2))  # delta(a,d) F[b,e]
            self.WF[0].fill(W1.reshape(nv * nv, nv * nv), lin(nv * nv), lin(1))
            W1.copy_(W)
            W1.diagonal(0, 0, 2).add_(F.unsqueeze(2))  # delta(b,d) F[c,e]
            self.WF[1].fill(W1.reshape(nv * nv, nv * nv), lin(nv * nv), lin(1))
            del W1
            ws = [self.WF[0], self.W.fill(W.reshape(nv * nv, nv * nv), lin(nv * nv), lin(1)), self.WF[1]]
        for (am, ak, er, ec), w in zip(self.maps, ws):
            self.A.fill(t3, am, ak)
            gemm_(self.A, w, r3, er, ec, alpha, 1.0, self.status)
        return r3


def wvvvv_t3_fp64_(r3, W, t3, alpha=1.0):
    """Plain FP64 GPU path of the same three einsums (cuBLAS DGEMM through torch)."""
    n, nv = t3.shape[0], t3.shape[1]
    W2 = W.reshape(nv * nv, nv * nv)
    # 'abde,dec->abc': (ab) x (de) . (de) x c per block
    r3.view(n, nv * nv, nv).add_(torch.matmul(W2, t3.view(n, nv * nv, nv)), alpha=alpha)
    # 'acde,dbe->abc': X[q,b,(ac)] = t3[q][d][b][e] as [q][b][(de)] . W2^T
    X = torch.matmul(t3.permute(0, 2, 1, 3).reshape(n, nv, nv * nv), W2.t())  # [q][b][(a c)]
    r3.add_(X.view(n, nv, nv, nv).permute(0, 2, 1, 3), alpha=alpha)
    # 'bcde,ade->abc': [q a][(de)] . W2^T -> [q a][(bc)]
    r3.view(n * nv, nv * nv).add_(torch.matmul(t3.view(n * nv, nv * nv), W2.t()), alpha=alpha)
    return r3


def wvvvv_flops(nblocks, nvir):
    """Algorithmic FLOPs of the three einsums (2 M N K each)."""
    return 3 * 2 * nblocks * nvir ** 5


def einsum_reference(W, t3):
    """numpy FP64 restatement of the three einsums (test oracle helper)."""
    r = np.zeros_like(t3)
    for q in range(t3.shape[0]):
        r[q] += np.einsum("abde,dec->abc", W, t3[q])
        r[q] += np.einsum("acde,dbe->abc", W, t3[q])
        r[q] += np.einsum("bcde,ade->abc", W, t3[q])
    return r
