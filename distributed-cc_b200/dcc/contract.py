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

_split = L.bind("dcc_split_operand_at4", [L.c_vp, L.c_vp, L.c_vp] + [L.c_i64] * 5 + [L.c_vp, L.c_int, L.c_vp])
_split_f32 = L.bind("dcc_split_operand_at4_f32", [L.c_vp, L.c_vp, L.c_vp] + [L.c_i64] * 5 + [L.c_vp, L.c_int, L.c_vp])
_gemm = L.bind("dcc_gemm_split3_ld4", [L.c_vp, L.c_vp, L.c_i64, L.c_vp, L.c_vp] + [L.c_i64] * 4 +
               [L.c_vp, L.c_vp, L.c_dbl, L.c_dbl, L.c_int, L.c_vp, L.c_vp])
_gemm_f32c = L.bind("dcc_gemm_split3_ld4_f32c", [L.c_vp, L.c_vp, L.c_i64, L.c_vp, L.c_vp] + [L.c_i64] * 4 +
                    [L.c_vp, L.c_vp, L.c_dbl, L.c_dbl, L.c_int, L.c_vp, L.c_vp])


def _gemm_fn(C):
    """The GEMM entry for C's storage type (FP64, or the FP32 accumulators of the split path)."""
    return _gemm_f32c if C.dtype == torch.float32 else _gemm

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


def four(R1, R2, R3, S0, S1, S2, S3):
    """m -> (m / (R1 R2 R3)) S0 + ((m / (R2 R3)) % R1) S1 + ((m / R3) % R2) S2 + (m % R3) S3."""
    return (R1, R2, R3, S0, S1, S2, S3)


def as4(f):
    """A three-digit map (5 values) as the equivalent four-digit map (7 values)."""
    if len(f) == 7:
        return tuple(f)
    if len(f) != 5:
        raise ValueError("a map has 5 (three-digit) or 7 (four-digit) values")
    R1, R2, S0, S1, S2 = f
    return (R1, R2, 1, S0, S1, S2, 0)


def _i64x14(f, g):
    """Two address maps as the HOST int64[14] (two four-digit maps) the C ABI takes."""
    return (ctypes.c_int64 * 14)(*[int(x) for x in as4(f) + as4(g)])


def _max_offset(f, n):
    """Upper bound of f(m) over m < n for a map with non-negative strides."""
    R1, R2, R3, S0, S1, S2, S3 = as4(f)
    if n <= 0:
        return 0
    top = (n - 1) // (R1 * R2 * R3)
    return (top * S0 + min(R1 - 1, (n - 1) // (R2 * R3)) * S1 + min(R2 - 1, (n - 1) // R3) * S2
            + min(R3 - 1, n - 1) * S3)


def _check_span(t, fm, M, fk, K, name, dtypes=(f64,)):
    """The maps stay inside t's storage (from t's first element); t is on a CUDA device, of one
    of `dtypes`."""
    if not isinstance(t, torch.Tensor) or t.dtype not in dtypes:
        raise TypeError("%s must be a %s torch.Tensor" % (name, " or ".join(str(d) for d in dtypes)))
    if not t.is_cuda:
        raise ValueError("%s must be on a CUDA device" % name)
    if any(x < 0 for x in as4(fm)[3:] + as4(fk)[3:]):
        raise ValueError("%s: negative map strides" % name)
    span = t.untyped_storage().nbytes() // t.element_size() - t.storage_offset()
    if M > 0 and K > 0 and _max_offset(fm, M) + _max_offset(fk, K) >= span:
        raise ValueError("%s: the address maps reach past the tensor's storage" % name)


def padded_k(K, kind):
    b = _KBLK[kind]
    return (K + b - 1) // b * b


class Split:
    """Two-piece K-major copy of an FP64 operand: rows M, contraction K padded to Kp.

    With pieces=[K0, K1, ...] the contraction is the concatenation of several
    operands (each piece starts on a multiple of 8 columns; the gaps and the
    tail are zero), filled one by one with fill_piece."""

    def __init__(self, M, K=None, kind=0, device="cuda", buffers=None, pieces=None, align=8):
        """align: pieces start on multiples of this many columns (8; the k-block, so that
        each piece can also be contracted on its own with gemm_range_)."""
        self.M, self.kind = int(M), int(kind)
        if pieces is None:
            pieces = [int(K)]
        offs, o = [], 0
        for k in pieces:
            offs.append(o)
            o += (int(k) + align - 1) // align * align
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
        """Columns of piece i: dst[m][off + k] = src[fm(m) + fk(k)] (zero past the piece's K).

        src may be any strided view: the maps address its storage from src's first element.
        src is FP64, or FP32 (the pieces of each value as a double)."""
        _check_span(src, fm, self.M, fk, self.pieces[i][1], "src", (f64, torch.float32))
        off, k, w = self.pieces[i]
        fn = _split_f32 if src.dtype == torch.float32 else _split
        L.check(fn(L.ptr(src), L.ptr(self.hi), L.ptr(self.lo), self.M, k, w, self.Kp, off, _i64x14(fm, fk),
                   self.kind, L.stream_ptr()))
        return self

    def fill(self, src, fm, fk):
        """dst[m][k] = src[fm(m) + fk(k)] for three-digit maps fm, fk."""
        if len(self.pieces) != 1:
            raise ValueError("a K-concatenated operand is filled with fill_piece")
        return self.fill_piece(0, src, fm, fk)


def gemm_(A, B, C, frow, fcol, alpha=1.0, beta=1.0, status=None, Kp=None):
    """C[frow(m) + fcol(n)] = alpha * A B^T + beta * C (A: Split [M,K], B: Split [N,K]).

    C is FP64, or FP32 (the sum still taken in FP64, rounded once per store).
    Kp (default: both operands' padded K) contracts only the leading Kp columns."""
    if A.kind != B.kind:
        raise ValueError("A and B must be split with the same kind")
    if Kp is None:
        if A.Kp != B.Kp:
            raise ValueError("A and B must have the same padded K (or pass Kp)")
        Kp = A.Kp
    if Kp > A.Kp or Kp > B.Kp:
        raise ValueError("Kp exceeds an operand's columns")
    _check_span(C, frow, A.M, fcol, B.M, "C", (f64, torch.float32))
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=C.device)
    L.check(_gemm_fn(C)(L.ptr(A.hi), L.ptr(A.lo), A.Kp, L.ptr(B.hi), L.ptr(B.lo), B.Kp, A.M, B.M, int(Kp), L.ptr(C),
                  _i64x14(frow, fcol), float(alpha), float(beta), A.kind, L.ptr(status), L.stream_ptr()))
    return status


def gemm_range_(A, B, C, frow, fcol, alpha, beta, status, col0, ncol):
    """gemm_ over the contraction columns [col0, col0 + ncol) of both operands (col0 and ncol
    multiples of the k-block, e.g. one piece of operands made with align = the k-block)."""
    if A.kind != B.kind or A.Kp != B.Kp:
        raise ValueError("A and B must be split with the same kind and padded K")
    blk = _KBLK[A.kind]
    if col0 % blk or ncol % blk or col0 + ncol > A.Kp:
        raise ValueError("column range must be whole k-blocks inside the operands")
    _check_span(C, frow, A.M, fcol, B.M, "C", (f64, torch.float32))
    es = A.hi.element_size()
    vp = lambda t: ctypes.c_void_p(t.data_ptr() + col0 * es)  # noqa: E731
    L.check(_gemm_fn(C)(vp(A.hi), vp(A.lo), A.Kp, vp(B.hi), vp(B.lo), B.Kp, A.M, B.M, int(ncol), L.ptr(C),
                  _i64x14(frow, fcol), float(alpha), float(beta), A.kind, L.ptr(status), L.stream_ptr()))
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


_status_cache = {}


def gemm_status(device):
    """Device status word shared by the einsum_gemm calls on `device` (zero = no timeout)."""
    key = str(device)
    if key not in _status_cache:
        _status_cache[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _status_cache[key]


def _group_digits(order, size, strides):
    """Merge consecutive indices of `order` into digits whose linear index is a
    single stride in every stride table (dict index -> stride) of `strides`.
    Returns [(indices, extent, {table: stride})] from slowest to fastest."""
    groups = []
    for c in order:
        if groups:
            g, ext, st = groups[-1]
            if all(st[t] == size[c] * tab[c] for t, tab in enumerate(strides)):
                groups[-1] = (g + [c], ext * size[c], [tab[c] for tab in strides])
                continue
        groups.append(([c], size[c], [tab[c] for tab in strides]))
    return groups


def _digit_orders(idx, size, strides, max_digits=4):
    """An order of idx whose digit grouping has at most max_digits digits (None if none)."""
    import itertools
    cand = [list(idx)] + [list(p) for p in itertools.permutations(idx)] if len(idx) <= 6 else [list(idx)]
    best = None
    for order in cand:
        g = _group_digits(order, size, strides)
        if len(g) <= max_digits:
            return g
        if best is None or len(g) < len(best):
            best = g
    return None


def _digit_orders_each(idx, size, strides, max_digits=4, prefer=None):
    """An order of idx in which every stride table, grouped on its own, has at most
    max_digits digits: one grouping per table (each addresses the same enumeration of
    idx).  prefer: a stride table whose descending order is tried first (so that
    consecutive indices are as close as possible in that tensor).  None if no order
    does."""
    import itertools
    first = sorted(idx, key=lambda c: -prefer[c]) if prefer is not None else list(idx)
    cand = [first] + [list(p) for p in itertools.permutations(idx)] if len(idx) <= 6 else [first]
    if prefer is not None:  # then orders whose fastest index is the closest one in `prefer`
        cand = [first] + sorted(cand[1:], key=lambda o: prefer[o[-1]])
    for order in cand:
        gs = [_group_digits(order, size, [tab]) for tab in strides]
        if all(len(g) <= max_digits for g in gs):
            return gs
    return None


def _map_of(groups, t):
    """Address map of a digit grouping for stride table t."""
    if not groups:
        return lin(0)
    if len(groups) == 1:
        return lin(groups[0][2][t])
    if len(groups) == 2:
        return two(groups[1][1], groups[0][2][t], groups[1][2][t])
    if len(groups) == 3:
        return three(groups[1][1], groups[2][1], groups[0][2][t], groups[1][2][t], groups[2][2][t])
    return four(groups[1][1], groups[2][1], groups[3][1], groups[0][2][t], groups[1][2][t], groups[2][2][t],
                groups[3][2][t])


_plan_cache = {}
_split_pool = {}


def _pooled_split(m, k, kind, device):
    """Split buffers reused across einsum_into calls of the same shape (one per role)."""
    key = (m, k, kind, str(device))
    if key not in _split_pool:
        _split_pool[key] = [Split(m, k, kind, device), Split(m, k, kind, device)]
    return _split_pool[key]


def einsum_into(subs, X, Y, out, alpha=1.0, beta=1.0, kind=0, status=None, max_k=None):
    """out = alpha * einsum(subs, X, Y) + beta * out as ONE split-precision GEMM
    that reads X and Y in place (no transposed copies) and accumulates straight
    into `out` (any strides) through the epilogue maps.  Every index must be
    kept by exactly one operand or contracted (no batch indices), and each of
    the row, column and contraction index sets must fold into at most four
    strided digits consistently for the tensors that carry it; otherwise the
    FP64 torch path is used.  max_k: contractions longer than this also take
    the FP64 path (FP32 accumulation over very long sums, e.g. the reductions
    of an adjoint, loses digits).  Returns out."""
    ins, o = subs.split("->")
    xs, ys = ins.split(",")
    K = [c for c in xs if c in ys]
    Mi = [c for c in xs if c not in ys]
    Ni = [c for c in ys if c not in xs]
    ok = (sorted(Mi + Ni) == sorted(o) and not any(c in o for c in K) and len(set(xs)) == len(xs)
          and len(set(ys)) == len(ys) and kind is not None and Mi and Ni and K)
    if ok and max_k is not None and int(np.prod([X.shape[xs.index(c)] for c in K])) > max_k:
        ok = False
    gM = gN = gK = None
    X0, Y0 = X, Y
    key = (subs, kind, tuple(X.shape), X.stride(), tuple(Y.shape), Y.stride(), out.stride()) if ok else None
    plan = _plan_cache.get(key)
    if plan is not None:
        gM, gN, gK, cx, cy = plan
        if cx is not None:
            X, xs = X.permute([xs.index(c) for c in cx]).contiguous(), cx
        if cy is not None:
            Y, ys = Y.permute([ys.index(c) for c in cy]).contiguous(), cy
        ok = False  # planned
    cx = cy = None
    if ok:
        size = {c: X.shape[xs.index(c)] for c in xs}
        size.update({c: Y.shape[ys.index(c)] for c in ys})
        sO = {c: out.stride(o.index(c)) for c in o}

        def strides(T, ts):
            return {c: T.stride(ts.index(c)) for c in ts}

        gM = _digit_orders(Mi, size, [strides(X, xs), sO])
        if gM is None:
            # copy X as [free indices in output order][contracted indices in Y's order]
            cx = "".join(sorted(Mi, key=o.index) + K)
            X, xs = X.permute([xs.index(c) for c in cx]).contiguous(), cx
            gM = _digit_orders(Mi, size, [strides(X, xs), sO])
        gN = _digit_orders(Ni, size, [strides(Y, ys), sO])
        if gN is None:
            cy = "".join(sorted(Ni, key=o.index) + [c for c in xs if c in K])
            Y, ys = Y.permute([ys.index(c) for c in cy]).contiguous(), cy
            gN = _digit_orders(Ni, size, [strides(Y, ys), sO])
        gK = _digit_orders(K, size, [strides(X, xs), strides(Y, ys)])
        if gK is None:
            cy = "".join([c for c in ys if c not in K] + [c for c in xs if c in K])
            Y, ys = Y.permute([ys.index(c) for c in cy]).contiguous(), cy
            gN = _digit_orders(Ni, size, [strides(Y, ys), sO])
            gK = _digit_orders(K, size, [strides(X, xs), strides(Y, ys)])
        if gM is not None and gN is not None and gK is not None:
            _plan_cache[key] = (gM, gN, gK, cx, cy)
    if gM is None or gN is None or gK is None:
        res = torch.einsum(subs, X0, Y0)
        if beta == 0.0:
            out.copy_(res).mul_(alpha) if alpha != 1.0 else out.copy_(res)
        else:
            if beta != 1.0:
                out.mul_(beta)
            out.add_(res, alpha=alpha)
        return out
    m = int(np.prod([g[1] for g in gM]))
    n = int(np.prod([g[1] for g in gN]))
    k = int(np.prod([g[1] for g in gK]))
    a = _pooled_split(m, k, kind, X.device)[0].fill(X, _map_of(gM, 0), _map_of(gK, 0))
    b = _pooled_split(n, k, kind, X.device)[1].fill(Y, _map_of(gN, 0), _map_of(gK, 1))
    st = status if status is not None else gemm_status(X.device)
    gemm_(a, b, out, _map_of(gM, 1), _map_of(gN, 1), alpha, beta, st)
    return out


# ----------------------------------------------------------------------------
# Grouped splits and GEMMs: many einsums in one launch each
# ----------------------------------------------------------------------------

_split_grouped_table = L.bind("dcc_split_grouped_table", [L.c_vp, L.c_int, L.c_vp, L.c_size, L.c_vp])
_split_grouped = L.bind("dcc_split_grouped", [L.c_vp, L.c_int, L.c_i64, L.c_vp, L.c_int, L.c_vp])
_gemm_grouped_table = L.bind("dcc_gemm_grouped_table", [L.c_vp, L.c_vp, L.c_int, L.c_int, L.c_vp, L.c_size,
                                                         L.c_vp])
_gemm_grouped = L.bind("dcc_gemm_grouped", [L.c_vp, L.c_int, L.c_i64, L.c_int, L.c_int, L.c_vp, L.c_vp])
L.bind("dcc_split_grouped_table_bytes", [L.c_int], L.c_size)
L.bind("dcc_gemm_grouped_table_bytes", [L.c_int], L.c_size)
SPLIT_SPEC, GEMM_SPEC = 22, 25


class GroupedSplit:
    """Operand splits of many einsums in one launch (dcc_split_grouped).

    spec: int64 [n, 22] rows (hi, lo, M, K, kw, ld, k0, row map(7), k map(7),
    source is float32); run(srcs) fills every operand from its source address."""

    def __init__(self, spec, kind, device):
        spec = np.ascontiguousarray(spec, dtype=np.int64)
        if spec.ndim != 2 or spec.shape[1] != SPLIT_SPEC:
            raise ValueError("spec must be int64 [n, %d]" % SPLIT_SPEC)
        self.n, self.kind = spec.shape[0], int(kind)
        nbytes = int(L.lib().dcc_split_grouped_table_bytes(self.n))
        self.table = torch.empty(nbytes, dtype=torch.uint8, device=device)
        total = ctypes.c_int64(0)
        L.check(_split_grouped_table(spec.ctypes.data_as(L.c_vp), self.n, L.ptr(self.table), nbytes,
                                     ctypes.byref(total)))
        self.total = total.value
        self._srcs = (L.c_vp * self.n)()

    def run(self, srcs):
        """srcs: n device addresses (ints), operand p read from srcs[p]."""
        if len(srcs) != self.n:
            raise ValueError("need %d sources" % self.n)
        for i, p in enumerate(srcs):
            self._srcs[i] = int(p)
        L.check(_split_grouped(L.ptr(self.table), self.n, self.total, self._srcs, self.kind, L.stream_ptr()))


class GroupedGemm:
    """Split-precision GEMMs of many einsums in one persistent launch
    (dcc_gemm_grouped): C_p[row(m) + col(n)] += alpha_p (A_p B_p^T)[m][n], added by
    reductions in L2 so several problems may share an output.

    spec: int64 [n, 25] rows (A_hi, A_lo, lda, B_hi, B_lo, ldb, M, N, Kp, C,
    C is float32, row map(7), col map(7)); alpha: float64 [n]."""

    def __init__(self, spec, alpha, kind, device):
        spec = np.ascontiguousarray(spec, dtype=np.int64)
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        if spec.ndim != 2 or spec.shape[1] != GEMM_SPEC or alpha.shape != (spec.shape[0],):
            raise ValueError("spec must be int64 [n, %d] with n alphas" % GEMM_SPEC)
        self.n, self.kind = spec.shape[0], int(kind)
        self.out_f32 = int(spec[0, 10])
        nbytes = int(L.lib().dcc_gemm_grouped_table_bytes(self.n))
        self.table = torch.empty(nbytes, dtype=torch.uint8, device=device)
        total = ctypes.c_int64(0)
        L.check(_gemm_grouped_table(spec.ctypes.data_as(L.c_vp), alpha.ctypes.data_as(L.c_vp), self.n, self.kind,
                                    L.ptr(self.table), nbytes, ctypes.byref(total)))
        self.total = total.value

    def run(self, status):
        L.check(_gemm_grouped(L.ptr(self.table), self.n, self.total, self.kind, self.out_f32, L.ptr(status),
                              L.stream_ptr()))


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

    def key(self):
        return ("wvvvv_t3", self.n, self.nv, self.kind)

    def tune(self, scratch, W, t3, F=None):
        """Pick the GEMM tile and pipeline shape (tile columns, k-block width, ring depth, raster
        group) of these launches with the autotuner (dcc.autotune: every candidate timed on this
        problem); the candidates accumulate into `scratch` (r3-shaped, contents discarded).
        Later calls apply the choice."""
        from . import autotune
        return autotune.tune(self.key(), lambda: self(scratch, W, t3, F=F))

    def __call__(self, r3, W, t3, alpha=1.0, F=None):
        from . import autotune
        L.as_tensor(r3, f64, "r3")
        L.as_tensor(t3, f64, "t3")
        with autotune.applied(self.key()):
            return self._run(r3, W, t3, alpha, F)

    def _run(self, r3, W, t3, alpha, F):
        nv = self.nv
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
