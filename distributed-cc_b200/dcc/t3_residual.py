"""Batched T3 residual on the GPU (distr_cc/rccsdt.py:368-732, 947-971).

The reference walks the canonical blocks and issues one `_einsum` per block
and einsum string.  Here the strings become a few large contractions over
all blocks.  With U the unpacked t3 of every ordered (i,j,k) (U is invariant
under simultaneous permutations of (i,j,k) and (a,b,c)), every W_vvvo.t2,
W_vooo.t2 and OO batch string (distr_cc/rccsdt.py:385-396, 435-732) is part
of one full symmetrization

    r3[ijk][abc] = sum_{p in S3} (S - Y)[p(ijk)][p(abc)]

of two tensors over every ordered (i,j,k):

    Y  = sum_l W_vooo[a,l,i,j] t2[l,k,b,c]                       (FP64, K = nocc)
    S  = X + T1 + T2 + T5/2 + (W_oooo.U - F_oo.U)/2
    X  = sum_d W_vvvo[a,b,d,j] t2[i,k,d,c]
    T1 = - sum_{l,d} W_ovov[l,b,i,d] U[jkl][d,c,a]
    T2 =   sum_{l,d} G2[l,a,i,d] U[jkl][d,c,b],   G2 = -(W_ovov[l,a,i,d] + W_ovvo[l,a,d,i]) / 2
    T5 =   sum_{l,d} W_ovvo[l,a,d,i] U[jkl][b,c,d]
    W_oooo.U = sum_{l,m} W_oooo[l,m,i,j] U[lmk][abc],   F_oo.U = sum_l F_oo[l,i] U[ljk][abc]

The reference's two remaining W_ovov strings are T1 and T2 composed with
(i,k,j; a,c,b) and drop out of the S3 sum; T5, F_oo.U and (for a W_oooo with
the pair symmetry W[l,m,i,j] = W[m,l,j,i]) W_oooo.U are invariant under that
permutation, hence the halves.  A W_oooo without the pair symmetry keeps its
antisymmetric part on the reference's own permutation set
{identity, (i,k,j; a,c,b), (j,k,i; b,c,a)}.

In mixed precision S (FP32, the accumulation type of the split products) is
built by five split-precision tcgen05 GEMMs written straight into S's
[i][j][k][a][b][c] layout (-Y first, which initializes S; X;
T2 and T5/2 as one GEMM over the concatenated contraction index; T1 reusing
T2's U operand; the K = nocc^2 W_oooo / F_oo part over a K-major split of U),
and one gather kernel applies the symmetrization to S (the FP64 path builds S
the same way from DGEMMs, one occupied slice at a time).  W_vvvv.t3 (three strings, the dominant cost) are
three split-precision GEMMs that accumulate straight into r3; the three
F_vv.t3 strings ride in them as extra terms of the W operand
(contract.WvvvvT3).  The FP64 path runs F_vv.t3 as batched DGEMMs.

precision = "fp64" runs every contraction in FP64 (cuBLAS DGEMM through
torch): the plain FP64 GPU path.  "bf16x3" / "tf32x3" run the large
contractions as split products with FP32 accumulation; the denominators,
update, norms and all sums stay FP64.
"""
from __future__ import annotations

import ctypes

import torch

from . import _c_rccsdt, contract
from . import _lib as L

f64 = torch.float64

_gather = L.bind("dcc_t3_s3_gather", [L.c_vp, L.c_vp, L.c_i64, L.c_i64, L.c_dbl, L.c_vp, L.c_dbl, L.c_vp, L.c_vp,
                                      L.c_dbl, L.c_vp, L.c_vp])


def _strides(s):
    return (ctypes.c_int64 * 6)(*[int(x) for x in s])


def s3_gather_(r3, ijk, nvir, beta, u0, scale0, strides0, u1=None, scale1=0.0, strides1=None):
    """r3 = beta*r3 + sum_s scale_s * sum over the six simultaneous permutations of U_s."""
    L.check(_gather(L.ptr(r3), L.ptr(ijk), r3.shape[0], nvir, float(beta), L.ptr(u0), float(scale0),
                    _strides(strides0), L.ptr(u1) if u1 is not None else L.c_vp(None), float(scale1),
                    _strides(strides1) if strides1 is not None else None, L.stream_ptr()))
    return r3


_pgather = L.bind("dcc_t3_perm_gather", [L.c_vp, L.c_vp, L.c_i64, L.c_i64, L.c_dbl, L.c_int, L.c_vp, L.c_vp,
                                         L.c_vp, L.c_vp, L.c_vp])

# permutation subsets of the gather (bit p: simultaneous permutation p of (i,j,k) and (a,b,c),
# p in the order (x,y,z), (x,z,y), (y,x,z), (y,z,x), (z,x,y), (z,y,x))
ALL_S3 = 63
OO_SET = (1 << 0) | (1 << 2) | (1 << 4)  # identity, (j,i,k;b,a,c), (k,i,j;c,a,b)
OOOO_SET = (1 << 0) | (1 << 1) | (1 << 3)  # identity, (i,k,j;a,c,b), (j,k,i;b,c,a)


_pgather_tma = L.bind("dcc_t3_perm_gather_tma", [L.c_vp, L.c_vp, L.c_i64, L.c_i64, L.c_i64, L.c_dbl, L.c_int, L.c_vp,
                                                 L.c_vp, L.c_vp, L.c_vp, L.c_vp, L.c_vp])
_status_cache = {}


def _default_status(device):
    key = str(device)
    if key not in _status_cache:
        _status_cache[key] = torch.zeros(1, dtype=torch.int32, device=device)
    return _status_cache[key]


def perm_gather_(r3, ijk, nvir, beta, sources, nocc=None, status=None):
    """r3 = beta*r3 + sum over sources (tensor, scale, strides6, mask) of the masked permutation sums.

    With nocc given the TMA-pipelined kernel runs (it reports bounded-wait
    timeouts in `status`, a device int32); without, the cp.async kernel."""
    n = len(sources)
    bases = (ctypes.c_void_p * n)(*[t.data_ptr() for t, _, _, _ in sources])
    scales = (ctypes.c_double * n)(*[float(sc) for _, sc, _, _ in sources])
    strides = (ctypes.c_int64 * (6 * n))(*[int(x) for _, _, st, _ in sources for x in st])
    masks = (ctypes.c_int * n)(*[int(m) for _, _, _, m in sources])
    if nocc is None:
        L.check(_pgather(L.ptr(r3), L.ptr(ijk), r3.shape[0], nvir, float(beta), n, bases, scales, strides, masks,
                         L.stream_ptr()))
    else:
        if status is None:
            status = _default_status(r3.device)
        L.check(_pgather_tma(L.ptr(r3), L.ptr(ijk), r3.shape[0], int(nocc), nvir, float(beta), n, bases, scales,
                             strides, masks, L.ptr(status), L.stream_ptr()))
    return r3


_gather_f32 = L.bind("dcc_t3_s3_gather_f32", [L.c_vp, L.c_vp, L.c_i64, L.c_i64, L.c_i64, L.c_dbl, L.c_vp, L.c_dbl,
                                              L.c_vp])


def s3_gather_f32_(r3, ijk, nvir, beta, S, scale, nocc):
    """r3 = beta*r3 + scale * sum over the six simultaneous permutations of an FP32 full-layout S."""
    if S.dtype != torch.float32 or r3.dtype != f64:
        raise TypeError("S must be float32 and r3 float64")
    if S.numel() != nocc ** 3 * nvir ** 3 or not S.is_contiguous():
        raise ValueError("S must be a contiguous [nocc^3][nvir^3] tensor")
    L.check(_gather_f32(L.ptr(r3), L.ptr(ijk), r3.shape[0], int(nocc), int(nvir), float(beta), L.ptr(S),
                        float(scale), L.stream_ptr()))
    return r3


_unpack_all = L.bind("dcc_t3_unpack_all", [L.c_vp, L.c_vp, L.c_i64, L.c_i64, L.c_vp])
_unpack_all_f32 = L.bind("dcc_t3_unpack_all_f32", [L.c_vp, L.c_vp, L.c_i64, L.c_i64, L.c_vp])

# Largest nvir with FP32 kernels for the full-layout T3 copies (the strip kernels)
F32_MAX_NVIR = 104


def unpack_all_(t3, U, nocc, nvir):
    """U[(x*nocc+y)*nocc+z] = T3[x,y,z] for every ordered triple (take_t3 of all orderings);
    U FP64, or FP32 (each value rounded once; nvir <= F32_MAX_NVIR)."""
    fn = _unpack_all_f32 if U.dtype == torch.float32 else _unpack_all
    L.check(fn(L.ptr(t3), L.ptr(U), nocc, nvir, L.stream_ptr()))
    return U


def full_dtype(precision, nvir):
    """Storage type of the full-layout T3 copies U and X: FP32 for the split precisions (their
    bf16 / tf32 pieces keep 16-22 of FP32's 24 significand bits, so the split of an FP32 copy
    equals that of the FP64 value to within the pieces' own rounding) where the FP32 kernels
    exist, FP64 otherwise.  Half the bytes of the unpack, the X pass and the operand splits."""
    return torch.float32 if precision != "fp64" and nvir <= F32_MAX_NVIR else f64


def full_strides(no, nv):
    """Strides (x,y,z,a,b,c) of a full ordered-triple tensor laid out [x][y][z][a][b][c]."""
    n3 = nv ** 3
    return (no * no * n3, no * n3, n3, nv * nv, nv, 1)


def s_plan(no, nv):
    """Operand and output maps of the split-precision GEMMs that build S.

    Each entry: A pieces and B pieces as (name, row map, k map), the output
    (row map, column map) into S = [i][j][k][a][b][c], alpha and beta.  The
    T1 GEMM takes the first piece of the T2/T5 GEMM's B operand (the same
    U layout) and contracts only its leading columns."""
    c = contract
    n3v = nv ** 3
    return {
        # X: rows (j,a,b) of W_vvvo[a,b,d,j], cols (i,k,c) of t2[i,k,d,c], K = d
        "x": dict(a=[("W_vvvo", c.two(nv * nv, 1, nv * no), c.lin(no))],
                  b=[("t2", c.two(nv, nv * nv, 1), c.lin(nv))],
                  out=(c.three(nv, nv, no * n3v, nv * nv, nv), c.three(no, nv, no * no * n3v, n3v, 1)),
                  alpha=1.0, beta=0.0),
        # T2 + T5/2: rows (i,a), cols (jk,b,c), K = (l,d) of G2, then (l,d) of W_ovvo/2
        "oo": dict(a=[("G2", c.lin(no * nv), c.lin(1)),
                      ("Wvo_half", c.two(nv, 1, nv * no), c.two(nv, nv * nv * no, no))],
                   b=[("U", c.three(nv, nv, no * n3v, 1, nv), c.two(nv, n3v, nv * nv)),     # U[jkl][d,c,b]
                      ("U", c.three(nv, nv, no * n3v, nv * nv, nv), c.two(nv, n3v, 1))],   # U[jkl][b,c,d]
                   out=(c.two(nv, no * no * n3v, nv * nv), c.three(nv, nv, n3v, nv, 1)),
                   alpha=1.0, beta=1.0),
        # T1: rows (i,b) of W_ovov[l,b,i,d], cols (jk,a,c) of U[jkl][d,c,a] (= piece 0 of oo.b)
        "t1": dict(a=[("W_ovov", c.two(nv, nv, no * nv), c.two(nv, nv * no * nv, 1))],
                   out=(c.two(nv, no * no * n3v, nv), c.three(nv, nv, n3v, nv * nv, 1)),
                   alpha=-1.0, beta=1.0),
    }


def woooo_k_pieces(no, nv, limit=(1 << 31) - 1):
    """Contraction pieces of the K-major split of U for the W_oooo / F_oo GEMM: K = nocc^2
    cut so that a piece's offsets (k * nocc nvir^3) stay below `limit`, every piece but the
    last a multiple of 8 columns."""
    stride, K = no * nv ** 3, no * no
    if (K - 1) * stride < limit:
        return [K]
    step = (limit // stride) // 8 * 8
    if step < 8:
        raise ValueError("nocc * nvir^3 = %d is too large for 31-bit split offsets" % stride)
    return [min(step, K - k0) for k0 in range(0, K, step)]


def woooo_foo_matrix(W_oooo, F_oo, sym_tol=1e-14, assume_symmetric=False):
    """(A, W_anti): A[(i,j)][(l,m)] = (Ws[l,m,i,j] - F_oo[l,i] delta_mj) / 2 with Ws the
    pair-symmetric part of W_oooo; W_anti = the antisymmetric part, or None when it is
    below sym_tol relative to max|W_oooo| (one device-to-host read of two scalars) or
    when assume_symmetric (no host read: usable inside CUDA-graph capture)."""
    no = W_oooo.shape[0]
    Wt = W_oooo.permute(1, 0, 3, 2)
    Wa = 0.5 * (W_oooo - Wt)
    if assume_symmetric:
        anti = False
    else:
        big = torch.stack([Wa.abs().max(), W_oooo.abs().max()]).cpu()
        anti = float(big[0]) > sym_tol * max(float(big[1]), 1e-300)
    Ws = W_oooo - Wa if anti else W_oooo
    eye = torch.eye(no, dtype=W_oooo.dtype, device=W_oooo.device)
    A = 0.5 * Ws.permute(2, 3, 0, 1) - 0.5 * torch.einsum("li,mj->ijlm", F_oo, eye)
    return A.reshape(no * no, no * no).contiguous(), (Wa.contiguous() if anti else None)


class T3Residual:
    """compute_r3_tri for all canonical blocks of one rank."""

    def __init__(self, nocc, nvir, precision="fp64", device="cuda", with_oo=True, woooo_pair_symmetric=False,
                 woooo_piece_limit=(1 << 31) - 1):
        self.no, self.nv, self.precision = int(nocc), int(nvir), precision
        # True: W_oooo has the pair symmetry of RHF (its antisymmetric part is not checked
        # for, so compute() reads nothing back to the host and can be captured in a graph)
        self.woooo_pair_symmetric = woooo_pair_symmetric
        no, nv = self.no, self.nv
        self.n3 = no * (no + 1) * (no + 2) // 6
        self.dev = device
        self.with_oo = with_oo
        full = (no ** 3, nv, nv, nv)
        self.udtype = full_dtype(precision, nvir)
        # [i][j][k][a][b][c]; in the split precisions the accumulator of the S GEMMs is FP32 like
        # their products' accumulation (half the bytes of the five epilogue read-modify-writes and
        # of the gather), FP64 on the FP64 path
        self.S = torch.empty(full, dtype=self.udtype, device=device)
        self.U = torch.empty(full, dtype=self.udtype, device=device) if with_oo else None
        self.Ganti = None
        self.gstatus = torch.zeros(1, dtype=torch.int32, device=device)  # gather pipeline timeouts
        self._sargs = {}  # the S GEMMs' last arguments, by name (tune)
        if precision != "fp64":
            k = contract.KIND[precision]
            self.kind = k
            self.plan = s_plan(no, nv)
            self.xa = contract.Split(no * nv * nv, nv, k, device)
            self.xb = contract.Split(no * no * nv, nv, k, device)
            self.wvvvv = contract.WvvvvT3(self.n3, nv, precision, device)
            self.ya = contract.Split(no * no * nv, no, k, device)
            self.yb = contract.Split(no * nv * nv, no, k, device)
            self.status = torch.zeros(1, dtype=torch.int32, device=device)
            if with_oo:
                K = no * nv
                self.ooa = contract.Split(no * nv, kind=k, device=device, pieces=[K, K])
                self.oob = contract.Split(no * no * nv * nv, kind=k, device=device, pieces=[K, K])
                self.t1a = contract.Split(no * nv, K, k, device)
                # W_oooo / F_oo . U: rows (i,j), columns (k,a,b,c), K = (l,m).  The split kernel
                # addresses a piece's contraction with 31-bit offsets and U's (l,m) stride is
                # nocc nvir^3, so K is cut into pieces of whole multiples of 8 below 2^31 / stride
                # (one piece up to about nocc=12 / nvir=90; two at nocc=15 / nvir=93)
                self.woo_pieces = woooo_k_pieces(no, nv, woooo_piece_limit)
                if len(self.woo_pieces) == 1:
                    self.wooa = contract.Split(no * no, no * no, k, device)
                    self.woob = contract.Split(no * nv ** 3, no * no, k, device)
                else:
                    self.wooa = contract.Split(no * no, kind=k, device=device, pieces=self.woo_pieces)
                    self.woob = contract.Split(no * nv ** 3, kind=k, device=device, pieces=self.woo_pieces)

    # ------------------------------------------------------------ pieces
    def _gemm(self, name, A, B, C, frow, fcol, alpha, beta, Kp=None):
        """One of the S GEMMs under the tile and raster configuration tuned for it (tune()); its
        arguments are kept so that tune() can time it alone."""
        from . import autotune
        self._sargs[name] = (A, B, C, frow, fcol, alpha, beta, Kp)
        with autotune.applied(self._gkey(name)):
            contract.gemm_(A, B, C, frow, fcol, alpha, beta, self.status, Kp=Kp)

    def _gkey(self, name):
        return ("s_gemm", name, self.no, self.nv, self.kind)

    def _y_into_s(self, d):
        """S = -Y in S's [i][j][k][a][b][c] layout (split path): rows (i,j,a), columns (k,b,c).  Y
        then rides in S's permutation sum, and the gather reads one source instead of two."""
        no, nv = self.no, self.nv
        c = contract
        self.ya.fill(d.W_vooo, c.three(no, nv, no, 1, no ** 3), c.lin(no * no))
        self.yb.fill(d.t2, c.lin(1), c.lin(no * nv * nv))
        self._gemm("y", self.ya, self.yb, self.S, c.three(no, nv, no * no * nv ** 3, no * nv ** 3, nv * nv),
                   c.two(nv * nv, nv ** 3, 1), -1.0, 0.0)

    def unpack_(self, t3):
        """U = t3 unpacked to every ordered (i,j,k) (the operand of the OO terms)."""
        return unpack_all_(t3, self.U, self.no, self.nv)

    def s_(self, d, t3, inputs_ready=None, unpacked=False):
        """S (see the module docstring); U = unpacked t3 when the OO terms are on (already
        there when `unpacked`).  The unpack reads only t3, so it runs before the wait on
        `inputs_ready` (an optional CUDA event that marks the arrival of d's tensors)."""
        no, nv = self.no, self.nv
        S = self.S
        if self.with_oo and not unpacked:
            self.unpack_(t3)
        if inputs_ready is not None:
            torch.cuda.current_stream().wait_event(inputs_ready)
        if self.precision == "fp64":
            self._s_fp64(d)
        else:
            self._s_split(d)
        if self.with_oo:
            A, Wa = woooo_foo_matrix(d.W_oooo, d.F_oo, assume_symmetric=self.woooo_pair_symmetric)
            if self.precision == "fp64":
                S.view(no * no, -1).addmm_(A, self.U.view(no * no, -1))
            else:
                # S[(i,j)][(k,abc)] += A[(i,j)][(l,m)] U[(l,m)][(k,abc)] as a split GEMM: the K-major split
                # of U (no nv^3 rows of no^2) costs one pass over U, the FP64 DGEMM took twice as long
                n = no * nv ** 3
                A = A.contiguous()
                if len(self.woo_pieces) == 1:
                    self.wooa.fill(A, contract.lin(no * no), contract.lin(1))
                    self.woob.fill(self.U, contract.lin(1), contract.lin(n))
                else:
                    k0 = 0
                    Uf = self.U.view(no * no, n)
                    for i, kk in enumerate(self.woo_pieces):
                        self.wooa.fill_piece(i, A[:, k0:k0 + kk], contract.lin(no * no), contract.lin(1))
                        self.woob.fill_piece(i, Uf[k0:k0 + kk], contract.lin(1), contract.lin(n))
                        k0 += kk
                # rows (k,abc) of U's split, columns (i,j): the nocc^2 (i,j) fill one 256-column tile
                # instead of leaving the lane quarters of a second 128-row tile idle (nocc^2 = 225 rows
                # at nocc=15, 36 at nocc=6), and each reduction of a warp covers 32 consecutive (k,abc)
                self._gemm("woooo", self.woob, self.wooa, S, contract.lin(1), contract.lin(n), 1.0, 1.0)
            if Wa is not None:
                if self.Ganti is None:
                    self.Ganti = torch.empty(self.S.shape, dtype=f64, device=self.S.device)
                Uf = self.U.view(no * no, -1)
                if Uf.dtype == f64:
                    torch.matmul(Wa.reshape(no * no, no * no).t(), Uf, out=self.Ganti.view(no * no, -1))
                else:  # an FP32 U (split precisions): the product in FP32, kept in FP64
                    self.Ganti.view(no * no, -1).copy_(torch.matmul(Wa.reshape(no * no, no * no).t().float(), Uf))
            else:
                self.Ganti = None
        return S

    def _s_split(self, d):
        c, pl, st = contract, self.plan, self.status
        no, nv = self.no, self.nv
        S = self.S
        x = pl["x"]
        self._y_into_s(d)  # writes S first
        self.xa.fill(d.W_vvvo, *x["a"][0][1:])
        self.xb.fill(d.t2, *x["b"][0][1:])
        self._gemm("x", self.xa, self.xb, S, *x["out"], x["alpha"], 1.0)
        if not self.with_oo:
            return
        src = {"G2": (-0.5 * (d.W_ovov + d.W_ovvo.permute(0, 1, 3, 2))).permute(2, 1, 0, 3).contiguous(),
               "Wvo_half": 0.5 * d.W_ovvo, "W_ovov": d.W_ovov, "U": self.U}
        oo, t1 = pl["oo"], pl["t1"]
        for i, (name, fm, fk) in enumerate(oo["a"]):
            self.ooa.fill_piece(i, src[name], fm, fk)
        for i, (name, fm, fk) in enumerate(oo["b"]):
            self.oob.fill_piece(i, src[name], fm, fk)
        name, fm, fk = t1["a"][0]
        self.t1a.fill(src[name], fm, fk)
        self._gemm("oo", self.ooa, self.oob, S, *oo["out"], oo["alpha"], oo["beta"])
        self._gemm("t1", self.t1a, self.oob, S, *t1["out"], t1["alpha"], t1["beta"], Kp=self.t1a.Kp)

    def _s_fp64(self, d):
        """S in FP64 (cuBLAS DGEMM through torch), one occupied slice at a time so the
        temporaries stay 1/nocc of S: S = X - Y (+ the OO terms when with_oo)."""
        no, nv = self.no, self.nv
        Sv = self.S.view(no, no, no, nv, nv, nv)
        # X[i,j,k,a,b,c] = sum_d W_vvvo[a,b,d,j] t2[i,k,d,c]: per j, [(a,b), d] . [d, (i,k,c)]
        T2m = d.t2.permute(2, 0, 1, 3).reshape(nv, no * no * nv)
        for j in range(no):
            Xj = torch.matmul(d.W_vvvo[..., j].reshape(nv * nv, nv), T2m)
            Sv[:, j].copy_(Xj.view(nv, nv, no, no, nv).permute(2, 3, 0, 1, 4))
        # - Y[i,j,k,a,b,c] = - sum_l W_vooo[a,l,i,j] t2[l,k,b,c]: per i, [(j,a), l] . [l, (k,b,c)]
        T2l = d.t2.reshape(no, no * nv * nv)
        for i in range(no):
            Yi = torch.matmul(d.W_vooo[:, :, i, :].permute(2, 0, 1).reshape(no * nv, no), T2l)
            Sv[i].sub_(Yi.view(no, nv, no, nv, nv).permute(0, 2, 1, 3, 4))
        if not self.with_oo:
            return
        Uv = self.U.view(no, no, no, nv, nv, nv)
        e = torch.einsum
        G2 = -0.5 * (d.W_ovov + d.W_ovvo.permute(0, 1, 3, 2))
        Wh = 0.5 * d.W_ovvo
        for j in range(no):
            Uj = Uv[j]  # [k][l][...]
            Sj = Sv[:, j]
            Sj.sub_(e('lbid,kldca->ikabc', d.W_ovov, Uj))
            Sj.add_(e('laid,kldcb->ikabc', G2, Uj))
            Sj.add_(e('ladi,klbcd->ikabc', Wh, Uj))

    def fvv_(self, r3, d, t3):
        """F_vv.t3 (distr_cc/rccsdt.py:400-402), FP64 in both precisions (bandwidth-bound)."""
        n, nv = t3.shape[0], self.nv
        F = d.F_vv
        r3.view(n, nv, nv * nv).add_(torch.matmul(F, t3.view(n, nv, nv * nv)))
        r3.view(n * nv, nv, nv).add_(torch.matmul(F, t3.view(n * nv, nv, nv)))
        r3.view(n * nv * nv, nv).add_(torch.matmul(t3.view(n * nv * nv, nv), F.t()))
        return r3

    def wvvvv_(self, r3, d, t3):
        """W_vvvv.t3 (distr_cc/rccsdt.py:421-427); in split precision F_vv.t3 rides in the same GEMMs."""
        if self.precision == "fp64":
            return contract.wvvvv_t3_fp64_(r3, d.W_vvvv, t3)
        return self.wvvvv(r3, d.W_vvvv, t3, F=d.F_vv)

    def tune(self, d, t3):
        """Autotune the split precisions' GEMMs (the FP64 path has nothing to tune): the tile width,
        pipeline shape and raster group of the W_vvvv.t3 GEMMs, then the tile width and raster
        group of each S GEMM, each timed alone on this problem (their operands from one pass of
        s_ over d and t3; S is rebuilt by the next compute).  Returns the W_vvvv choice
        (k-block bytes, stages, group, tile columns); s_tuning() lists the others."""
        if self.precision == "fp64":
            return None
        from . import autotune
        best = self.wvvvv.tune(torch.empty_like(t3), d.W_vvvv, t3, F=d.F_vv)
        self.s_(d, t3)
        for name, (A, B, C, frow, fcol, alpha, beta, Kp) in self._sargs.items():
            old = autotune.get_config()
            autotune.tune(self._gkey(name),
                          lambda: contract.gemm_(A, B, C, frow, fcol, alpha, beta, self.status, Kp=Kp),
                          cands=autotune.tile_candidates())
            autotune.set_config(*old)
        return best

    def s_tuning(self):
        """{S GEMM: (chosen configuration, {candidate: ms})} after tune()."""
        from . import autotune
        return {name: (autotune.chosen(self._gkey(name)), autotune.timings(self._gkey(name)))
                for name in self._sargs if autotune.timings(self._gkey(name)) is not None}

    def compute(self, d, t3, r3=None, wvvvv_ready=None, inputs_ready=None, unpacked=False):
        """r3 = compute_r3_tri for canonical t3 (the OO batch terms included when with_oo).

        wvvvv_ready: optional CUDA event the W_vvvv.t3 part waits for, so a caller can
        stream W_vvvv to the device while the other terms run; or a callable, called once
        every other term is enqueued, that brings d.W_vvvv in and returns that event (a
        caller holding W_vvvv in pageable host memory copies it while the device works on
        the rest).  inputs_ready: optional CUDA
        event for d's other tensors, waited for after the unpack of t3 (which needs none of
        them), so their upload overlaps it.  unpacked: U holds t3 unpacked already (unpack_)."""
        if r3 is None:
            r3 = torch.empty_like(t3)
        no, nv = self.no, self.nv
        S = self.s_(d, t3, inputs_ready, unpacked=unpacked)
        if S.dtype == torch.float32:  # S holds -Y already
            s3_gather_f32_(r3, d.ijk, nv, 0.0, S, 1.0, no)
        else:
            perm_gather_(r3, d.ijk, nv, 0.0, [(S, 1.0, full_strides(no, nv), ALL_S3)], nocc=no, status=self.gstatus)
        if self.Ganti is not None:
            perm_gather_(r3, d.ijk, nv, 1.0, [(self.Ganti, 1.0, full_strides(no, nv), OOOO_SET)], nocc=no,
                         status=self.gstatus)
        if callable(wvvvv_ready):
            wvvvv_ready = wvvvv_ready()
        if wvvvv_ready is not None:
            torch.cuda.current_stream().wait_event(wvvvv_ready)
        if self.precision == "fp64":
            self.fvv_(r3, d, t3)
        self.wvvvv_(r3, d, t3)
        return r3

    def status_ok(self):
        if int(self.gstatus.item()) != 0:
            return False
        if self.precision == "fp64":
            return True
        return int(self.status.item()) == 0 and int(self.wvvvv.status.item()) == 0


def update_t3_(t3, r3, d, nvir_active=None, norms=None, workspace=None, write_r3=True):
    """P3_full symmetrize (-1/6, 1), divide by D, t3 += r3, squared norms
    (distr_cc/rccsdt.py:947-971).  Returns the device norms [|r3|^2, |r3_active|^2]."""
    nv = r3.shape[1]
    _c_rccsdt.t3_spin_summation_inplace_(r3, r3.shape[0], nv, "P3_full", -1.0 / 6.0, 1.0)
    return _c_rccsdt.t3_divide_update_(t3, r3, d.eia, d.ijk, nvir_active=nvir_active, write_r3=write_r3,
                                       norms=norms, workspace=workspace)
