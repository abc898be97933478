"""Batched T3 residual on the GPU (distr_cc/rccsdt.py:368-433, 947-971).

The reference walks the canonical blocks and issues one `_einsum` per block
and einsum string.  Here each group of strings becomes one large contraction
over all blocks:

* The twelve W_vvvo.t2 / W_vooo.t2 strings (distr_cc/rccsdt.py:385-396) are
  the simultaneous S3 symmetrization of two contractions taken over every
  ordered (i,j,k):
      X[ijk][abc] = sum_d W_vvvo[a,b,d,j] t2[i,k,d,c]
      Y[ijk][abc] = sum_l W_vooo[a,l,i,j] t2[l,k,b,c]
      r3[ijk][abc] = sum_sigma (X - Y)[sigma(ijk)][sigma(abc)]
  so they are two GEMMs and one gather (dcc_t3_perm_gather).
* The OO batch terms (distr_cc/rccsdt.py:435-732: masked W_ovov / W_ovvo
  einsums per batch block and the F_oo / W_oooo prefactor matrices) are the
  partial symmetrization over {identity, (jik;bac), (kij;cab)} of one tensor
  Z over every ordered (i,j,k), built by five GEMMs over the unpacked t3
  (K = nocc*nvir) and two small FP64 GEMMs; the same gather adds it.
* F_vv.t3 (three strings) are three batched GEMMs.
* W_vvvv.t3 (three strings, the dominant cost) are three GEMMs over all
  blocks; in mixed precision they run on the tcgen05 split-BF16x3 kernel and
  accumulate straight into r3.

precision = "fp64" runs every contraction in FP64 (cuBLAS DGEMM through
torch): the plain FP64 GPU path.  "bf16x3" / "tf32x3" run the large
contractions (X and W_vvvv.t3) as split products with FP32 accumulation;
the denominators, update, norms and all sums stay FP64.
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


def perm_gather_(r3, ijk, nvir, beta, sources):
    """r3 = beta*r3 + sum over sources (tensor, scale, strides6, mask) of the masked permutation sums."""
    n = len(sources)
    bases = (ctypes.c_void_p * n)(*[t.data_ptr() for t, _, _, _ in sources])
    scales = (ctypes.c_double * n)(*[float(sc) for _, sc, _, _ in sources])
    strides = (ctypes.c_int64 * (6 * n))(*[int(x) for _, _, st, _ in sources for x in st])
    masks = (ctypes.c_int * n)(*[int(m) for _, _, _, m in sources])
    L.check(_pgather(L.ptr(r3), L.ptr(ijk), r3.shape[0], nvir, float(beta), n, bases, scales, strides, masks,
                     L.stream_ptr()))
    return r3


def full_strides(no, nv):
    """Strides (x,y,z,a,b,c) of a full ordered-triple tensor laid out [x][y][z][a][b][c]."""
    n3 = nv ** 3
    return (no * no * n3, no * n3, n3, nv * nv, nv, 1)


class T3Residual:
    """compute_r3_tri for all canonical blocks of one rank."""

    def __init__(self, nocc, nvir, precision="fp64", device="cuda", with_oo=True):
        self.no, self.nv, self.precision = int(nocc), int(nvir), precision
        no, nv = self.no, self.nv
        self.n3 = no * (no + 1) * (no + 2) // 6
        self.dev = device
        self.with_oo = with_oo
        if with_oo:
            self.U = torch.empty((no ** 3, nv, nv, nv), dtype=f64, device=device)  # every ordered (x,y,z)
            self.Z = torch.empty_like(self.U)
            trip = [(x, y, z) for x in range(no) for y in range(no) for z in range(no)]
            self.all_xyz = torch.tensor(trip, dtype=torch.int32, device=device)
            self.loc = torch.arange(self.n3, dtype=torch.int64, device=device)
        self.X = torch.empty((no * nv * nv, no * no * nv), dtype=f64, device=device)  # [(j,a,b),(i,k,c)]
        self.Y = (torch.empty((no * no * nv, no * nv * nv), dtype=f64, device=device)  # [(i,j,a),(k,b,c)]
                  if precision == "fp64" else None)
        N = no * no * nv
        self.x_strides = (no * nv, nv * nv * N, nv, nv * N, N, 1)
        Ny = no * nv * nv
        self.y_strides = (no * nv * Ny, nv * Ny, nv * nv, Ny, nv, 1)
        if precision != "fp64":
            k = contract.KIND[precision]
            self.kind = k
            self.xa = contract.Split(no * nv * nv, nv, k, device)
            self.xb = contract.Split(no * no * nv, nv, k, device)
            self.ya = contract.Split(no * no * nv, no, k, device)
            self.yb = contract.Split(no * nv * nv, no, k, device)
            self.wvvvv = contract.WvvvvT3(self.n3, nv, precision, device)
            self.status = torch.zeros(1, dtype=torch.int32, device=device)
            if with_oo:
                K = no * nv
                self.oa = contract.Split(no * nv, K, k, device)           # W side, rows (i,x), K (l,d)
                self.ob = contract.Split(no * no * nv * nv, K, k, device)  # U side, rows (jk,y,z), K (l,d)

    # ------------------------------------------------------------ pieces
    def vt2_(self, d):
        """X such that the twelve W_vvvo.t2 / W_vooo.t2 strings are sum_{p in S3} X[p(ijk)][p(abc)].

        X[(j,a,b),(i,k,c)] = sum_d W_vvvo[a,b,d,j] t2[i,k,d,c] is formed first;
        Y[ijk][abc] = sum_l W_vooo[a,l,i,j] t2[l,k,b,c] is then subtracted in X's layout."""
        no, nv = self.no, self.nv
        N = no * no * nv
        if self.precision == "fp64":
            Wt = d.W_vvvo.permute(3, 0, 1, 2).reshape(no * nv * nv, nv)
            T2m = d.t2.permute(0, 1, 3, 2).reshape(no * no * nv, nv)
            torch.matmul(Wt, T2m.t(), out=self.X)
            A = d.W_vooo.permute(2, 3, 0, 1).reshape(no * no * nv, no)
            Bm = d.t2.permute(1, 2, 3, 0).reshape(no * nv * nv, no)
            torch.matmul(A, Bm.t(), out=self.Y)
            # X[j,a,b,i,k,c] -= Y[i,j,a,k,b,c]
            self.X.view(no, nv, nv, no, no, nv).sub_(self.Y.view(no, no, nv, no, nv, nv).permute(1, 2, 4, 0, 3, 5))
        else:
            c = contract
            self.xa.fill(d.W_vvvo, c.two(nv * nv, 1, nv * no), c.lin(no))
            self.xb.fill(d.t2, c.two(nv, nv * nv, 1), c.lin(nv))
            c.gemm_(self.xa, self.xb, self.X, c.lin(N), c.lin(1), 1.0, 0.0, self.status)
            # Y rows (i,j,a) from W_vooo[a,l,i,j], cols (k,b,c) from t2[l,k,b,c], K = l;
            # accumulated with alpha = -1 straight into X[(j,a,b),(i,k,c)]
            self.ya.fill(d.W_vooo, c.three(no, nv, no, 1, no ** 3), c.lin(no * no))
            self.yb.fill(d.t2, c.lin(1), c.lin(no * nv * nv))
            c.gemm_(self.ya, self.yb, self.X, c.three(no, nv, no * nv, nv * nv * N, nv * N),
                    c.three(nv, nv, nv, N, 1), -1.0, 1.0, self.status)
        return self.X

    # ------------------------------------------------------------ OO batch terms
    def oo_(self, d, t3):
        """Z[ijk][abc] over every ordered (i,j,k) such that the OO batch terms of
        compute_r3_tri (distr_cc/rccsdt.py:435-732) are sum_{p in OO_SET} Z[p(ijk)][p(abc)].

        With U the unpacked t3 of every ordered triple,
          Z = - sum Wov[l,b,i,d] U[jkl][d,c,a] + sum G2[l,a,i,d] (U[jkl][d,c,b] + U[jkl][b,d,c])
              - sum Wov[l,c,i,d] U[jkl][b,d,a] + sum Wvo[l,a,d,i] U[jkl][b,c,d]
              + sum W_oooo[l,m,j,k] U[lmi][b,c,a] - sum F_oo[l,i] U[ljk][a,b,c],
          G2[l,a,i,d] = -(Wov[l,a,i,d] + Wvo[l,a,d,i]) / 2,
        Wov = W_ovov, Wvo = W_ovvo (sums over l and d, or l and m)."""
        no, nv = self.no, self.nv
        n3v = nv ** 3
        _c_rccsdt.take_t3_batched(t3, self.U, self.all_xyz, self.loc, no, nv)
        U, Z = self.U, self.Z
        G2 = (-0.5 * (d.W_ovov + d.W_ovvo.permute(0, 1, 3, 2))).permute(2, 1, 0, 3).contiguous()  # [i][x][l][d]
        if self.precision == "fp64":
            Zv = Z.view(no, no, no, nv, nv, nv)
            e = torch.einsum
            Zv.copy_(-e('lbid,jkldca->ijkabc', d.W_ovov, U.view(no, no, no, nv, nv, nv)))
            Zv.add_(e('iald,jkldcb->ijkabc', G2, U.view(no, no, no, nv, nv, nv)))
            Zv.add_(e('iald,jklbdc->ijkabc', G2, U.view(no, no, no, nv, nv, nv)))
            Zv.sub_(e('lcid,jklbda->ijkabc', d.W_ovov, U.view(no, no, no, nv, nv, nv)))
            Zv.add_(e('ladi,jklbcd->ijkabc', d.W_ovvo, U.view(no, no, no, nv, nv, nv)))
        else:
            c = contract
            Zrow = lambda xs: c.two(nv, no * no * n3v, xs)  # noqa: E731  (i, x): x placed at stride xs
            Zcol = lambda ys, zs: c.three(nv, nv, n3v, ys, zs)  # noqa: E731  (jk, y, z)
            wov_rows, wov_k = c.two(nv, nv, no * nv), c.two(nv, nv * no * nv, 1)   # Wov[l,x,i,d]
            g2_rows, g2_k = c.lin(no * nv), c.lin(1)                              # G2[i][x][l][d]
            wvo_rows, wvo_k = c.two(nv, 1, nv * no), c.two(nv, nv * nv * no, no)  # Wvo[l,x,d,i]
            urow = lambda ys, zs: c.three(nv, nv, no * n3v, ys, zs)  # noqa: E731  U[j,k,.] rows (jk, y, z)
            st = self.status
            # U[jkl][d, y, z]
            self.ob.fill(U, urow(nv, 1), c.two(nv, n3v, nv * nv))
            self.oa.fill(d.W_ovov, wov_rows, wov_k)
            c.gemm_(self.oa, self.ob, Z, Zrow(nv), Zcol(1, nv * nv), -1.0, 0.0, st)       # a=z, b=x, c=y
            self.oa.fill(G2, g2_rows, g2_k)
            c.gemm_(self.oa, self.ob, Z, Zrow(nv * nv), Zcol(1, nv), 1.0, 1.0, st)         # a=x, b=z, c=y
            # U[jkl][y, d, z]
            self.ob.fill(U, urow(nv * nv, 1), c.two(nv, n3v, nv))
            c.gemm_(self.oa, self.ob, Z, Zrow(nv * nv), Zcol(nv, 1), 1.0, 1.0, st)         # a=x, b=y, c=z
            self.oa.fill(d.W_ovov, wov_rows, wov_k)
            c.gemm_(self.oa, self.ob, Z, Zrow(1), Zcol(nv, nv * nv), -1.0, 1.0, st)        # a=z, b=y, c=x
            # U[jkl][y, z, d]
            self.ob.fill(U, urow(nv * nv, nv), c.two(nv, n3v, 1))
            self.oa.fill(d.W_ovvo, wvo_rows, wvo_k)
            c.gemm_(self.oa, self.ob, Z, Zrow(nv * nv), Zcol(nv, 1), 1.0, 1.0, st)         # a=x, b=y, c=z
        # W_oooo and F_oo pieces: bandwidth-bound, FP64 in both precisions
        Zv = Z.view(no, no, no, nv, nv, nv)
        G = torch.matmul(d.W_oooo.reshape(no * no, no * no).t(), U.view(no * no, no * n3v))  # [(j,k),(i,b,c,a)]
        Zv.add_(G.view(no, no, no, nv, nv, nv).permute(2, 0, 1, 5, 3, 4))
        Z.view(no, -1).sub_(torch.matmul(d.F_oo.t(), U.view(no, -1)))
        return Z

    def fvv_(self, r3, d, t3):
        """F_vv.t3 (distr_cc/rccsdt.py:400-402), FP64 in both precisions (bandwidth-bound)."""
        n, nv = t3.shape[0], self.nv
        F = d.F_vv
        r3.view(n, nv, nv * nv).add_(torch.matmul(F, t3.view(n, nv, nv * nv)))
        r3.view(n * nv, nv, nv).add_(torch.matmul(F, t3.view(n * nv, nv, nv)))
        r3.view(n * nv * nv, nv).add_(torch.matmul(t3.view(n * nv * nv, nv), F.t()))
        return r3

    def wvvvv_(self, r3, d, t3):
        if self.precision == "fp64":
            return contract.wvvvv_t3_fp64_(r3, d.W_vvvv, t3)
        return self.wvvvv(r3, d.W_vvvv, t3)

    def compute(self, d, t3, r3=None):
        """r3 = compute_r3_tri for canonical t3 (the OO batch terms included when with_oo)."""
        if r3 is None:
            r3 = torch.empty_like(t3)
        nv = self.nv
        X = self.vt2_(d)
        src = [(X, 1.0, self.x_strides, ALL_S3)]
        if self.with_oo:
            Z = self.oo_(d, t3)
            src.append((Z, 1.0, full_strides(self.no, nv), OO_SET))
        perm_gather_(r3, d.ijk, nv, 0.0, src)
        self.fvv_(r3, d, t3)
        self.wvvvv_(r3, d, t3)
        return r3

    def status_ok(self):
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
