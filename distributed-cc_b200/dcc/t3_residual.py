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
  so they are two GEMMs and one gather (dcc_t3_s3_gather).
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
    L.check(_gather(L.ptr(r3), L.ptr(ijk), r3.shape[0], nvir, float(beta), L.ptr(u0), float(scale0),
                    _strides(strides0), L.ptr(u1) if u1 is not None else L.c_vp(None), float(scale1),
                    _strides(strides1) if strides1 is not None else None, L.stream_ptr()))
    return r3


class T3Residual:
    """compute_r3_tri for all canonical blocks of one rank (OO batch terms excluded
    unless with_oo; see oo_terms)."""

    def __init__(self, nocc, nvir, precision="fp64", device="cuda"):
        self.no, self.nv, self.precision = int(nocc), int(nvir), precision
        no, nv = self.no, self.nv
        self.n3 = no * (no + 1) * (no + 2) // 6
        self.dev = device
        self.X = torch.empty((no * nv * nv, no * no * nv), dtype=f64, device=device)  # [(j,a,b),(i,k,c)]
        self.Y = torch.empty((no * no * nv, no * nv * nv), dtype=f64, device=device)  # [(i,j,a),(k,b,c)]
        N = no * no * nv
        self.x_strides = (no * nv, nv * nv * N, nv, nv * N, N, 1)
        Ny = no * nv * nv
        self.y_strides = (no * nv * Ny, nv * Ny, nv * nv, Ny, nv, 1)
        if precision != "fp64":
            k = contract.KIND[precision]
            self.kind = k
            self.xa = contract.Split(no * nv * nv, nv, k, device)
            self.xb = contract.Split(no * no * nv, nv, k, device)
            self.wvvvv = contract.WvvvvT3(self.n3, nv, precision, device)
            self.status = torch.zeros(1, dtype=torch.int32, device=device)

    # ------------------------------------------------------------ pieces
    def vt2_(self, r3, d):
        """r3 = W_vvvo.t2 - W_vooo.t2 (12 strings), overwriting r3."""
        no, nv = self.no, self.nv
        if self.precision == "fp64":
            Wt = d.W_vvvo.permute(3, 0, 1, 2).reshape(no * nv * nv, nv)
            T2m = d.t2.permute(0, 1, 3, 2).reshape(no * no * nv, nv)
            torch.matmul(Wt, T2m.t(), out=self.X)
        else:
            B = contract.BIG
            self.xa.fill(d.W_vvvo, (nv * nv, 1, nv * no, B, 0, no))
            self.xb.fill(d.t2, (nv, nv * nv, 1, B, 0, nv))
            contract.gemm_(self.xa, self.xb, self.X, (B, 0, self.X.shape[1], B, 0, 1), 1.0, 0.0, self.status)
        A = d.W_vooo.permute(2, 3, 0, 1).reshape(no * no * nv, no)
        Bm = d.t2.permute(1, 2, 3, 0).reshape(no * nv * nv, no)
        torch.matmul(A, Bm.t(), out=self.Y)
        s3_gather_(r3, d.ijk, nv, 0.0, self.X, 1.0, self.x_strides, self.Y, -1.0, self.y_strides)
        return r3

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
        """r3 = compute_r3_tri (without the OO batch terms) for canonical t3."""
        if r3 is None:
            r3 = torch.empty_like(t3)
        self.vt2_(r3, d)
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
