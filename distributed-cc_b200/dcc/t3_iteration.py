"""The T3 half of one RCCSDT iteration on one GPU, with T3 resident in HBM.

The reference runs these steps of update_amps_rccsdt_tri_ and its caller
(distr_cc/rccsdt.py) on every rank's host memory:

  r1r2_add_t3_tri_             :916   T3 -> r1, r2
  intermediates_t3_add_t3_tri  :936   T3 -> W_vooo, W_vvvo
  compute_r3_tri               :941   the T3 residual (OO batch included)
  P3_full, r3_tri_divide_e_,
  norms, t3_local += r3        :947-971
  run_diis_t3                  :1026-1067 (unified T1/T2/T3 DIIS)

Here every one of them is a device step over the same resident T3.  The two
feedback passes share one X = P3_201 of every ordered block (t3 does not
change between them, distr_cc/rccsdt.py:916-936), built in the residual's S
buffer from the residual's unpacked U (the unpack is done once per
iteration).  In the split precisions the feedback strings are tcgen05 GEMMs
over X read in place (t3_feedback.SplitFeedback); the FP64 path runs them as
DGEMMs one occupied slice at a time.
The lower-order steps between the passes (PySCF's compute_r1r2,
intermediates_t3, the r1/r2 update) stay with the caller: they are small
and are not on this path.
"""
from __future__ import annotations

import torch

from . import t3_feedback as fb
from .diis import DIIS
from .synthetic import canonical_ijk
from .t3_residual import T3Residual, update_t3_

f64 = torch.float64


class T3Iteration:
    """Device state of the T3 half-iteration for one (nocc, nvir, precision)."""

    def __init__(self, nocc, nvir, precision="bf16x3", device="cuda", woooo_pair_symmetric=False):
        self.no, self.nv, self.precision, self.dev = int(nocc), int(nvir), precision, device
        self.res = T3Residual(nocc, nvir, precision, device, with_oo=True,
                              woooo_pair_symmetric=woooo_pair_symmetric)
        self.n3 = self.res.n3
        self.ijk = torch.tensor(canonical_ijk(self.no), dtype=torch.int32, device=device)
        self.r3 = torch.empty((self.n3, nvir, nvir, nvir), dtype=f64, device=device)
        self.norms = torch.zeros(2, dtype=f64, device=device)
        self._X = None
        self._dW = None
        # the feedback strings as split GEMMs in the split precisions (FP64 einsums otherwise)
        self.sfb = fb.SplitFeedback(nocc, nvir, precision, device) if precision != "fp64" else None
        self.diis = None
        self._diis_key = None
        self._active = None

    # --------------------------------------------------------------- feedback
    def feedback_r1r2(self, t3, fock_ov, oovv, vovv, ooov):
        """(dr1, dr2): the T3 parts of r1 and r2 (distr_cc/rccsdt.py:253-321) on the device.
        Unpacks t3 into the residual's U and builds X in its S buffer for feedback_w."""
        no, nv = self.no, self.nv
        dr1 = torch.zeros((no, nv), dtype=f64, device=self.dev)
        dr2 = torch.zeros((no, no, nv, nv), dtype=f64, device=self.dev)
        fb.r1_add_t3_(dr1, None, t3, self.ijk, no, oovv=oovv, V=self.r3)
        # the unpack, then X = P3_201(U) (two passes: the one-pass dcc_t3_unpack_p3 measured
        # 53.6 ms against 8.0 + 8.5 ms at nocc=15 / nvir=93)
        self.res.unpack_(t3)
        self._X = fb.p3_201_all(t3, no, U=self.res.U, out=self.res.S)
        if self.sfb is None:
            fb.r2_add_t3_x_(dr2, fock_ov, vovv, ooov, self._X)
        else:
            # all four strings here, two splits of X between them; the W parts wait in dW for
            # feedback_w (the host builds W_vooo / W_vvvo in between)
            dr2.view(no * no, nv * nv).add_(self._fock_term(fock_ov), alpha=0.5)
            self._dW = (torch.zeros((nv, no, no, no), dtype=f64, device=self.dev),
                        torch.zeros((nv, nv, nv, no), dtype=f64, device=self.dev))
            self.sfb.run(self._X, {"vovv": vovv, "ooov": ooov, "oovv": oovv},
                         {"r2": dr2, "W_vooo": self._dW[0], "W_vvvo": self._dW[1]})
        return dr1, dr2

    def _fock_term(self, fock_ov):
        """sum_{x,a} f[x,a] X[x,y,z,a,b,c] as [(y,z), (b,c)], summed over x in FP64 (each x's
        product in X's type)."""
        no, nv = self.no, self.nv
        out = torch.zeros((no * no, nv * nv), dtype=f64, device=self.dev)
        f = fock_ov.to(self._X.dtype)
        for x in range(no):
            out += torch.matmul(f[x].view(1, 1, nv), self._X[x].reshape(no * no, nv, nv * nv)).view(no * no, nv * nv)
        return out

    def feedback_w(self, W_vooo, W_vvvo, oovv):
        """W_vooo, W_vvvo += their T3 parts (distr_cc/rccsdt.py:323-366), in place, from the X of
        the preceding feedback_r1r2 (same T3)."""
        if self._X is None:
            raise RuntimeError("feedback_w needs the X of feedback_r1r2 of the same T3")
        if self.sfb is None:
            fb.intermediates_t3_add_x_(W_vooo, W_vvvo, oovv, self._X)
        elif self._dW is not None:
            W_vooo += self._dW[0]
            W_vvvo += self._dW[1]
            self._dW = None
        else:  # X built without feedback_r1r2 (the route of intermediates_t3_add_t3_tri alone)
            self.sfb.run(self._X, {"oovv": oovv}, {"W_vooo": W_vooo, "W_vvvo": W_vvvo}, names=("wvooo", "wvvvo"))
        return W_vooo, W_vvvo

    # --------------------------------------------------------------- residual + update
    def residual(self, d, t3, wvvvv_ready=None, inputs_ready=None):
        """r3 = compute_r3_tri (distr_cc/rccsdt.py:368-732) into the iteration's r3 buffer; the
        U unpacked by feedback_r1r2 is reused (X in S is overwritten)."""
        unpacked = self._X is not None
        self._X = None
        r3 = self.res.compute(d, t3, self.r3, wvvvv_ready=wvvvv_ready, inputs_ready=inputs_ready,
                              unpacked=unpacked)
        return r3

    def update(self, t3, eia, nvir_active=None):
        """P3_full (-1/6, 1), divide by the denominators, norms, t3 += r3
        (distr_cc/rccsdt.py:947-971).  Returns the device norms [|r3|^2, |r3_active|^2].
        The divided r3 is not stored back (the reference drops r3 after t3 += r3; the buffer is
        the next iteration's scratch), which saves one pass of writes over r3."""
        d = _Eia(eia, self.ijk)
        return update_t3_(t3, self.r3, d, nvir_active=nvir_active, norms=self.norms, write_r3=False)

    def status_ok(self):
        ok = self.res.status_ok()
        if self.sfb is not None:
            ok = ok and int(self.sfb.status.item()) == 0
        return ok

    # --------------------------------------------------------------- DIIS
    def diis_update(self, lower, t3, space, key=None, nvir_diis=None):
        """One unified DIIS step (distr_cc/rccsdt.py:1026-1067, distr_cc/diis.py:105-177) over the
        vector [lower | t3[:, :nd, :nd, :nd]], in place: `lower` is the packed, scaled unique
        T1/T2 (a device vector), t3 the resident T3.  `key` identifies the caller's DIIS
        object: a new key starts a new history.  Returns last_delta_norm_sq (None on the
        first call, which only records the vector)."""
        if self.diis is None or self._diis_key is not key or self.diis.space != int(space):
            self.diis = DIIS(space, self.dev)
            self._diis_key = key
        nd = self.nv if nvir_diis is None else min(int(nvir_diis), self.nv)
        if nd < self.nv:
            if self._active is None or self._active.shape[1] != nd:
                self._active = torch.empty((self.n3, nd, nd, nd), dtype=f64, device=self.dev)
            self._active.copy_(t3[:, :nd, :nd, :nd])
            self.diis.update([lower, self._active])
            t3[:, :nd, :nd, :nd].copy_(self._active)
        else:
            self.diis.update([lower, t3])
        return self.diis.last_delta_norm_sq


class _Eia:
    def __init__(self, eia, ijk):
        self.eia, self.ijk = eia, ijk
