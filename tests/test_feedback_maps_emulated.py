"""The split-precision T3 feedback plan (dcc.t3_feedback.SplitFeedback) on the CPU:
every operand split (row / contraction maps, the permuted E slices, one piece per
value of the contracted occupied index) and every per-piece GEMM with its epilogue
map emulated in numpy FP64, against the FP64 feedback strings
(distr_cc/rccsdt.py:300-316, 340-358).  Relative 1e-12."""
import numpy as np
import pytest
import torch

from dcc import contract, t3_feedback as fb
from test_maps_emulated import fmap


class _EmuSplit:
    """contract.Split with the two pieces replaced by one FP64 array (same maps, same pieces)."""

    def __init__(self, M, K=None, kind=0, device="cpu", buffers=None, pieces=None, align=8):
        ref = contract.Split(M, K, kind, device="meta", pieces=pieces, align=align)
        self.M, self.K, self.Kp, self.pieces, self.kind = ref.M, ref.K, ref.Kp, ref.pieces, kind
        self.a = np.zeros((self.M, self.Kp))

    def fill_piece(self, i, src, fm, fk):
        off, k, _ = self.pieces[i]
        # read through the maps from src's first element, over its storage
        st = src.untyped_storage()
        n = st.nbytes() // 8 - src.storage_offset()
        buf = torch.empty(0, dtype=torch.float64).set_(st, src.storage_offset(), (n,), (1,)).numpy()
        idx = fmap(fm, np.arange(self.M))[:, None] + fmap(fk, np.arange(k))[None, :]
        self.a[:, off:off + k] = buf[idx]
        return self

    def fill(self, src, fm, fk):
        return self.fill_piece(0, src, fm, fk)


def _emu_gemm(A, B, C, frow, fcol, alpha=1.0, beta=1.0, status=None, Kp=None):
    idx = fmap(frow, np.arange(A.M))[:, None] + fmap(fcol, np.arange(B.M))[None, :]
    assert len(np.unique(idx)) == idx.size
    flat = C.view(-1).numpy()
    # beta = 0 overwrites without reading C (BLAS semantics, as the kernel's epilogue)
    flat[idx] = alpha * (A.a @ B.a.T) + (beta * flat[idx] if beta != 0.0 else 0.0)
    return status


def _emu_gemm_range(A, B, C, frow, fcol, alpha, beta, status, col0, ncol):
    assert col0 % 64 == 0 and ncol % 64 == 0
    idx = fmap(frow, np.arange(A.M))[:, None] + fmap(fcol, np.arange(B.M))[None, :]
    flat = C.view(-1).numpy()
    flat[idx] = alpha * (A.a[:, col0:col0 + ncol] @ B.a[:, col0:col0 + ncol].T) + \
        (beta * flat[idx] if beta != 0.0 else 0.0)
    return status


class _EmuContract:
    KIND, padded_k, lin, three, _KBLK = contract.KIND, staticmethod(contract.padded_k), \
        staticmethod(contract.lin), staticmethod(contract.three), contract._KBLK
    Split = _EmuSplit
    gemm_ = staticmethod(_emu_gemm)
    gemm_range_ = staticmethod(_emu_gemm_range)


@pytest.mark.parametrize("no,nv", [(3, 5), (4, 6), (5, 4)])
def test_split_feedback_maps(no, nv):
    rng = np.random.default_rng(no * nv)
    nmo = no + nv
    g = torch.from_numpy(rng.standard_normal((nmo,) * 4))
    X = torch.from_numpy(rng.standard_normal((no, no, no, nv, nv, nv)))
    sl = {k: v.contiguous() for k, v in fb.eris_slices(g, None, no).items()}
    sfb = fb.SplitFeedback(no, nv, "bf16x3", device="cpu")
    assert all(len(p[0]) == no for p in sfb.plans.values())  # one piece per x
    sfb.c = _EmuContract
    r2 = torch.zeros(no, no, nv, nv, dtype=torch.float64)
    Wo = torch.zeros(nv, no, no, no, dtype=torch.float64)
    Wv = torch.zeros(nv, nv, nv, no, dtype=torch.float64)
    sfb.run(X, sl, {"r2": r2, "W_vooo": Wo, "W_vvvo": Wv})
    e = torch.einsum
    o, v = slice(0, no), slice(no, None)
    want_r2 = e('cxad,xyzdba->yzbc', g[v, o, v, v], X) - e('zxla,xyzabc->ylbc', g[o, o, o, v], X)
    E = g[o, o, v, v]
    want_wo = e('mxde,xyzead->amyz', E, X)
    want_wv = -e('zxde,xyzeba->abdy', E, X)
    for got, want in ((r2, want_r2), (Wo, want_wo), (Wv, want_wv)):
        np.testing.assert_allclose(got.numpy(), want.numpy(), rtol=0, atol=1e-12 * want.abs().max().item())
